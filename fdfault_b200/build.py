"""Build recipe for libfdfault_b200.so and the fdfault_b200 command-line driver.

Device code is compiled for sm_100a only.  Files whose FP64 arithmetic must
round exactly as the reference's x86-64 build does (geometry set-up, the
exact-order stage kernel, the interface/friction kernel) are compiled with
``-fmad=false`` so no multiply-add is contracted; host code is compiled with
``-ffp-contract=off`` for the same reason.  The tiled FP32 kernel keeps FMA
contraction.  Outputs are written next to this file (in-tree).
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfdfault_b200.so")
EXE = os.path.join(HERE, "fdfault_b200")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

EXACT_CU = ["geometry.cu", "stage_exact.cu", "iface.cu", "noalloc.cu", "ensemble.cu", "energy.cu"]
FAST_CU = ["stage_fast.cu", "stage_fast2d.cu", "stage_tma.cu", "stage_reg.cu", "mlp.cu", "slab.cu"]
HOST_CPP = ["input.cpp", "solver.cpp", "output.cpp", "api.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _newer(out, deps):
    if not os.path.exists(out):
        return False
    t = os.path.getmtime(out)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "fdfault_b200.h"))
    jobs = []
    common_nv = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", CSRC] + ARCH
    for f in EXACT_CU:
        jobs.append((f, [NVCC, "-c", "-fmad=false", "-prec-div=true", "-prec-sqrt=true"] + common_nv))
    for f in FAST_CU:
        jobs.append((f, [NVCC, "-c", "-Xptxas", "-v"] + common_nv))
    for f in HOST_CPP:
        jobs.append((f, ["g++", "-c", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-I", CSRC,
                         "-I", os.path.join(CUDA_HOME, "include")]))
    objs = []

    def compile_one(job):
        f, base = job
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f + ".o")
        if force or not _newer(obj, [src] + headers):
            r = _run(base + ["-o", obj, src])
            if verbose and (r.stderr or r.stdout):
                sys.stdout.write(r.stdout + r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=8) as ex:
        objs = list(ex.map(compile_one, jobs))
    if force or not _newer(LIB, objs):
        _run([NVCC, "-shared", "-o", LIB] + objs + ARCH + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    main_obj = os.path.join(BUILD, "main.o")
    src = os.path.join(CSRC, "main.cpp")
    if force or not _newer(main_obj, [src] + headers):
        _run(["g++", "-c", "-O2", "-std=c++17", "-o", main_obj, src])
    if force or not _newer(EXE, [main_obj, LIB]):
        _run(["g++", "-o", EXE, main_obj, "-L", HERE, "-lfdfault_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


def clean() -> None:
    shutil.rmtree(BUILD, ignore_errors=True)
    for p in (LIB, EXE):
        if os.path.exists(p):
            os.remove(p)


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose=True, force="--force" in sys.argv))
