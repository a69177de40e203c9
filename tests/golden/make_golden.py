"""Regenerate the golden fixtures from the reference solver.

For every case in tests/cases.py this writes the problem (with its output
units and front), runs the unmodified fdfault reference solver built by
``make -C oracle ref`` (oracle/_ref/fdfault_ref), and stores every output unit
and the rupture front as arrays in tests/golden/<case>.npz.  Requires the
reference sources (to build the binary); the fixtures it writes are what the
tests read on machines without them.

    python tests/golden/make_golden.py [case ...]
    python tests/golden/make_golden.py --files   # output_files.npz (below)

``--files`` stores, for the cases in FILE_CASES, the bytes of every file the
reference writes for its output units and fronts (data, time, coordinate and
.m/.py metadata files) in tests/golden/output_files.npz, keyed "case/file".
"""

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from cases import CASES, build_case  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def read_outputs(prob, datadir):
    out = {}
    for o in prob.outputs:
        u = oracle.read_unit(datadir, prob.name, o.name, o.field)
        out["unit/" + o.name] = u["data"]
        if "t" in u:
            out["t/" + o.name] = u["t"]
    for n, itf in enumerate(prob.interfaces):
        fn = os.path.join(datadir, "%s_front_%d_t.dat" % (prob.name, n))
        if os.path.exists(fn):
            out["front/%d" % n] = np.fromfile(fn, dtype="<f8")
    return out


FILE_CASES = ["m2_sw", "p3_sw", "m2_curve"]


def main_files():
    if not os.path.exists(oracle.REF_BIN):
        oracle.build()
    arrays = {}
    for name in FILE_CASES:
        tmp = tempfile.mkdtemp(prefix="golden_files_")
        prob = build_case(name, tmp)
        infile = prob.write(os.path.join(tmp, prob.name + ".in"))
        oracle.run_reference(infile, tmp)
        for fn in sorted(os.listdir(tmp)):
            if fn.startswith(prob.name + "_"):
                with open(os.path.join(tmp, fn), "rb") as fh:
                    arrays["%s/%s" % (name, fn)] = np.frombuffer(fh.read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "output_files.npz"), **arrays)
    print(len(arrays), "files", sum(a.size for a in arrays.values()), "bytes")


def main(names):
    if not os.path.exists(oracle.REF_BIN):
        oracle.build()
    for name in names or sorted(CASES):
        tmp = tempfile.mkdtemp(prefix="golden_")
        prob = build_case(name, tmp)
        infile = prob.write(os.path.join(tmp, prob.name + ".in"))
        oracle.run_reference(infile, tmp)
        arrays = read_outputs(prob, tmp)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        print(name, sum(a.size for a in arrays.values()), "values")


if __name__ == "__main__":
    if sys.argv[1:] == ["--files"]:
        main_files()
    else:
        main(sys.argv[1:])
