"""CPU oracle for the fdfault time-stepping path -- TEST INFRASTRUCTURE ONLY.

``Oracle`` wraps ``oracle/liboracle.so``, the C restatement of the reference
solver's per-stage update (fdf_oracle.c).  ``run_reference`` runs the
unmodified reference solver binary ``oracle/_ref/fdfault_ref`` (compiled from
the reference's own sources by ``oracle/Makefile``) on a problem file and
reads back its output units.  Only the test suite, the smoke check and the
CPU-baseline leg of bench.py use this package, always as the checker.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "fdfault_ref")

F, DF, X, METRIC, JAC, S = range(6)
U, DU, V, SS, SN, UX, DUX, VX, SX, STATE, DSTATE, DSTATEDT, TFRONT = range(13)

_lib = None


def reference_dir() -> str:
    """The fdfault reference checkout: $FDFAULT_REFERENCE, else the directory
    ``reference`` beside this repository (it may not exist, e.g. on machines
    that only run the tests against the committed fixtures)."""
    env = os.environ.get("FDFAULT_REFERENCE")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, os.pardir, os.pardir, "reference"))


def build(ref_src: Optional[str] = None, quiet: bool = True) -> None:
    """Compile the oracle port, and the reference binary when its sources
    exist (ref_src: the reference's src directory, default under reference_dir())."""
    if ref_src is None:
        ref_src = os.path.join(reference_dir(), "src")
    out = subprocess.DEVNULL if quiet else None
    subprocess.check_call(["make", "-C", HERE, "port"], stdout=out)
    if ref_src and os.path.isdir(ref_src):
        subprocess.check_call(["make", "-C", HERE, "ref", "REFSRC=" + ref_src, "-j8"], stdout=out)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref_src=None)
        L = ctypes.CDLL(LIB_PATH)
        L.orc_load.restype = ctypes.c_void_p
        L.orc_load.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int]
        L.orc_free.argtypes = [ctypes.c_void_p]
        L.orc_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
        L.orc_field.restype = ctypes.POINTER(ctypes.c_double)
        L.orc_field.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_fault.restype = ctypes.POINTER(ctypes.c_double)
        L.orc_fault.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                ctypes.POINTER(ctypes.c_int)]
        L.orc_iface_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.orc_do_rk_stage.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_double]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_set_stress.argtypes = [ctypes.c_void_p]
        L.orc_remove_stress.argtypes = [ctypes.c_void_p]
        L.orc_abs_field.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_last_error.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


class Oracle:
    """One problem held by the C oracle (single process, FP64)."""

    def __init__(self, infile: str):
        L = lib()
        err = ctypes.create_string_buffer(2048)
        self._p = L.orc_load(infile.encode(), err, 2048)
        if not self._p:
            raise RuntimeError("oracle failed to load %s: %s" % (infile, err.value.decode()))
        ints = (ctypes.c_int * 16)()
        dbls = (ctypes.c_double * 3)()
        L.orc_info(self._p, ints, dbls)
        (self.ndim, self.mode, nx, ny, nz, self.nfields, self.nfieldsp, self.nifaces, self.nstages, self.nt,
         self.sbporder, nb0, nb1, nb2, plastic, self.rkorder) = list(ints)
        self.nx = (nx, ny, nz)
        self.nblocks = (nb0, nb1, nb2)
        self.is_plastic = bool(plastic)
        self.dt, self.ttot, self.cfl = list(dbls)
        self.nxyz = nx * ny * nz
        self.step_index = 0

    def close(self) -> None:
        if self._p:
            lib().orc_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, which: int = F) -> np.ndarray:
        """Live view of a whole field array (components stacked, reference layout)."""
        n = {F: self.nfields + self.nfieldsp, DF: self.nfields, X: self.ndim, METRIC: self.ndim * self.ndim,
             JAC: 1, S: 6}[which]
        ptr = lib().orc_field(self._p, which)
        if not ptr:
            return None
        return np.ctypeslib.as_array(ptr, shape=(n, self.nxyz))

    def abs_field(self, comp: int) -> np.ndarray:
        out = np.empty(self.nxyz)
        lib().orc_abs_field(self._p, comp, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def fault(self, iface: int, which: int) -> Optional[np.ndarray]:
        n0, n1 = ctypes.c_int(), ctypes.c_int()
        ptr = lib().orc_fault(self._p, iface, which, ctypes.byref(n0), ctypes.byref(n1))
        if not ptr:
            return None
        n = n0.value * n1.value
        if which in (UX, DUX, VX, SX):
            n *= self.ndim - 1
        return np.ctypeslib.as_array(ptr, shape=(n,))

    def iface_info(self, iface: int) -> dict:
        ints = (ctypes.c_int * 13)()
        lib().orc_iface_info(self._p, iface, ints)
        v = list(ints)
        return {"kind": v[0], "direction": v[1], "n": (v[2], v[3]), "mlb": tuple(v[4:7]),
                "xm": tuple(v[7:10]), "xp": tuple(v[10:13])}

    def do_rk_stage(self, dt: float, stage: int, t: float) -> None:
        rc = lib().orc_do_rk_stage(self._p, dt, stage, t)
        if rc:
            raise RuntimeError(lib().orc_last_error(self._p).decode())

    def step(self) -> None:
        rc = lib().orc_step(self._p, self.step_index)
        if rc:
            raise RuntimeError(lib().orc_last_error(self._p).decode())
        self.step_index += 1

    def run(self, nsteps: int) -> None:
        rc = lib().orc_run(self._p, self.step_index, nsteps)
        if rc:
            raise RuntimeError(lib().orc_last_error(self._p).decode())
        self.step_index += nsteps


def run_reference(infile: str, workdir: str, timeout: float = 600.0,
                  timing_file: Optional[str] = None) -> subprocess.CompletedProcess:
    """Run the reference solver binary on ``infile`` from ``workdir``."""
    if not os.path.exists(REF_BIN):
        raise FileNotFoundError(REF_BIN)
    env = dict(os.environ)
    if timing_file:
        env["FDF_REF_TIMING"] = timing_file
    return subprocess.run([REF_BIN, infile], cwd=workdir, env=env, capture_output=True, text=True,
                          timeout=timeout, check=True)


def read_unit(datadir: str, probname: str, unit: str, field: str) -> Dict[str, np.ndarray]:
    """Read one output unit written by the reference (outputunit.cpp file layout)."""
    meta: Dict[str, object] = {}
    with open(os.path.join(datadir, "%s_%s.py" % (probname, unit))) as fh:
        exec(fh.read(), {}, meta)
    nt, nx, ny, nz = int(meta["nt"]), int(meta["nx"]), int(meta["ny"]), int(meta["nz"])
    data = np.fromfile(os.path.join(datadir, "%s_%s_%s.dat" % (probname, unit, field)), dtype="<f8")
    out = {"data": data.reshape(nt, nx, ny, nz)}
    tfile = os.path.join(datadir, "%s_%s_t.dat" % (probname, unit))
    if os.path.exists(tfile):
        out["t"] = np.fromfile(tfile, dtype="<f8")
    return out
