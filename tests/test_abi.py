"""The C-ABI library loads and exports every entry point the header declares,
and its host-side input checks reject bad problems without touching a GPU."""

import ctypes
import os
import re

import pytest

from fdfault_b200 import problems as P
from fdfault_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fdfault_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdf_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ["fdf_create", "fdf_destroy", "fdf_do_rk_stage", "fdf_step", "fdf_solve", "fdf_get_field",
              "fdf_get_fault", "fdf_last_error"]:
        assert n in names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(solver.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_create_rejects_missing_file(tmp_path):
    L = solver.load_library()
    h = ctypes.c_void_p()
    rc = L.fdf_create(str(tmp_path / "nope.in").encode(), 0, 0, ctypes.byref(h))
    assert rc == -2
    assert b"input file" in L.fdf_last_error(None)


@pytest.mark.parametrize("mutate,message", [
    (lambda p: setattr(p, "sbporder", 5), b"sbporder"),
    (lambda p: setattr(p.interfaces[0], "kind", "bogus"), b"interface type"),
    (lambda p: setattr(p, "nx_block", ([61], [31, 10], [1])), b"too few points"),
    # the reference's time step would read a third material array mode III lacks
    (lambda p: (setattr(p, "mode", 3), setattr(p, "matfile", "m.mat")), b"mode III"),
])
def test_create_rejects_invalid_problem(tmp_path, mutate, message):
    p = P.mode2_rupture(nx=61, ny=31, nt=5, datadir=str(tmp_path) + "/")
    mutate(p)
    infile = p.write(str(tmp_path / "bad.in"))
    L = solver.load_library()
    h = ctypes.c_void_p()
    rc = L.fdf_create(infile.encode(), 0, 0, ctypes.byref(h))
    assert rc == -2
    assert message in L.fdf_last_error(None)


def test_null_handle_is_an_argument_error():
    L = solver.load_library()
    assert L.fdf_step(None, 1) == -1
    assert L.fdf_do_rk_stage(None, 0.1, 0, 0.0) == -1
    assert L.fdf_set_plastic_rule(None, 1) == -1
    assert L.fdf_get_fault_async(None, 0, 0, None) == -1
    # x-slab entry points
    assert L.fdf_step_stage(None, 0) == -1
    assert L.fdf_set_x_range(None, 0, 16) == -1
    assert L.fdf_pack_ghosts(None, 0, None) == -1
    assert L.fdf_unpack_ghosts(None, 1, None) == -1
    assert L.fdf_set_stream(None, 1, None) == -1
    g, n, e = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_int()
    assert L.fdf_ghost_info(None, ctypes.byref(g), ctypes.byref(n), ctypes.byref(e)) == -1
    lo, cnt = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
    assert L.fdf_get_block(None, 0, lo, cnt) == -1
    assert L.fdf_get_interface(None, 0, ctypes.byref(g), lo, cnt) == -1
