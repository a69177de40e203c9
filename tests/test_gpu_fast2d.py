"""The tiled FP32 2D kernel (mode II and mode III, elastic) computes the same
operator as the one-thread-per-node FP32 kernel, which follows the
reference's operation order, up to FP32 rounding; and a rupture run with it
stays within the FP32 tolerance of the FP64 oracle.  Cases cover orders 2-4,
RK3 and RK4, one tile (ny = 32), overlapping last tiles, wide blocks, free,
rigid and absorbing outer faces, corners where an outer face meets the
fault, and a fault between blocks split in x (interface on x faces)."""

import os

import numpy as np
import pytest

import oracle
from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def mode3(tmp, name, nx=51, ny=45, h=0.1, nt=20, sbporder=4):
    lx, ly = (nx - 1) * h, (ny - 1) * h
    p = P.Problem(name=name, ndim=2, mode=3, nx_block=([nx], [ny, ny], [1]), datadir=tmp + "/", nt=nt,
                  sbporder=sbporder)
    p.blocks[(0, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (0.0, 0.0), (lx, ly), ["absorbing", "free", "rigid", "none"])
    p.blocks[(0, 1, 0)] = P.Block(P.RHO, P.LAM, P.G, (0.0, ly), (lx, ly), ["free", "absorbing", "none", "absorbing"])
    itf = P.Interface("y", (0, 0, 0), (0, 1, 0), "slipweak")
    itf.loads = [P.load("constant", 0.0, 0.0, 0.0, 0.0, 0.0, -120.0, 0.0, 70.0),
                 P.load("boxcar", 0.0, 0.5 * lx, 1.0, 0.0, 0.0, 0.0, 0.0, 11.6)]
    itf.perts = [P.swparam("constant", 0.0, 0.0, 0.0, 0.0, 0.0, 0.4, 0.677, 0.525)]
    p.interfaces.append(itf)
    return p


def xsplit(tmp, name, nx=40, ny=50, h=0.1, nt=20):
    """Mode II fault on the x faces between two blocks side by side."""
    lx, ly = (nx - 1) * h, (ny - 1) * h
    p = P.Problem(name=name, ndim=2, mode=2, nx_block=([nx, nx], [ny], [1]), datadir=tmp + "/", nt=nt)
    p.blocks[(0, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (0.0, 0.0), (lx, ly), ["absorbing", "none", "free", "absorbing"])
    p.blocks[(1, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (lx, 0.0), (lx, ly), ["none", "absorbing", "rigid", "free"])
    itf = P.Interface("x", (0, 0, 0), (1, 0, 0), "slipweak")
    itf.loads = [P.load("constant", 0.0, 0.0, 0.0, 0.0, 0.0, -120.0, 70.0, 0.0),
                 P.load("boxcar", 0.0, 0.5 * ly, 1.0, 0.0, 0.0, 0.0, 11.6, 0.0)]
    itf.perts = [P.swparam("constant", 0.0, 0.0, 0.0, 0.0, 0.0, 0.4, 0.677, 0.525)]
    p.interfaces.append(itf)
    return p


def m2(tmp, name, **kw):
    base = dict(nx=61, ny=40, h=0.1, nt=20, name=name, datadir=tmp + "/", nuc_half=1.0)
    base.update(kw)
    return P.mode2_rupture(**base)


CASES = {
    # two tiles in j, the last overlapping the first (closure rows in both)
    "m2_o4": lambda t: m2(t, "m2_o4"),
    "m2_o3_rk4": lambda t: m2(t, "m2_o3_rk4", nx=50, ny=33, sbporder=3, rkorder=4, nt=12),
    # a single tile (ny = 32): both y faces in one warp
    "m2_o2_one_tile": lambda t: m2(t, "m2_o2_one_tile", ny=32, sbporder=2),
    # five tiles in j, rows longer than one x chunk
    "m2_wide": lambda t: m2(t, "m2_wide", nx=150, ny=150, nt=10),
    "m3_o4": lambda t: mode3(t, "m3_o4"),
    "m3_o3": lambda t: mode3(t, "m3_o3", ny=33, sbporder=3, nt=12),
    "xsplit": lambda t: xsplit(t, "xsplit"),
}


def stage_from_random_state(infile, kind, seed=33):
    """Fields and rates after each stage of one step from a seeded random state,
    with volume kernel `kind` (0 reference order, 1 tiled)."""
    rng = np.random.default_rng(seed)
    out = []
    with fs.Problem(infile, precision=fs.FP32) as p:
        active = p.set_volume_kernel(kind)
        for c in range(p.nfields):
            p.set_field(c, rng.uniform(-1, 1, p.nxyz))
            p.set_rate(c, rng.uniform(-1e-3, 1e-3, p.nxyz))
        for stage in range(p.nstages):
            p.do_rk_stage(p.dt, stage, 0.0)
            out.append({"f%d" % c: p.field(c) for c in range(p.nfields)})
            out[-1].update({"df%d" % c: p.rate(c) for c in range(p.nfields)})
    return active, out


@pytest.mark.parametrize("name", sorted(CASES))
def test_tiled2d_matches_reference_order_kernel(name, tmp_path):
    prob = CASES[name](str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    act_fast, a = stage_from_random_state(infile, 1)
    act_slow, b = stage_from_random_state(infile, 0)
    assert act_fast == 1 and act_slow == 0
    for s in range(len(a)):
        for k in a[s]:
            e = rel_l2(a[s][k], b[s][k])
            assert e < 1e-5, (s, k, e)


@pytest.mark.parametrize("name", sorted(CASES))
def test_tiled2d_rupture_close_to_fp64(name, tmp_path):
    prob = CASES[name](str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    with fs.Problem(infile, precision=fs.FP32) as p:
        assert p.set_volume_kernel(1) == 1
        p.step(prob.nt)
        p.synchronize()
        v, s, f0 = p.fault(0, fs.V), p.fault(0, fs.S), p.field(0)
    o = oracle.Oracle(infile)
    o.run(prob.nt)
    assert rel_l2(v, o.fault(0, oracle.V)) < 2e-3
    assert rel_l2(s, o.fault(0, oracle.SS)) < 2e-3
    assert rel_l2(f0, o.field(oracle.F)[0]) < 2e-3
    o.close()


def test_tiled2d_selection(tmp_path):
    prob = CASES["m2_o4"](str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    with fs.Problem(infile, precision=fs.FP32) as p:
        assert p.set_volume_kernel(1) == 1
        assert p.set_volume_kernel(2) == 0   # the staged kernel is 3D only
    with fs.Problem(infile, precision=fs.FP64) as p:
        assert p.set_volume_kernel(1) == 0   # FP64 keeps the reference order
