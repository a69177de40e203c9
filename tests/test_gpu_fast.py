"""The tiled FP32 3D kernel computes the same operator as the one-thread-per-node
FP32 kernel (which follows the reference's operation order), up to FP32
rounding, on problems large enough for its tiles (ny >= 8, nz >= 32 per block)."""

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


def planar(tmp, name, **kw):
    base = dict(nx=41, ny=21, nz=41, h=0.25, nt=24, name=name, datadir=tmp + "/", workdir=tmp, corr=1.0,
                region=(8.0, 6.0), nuc_half=1.0)
    base.update(kw)
    return P.planar3d(**base)


def xfault(tmp, name):
    p = P.Problem(name=name, ndim=3, nx_block=([21, 21], [17], [40]), nt=16, datadir=tmp + "/")
    p.blocks[(0, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (0., 0., 0.), (5., 4., 9.75),
                                  ["absorbing", "none", "rigid", "absorbing", "absorbing", "free"])
    p.blocks[(1, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (5., 0., 0.), (5., 4., 9.75),
                                  ["none", "absorbing", "absorbing", "free", "absorbing", "free"])
    itf = P.Interface("x", (0, 0, 0), (1, 0, 0), "slipweak")
    itf.loads = [P.load("constant", 0., 0., 0., 0., 0., -120., 40., 50.),
                 P.load("boxcar", 0., 2.0, 1.0, 4.9, 1.0, 0., 25., 25.)]
    itf.perts = [P.swparam("constant", 0., 0., 0., 0., 0., 0.4, 0.677, 0.525)]
    p.interfaces.append(itf)
    return p


CASES = {
    "planar_o4": lambda t: planar(t, "planar_o4"),
    "planar_o3_rk4": lambda t: planar(t, "planar_o3_rk4", sbporder=3, rkorder=4, nt=12),
    "planar_o2": lambda t: planar(t, "planar_o2", sbporder=2),
    "xfault": lambda t: xfault(t, "xfault"),
    # three tiles in j and two in k whose last tile overlaps the one before
    # (closure rows in both)
    "small_o4": lambda t: planar(t, "small_o4", nx=25, ny=25, nz=37, nt=12),
    "small_o3": lambda t: planar(t, "small_o3", nx=25, ny=25, nz=37, nt=12, sbporder=3),
    # curvilinear rough fault from surface files, plasticity, depth-dependent stress file
    "rough_plastic": lambda t: P.rough3d(nx=25, ny=25, nz=37, h=0.25, nt=10, name="rough_plastic",
                                         datadir=t + "/", workdir=t, nuc_half=0.75),
}


def stage_from_random_state(infile, kind, seed=21):
    """Fields and rates after each stage of one step from a seeded random state,
    with volume kernel `kind` (0 reference order, 1 tiled, 2 staged, 3 register window)."""
    rng = np.random.default_rng(seed)
    out = []
    with fs.Problem(infile, precision=fs.FP32) as p:
        active = p.set_volume_kernel(kind)
        for c in range(p.nfields):
            p.set_field(c, rng.uniform(-1, 1, p.nxyz))
            p.set_rate(c, rng.uniform(-1e-3, 1e-3, p.nxyz))
        for stage in range(p.nstages):
            p.do_rk_stage(p.dt, stage, 0.0)
            out.append({"f%d" % c: p.field(c) for c in range(p.nfields + p.nfieldsp)})
            out[-1].update({"df%d" % c: p.rate(c) for c in range(p.nfields)})
    return active, out


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fast_kernel_matches_reference_order_kernel(name, kind, tmp_path):
    """Same operator: one step from a random state agrees to FP32 rounding
    (tiled kernel, kind 1, and staged kernel, kind 2)."""
    prob = CASES[name](str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    act_fast, a = stage_from_random_state(infile, kind)
    act_slow, b = stage_from_random_state(infile, 0)
    assert act_fast == kind and act_slow == 0
    for s in range(len(a)):
        for k in a[s]:
            e = rel_l2(a[s][k], b[s][k])
            assert e < 1e-5, (s, k, e)


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fast_kernel_rupture_close_to_fp64(name, kind, tmp_path):
    """A rupture run with the tiled or staged kernel stays within the FP32 tolerance of the FP64 oracle."""
    prob = CASES[name](str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    with fs.Problem(infile, precision=fs.FP32) as p:
        assert p.set_volume_kernel(kind) == kind
        p.step(prob.nt)
        p.synchronize()
        v, f0 = p.fault(0, fs.V), p.field(0)
    o = oracle.Oracle(infile)
    o.run(prob.nt)
    assert rel_l2(v, o.fault(0, oracle.V)) < 2e-3
    assert rel_l2(f0, o.field(oracle.F)[0]) < 2e-3
    o.close()
