"""x slabs on one GPU: two or three slabs of a problem, each a separate
handle that updates only its own x planes and exchanges ghost planes after
every stage through fdf_pack_ghosts / fdf_unpack_ghosts, give the same fields
and fault arrays, bit for bit, as the whole domain stepped by fdf_step.

The slabs run one after another on one device (LocalSlabs); the pack,
unpack and stage calls are those a rank of a multi-GPU run makes, with the
NCCL send replaced by a device copy."""

import os

import numpy as np
import pytest

from fdfault_b200 import problems as P
from fdfault_b200 import slabs
from fdfault_b200.solver import FP32, FP64, FdfaultError, Problem

pytestmark = pytest.mark.gpu


def _planar(tmp, nx=72, nt=12, **kw):
    p = P.planar3d(nx=nx, ny=16, nz=40, h=0.25, nt=nt, name="slab_planar", workdir=tmp, datadir=tmp + "/",
                   corr=1.0, region=(12.0, 7.0), nuc_half=1.0, **kw)
    return p


def _xfault(tmp):
    # two x blocks and an x-normal fault between them: the fault and both
    # blocks' x faces stay with the slab that holds the first block's end
    p = P.Problem(name="slab_xfault", ndim=3, nx_block=([40, 40], [16], [36]), nt=10, datadir=tmp + "/")
    p.blocks[(0, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (0., 0., 0.), (9.75, 3.75, 8.75),
                                  ["absorbing", "none", "absorbing", "absorbing", "absorbing", "free"])
    p.blocks[(1, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (9.75, 0., 0.), (9.75, 3.75, 8.75),
                                  ["none", "absorbing", "absorbing", "absorbing", "absorbing", "free"])
    itf = P.Interface("x", (0, 0, 0), (1, 0, 0), "slipweak")
    itf.loads = [P.load("constant", 0., 0., 0., 0., 0., -120., 40., 50.),
                 P.load("boxcar", 0., 1.9, 0.8, 4.4, 0.8, 0., 20., 20.)]
    itf.perts = [P.swparam("constant", 0., 0., 0., 0., 0., 0.4, 0.677, 0.525)]
    p.interfaces.append(itf)
    return p


def _plastic(p):
    # at the Drucker-Prager limit for mu = 0.5: the return map yields
    p.material = "plastic"
    p.plastic_tensor = True
    for b in p.blocks.values():
        b.plastic = (0.5, 0.0, 0.2, 0.01 * b.g)
    p.s0 = (-120., 60., 0., -120., 0., -120.)
    p.interfaces[0].loads[0] = P.load("constant", 0., 0., 0., 0., 0., 0., 10., 0.)
    return p


def _compare(whole, loc, nifaces):
    ncomp = 9 + whole.nfieldsp
    for c in range(ncomp):
        a, b = whole.field(c), loc.field(c)
        assert np.array_equal(a, b), "component %d: max diff %g" % (c, np.max(np.abs(a - b)))
    for i in range(nifaces):
        for which in range(13):
            if whole.fault_count(i, which) == 0:
                continue
            a, b = whole.fault(i, which), loc.fault(i, which)
            assert np.array_equal(a, b), "interface %d array %d" % (i, which)


def _run(infile, precision, nslabs, nsteps, rule=None, slabs_plan=None, stream=None):
    whole = Problem(infile, precision)
    parts = [Problem(infile, precision) for _ in range(nslabs)]
    if rule is not None:
        for q in [whole] + parts:
            q.set_plastic_rule(rule)
    loc = slabs.LocalSlabs(parts, slabs_plan, stream=stream)
    whole.step(nsteps)
    loc.step(nsteps)
    whole.synchronize()
    return whole, loc


@pytest.mark.parametrize("precision,nslabs", [(FP32, 2), (FP32, 3), (FP64, 2)])
def test_planar_slabs_match_whole(tmp_path, precision, nslabs):
    tmp = str(tmp_path)
    infile = _planar(tmp).write(os.path.join(tmp, "planar.in"))
    whole, loc = _run(infile, precision, nslabs, 12)
    assert all(r.problem.step_index == whole.step_index == 12 for r in loc.runs)
    if precision == FP32:
        assert whole.set_volume_kernel(3) == 3   # the register-window kernel ran in both
    _compare(whole, loc, 1)


def test_slabs_on_the_callers_stream(tmp_path):
    # every slab launches on one torch stream and the ghost copies queue
    # behind the packs on it: no host synchronisation between stages
    import torch

    tmp = str(tmp_path)
    infile = _planar(tmp).write(os.path.join(tmp, "planar.in"))
    stream = torch.cuda.Stream()
    whole, loc = _run(infile, FP32, 3, 12, stream=stream)
    _compare(whole, loc, 1)
    for r in loc.runs:
        r.release()   # back to the problem's own stream and the whole domain
        r.problem.step(2)   # whole-domain steps (graph capture on the own stream) run again
        r.problem.synchronize()


def test_plastic_slabs_match_whole(tmp_path):
    tmp = str(tmp_path)
    infile = _plastic(_planar(tmp, nt=8)).write(os.path.join(tmp, "plastic.in"))
    whole, loc = _run(infile, FP32, 2, 8, rule=Problem.PLASTIC_EVERY_NODE)
    _compare(whole, loc, 1)
    gp = whole.field(10)
    assert np.max(gp) > 0.0   # the return map yielded somewhere


@pytest.mark.parametrize("cut", [20, 60])
def test_xfault_slabs_match_whole(tmp_path, cut):
    # the cut in the first block (the fault goes with the upper slab) or in
    # the second (with the lower one)
    tmp = str(tmp_path)
    infile = _xfault(tmp).write(os.path.join(tmp, "xfault.in"))
    for precision in (FP32, FP64):
        whole, loc = _run(infile, precision, 2, 10, slabs_plan=[(0, cut), (cut, 80)])
        _compare(whole, loc, 1)


def test_energy_sums_over_slabs_and_keeps_ghosts(tmp_path):
    tmp = str(tmp_path)
    infile = _planar(tmp).write(os.path.join(tmp, "planar.in"))
    whole, loc = _run(infile, FP64, 2, 6)
    e = whole.energy(rate=True)
    parts = [r.problem.energy(rate=True) for r in loc.runs]
    for k in ("kinetic", "strain", "rate", "friction_power"):
        s = sum(q[k] for q in parts)
        assert abs(s - e[k]) <= 1e-12 * max(abs(e[k]), e["rate_scale"], 1e-300), k
    # the rate evaluation swapped the field buffers: the slabs carried their
    # ghost planes across, so stepping on stays identical
    whole.step(3)
    loc.step(3)
    whole.synchronize()
    _compare(whole, loc, 1)


def test_slab_rejections(tmp_path):
    tmp = str(tmp_path)
    infile = _planar(tmp).write(os.path.join(tmp, "planar.in"))
    p = Problem(infile, FP32)
    with pytest.raises(FdfaultError, match="16 planes"):
        p.set_x_range(0, 10)
    with pytest.raises(FdfaultError):
        p.set_x_range(30, 30)
    p.set_x_range(0, 36)
    with pytest.raises(FdfaultError, match="stage at a time"):
        p.step(1)
    with pytest.raises(FdfaultError, match="whole domain"):
        p.solve()
    with pytest.raises(FdfaultError, match="expected stage 0"):
        p.step_stage(1)
    with pytest.raises(FdfaultError, match="no neighbour"):
        p.pack_ghosts(0, 1 << 20)
    p.set_volume_kernel(1)
    with pytest.raises(FdfaultError, match="volume kernel"):
        p.step_stage(0)
    p.set_volume_kernel(3)
    p.set_x_range(0, 72)   # whole domain again
    p.step(1)
    p.synchronize()
    q = P.mode2_rupture(nx=61, ny=31, nt=5, datadir=tmp + "/")
    p2 = Problem(q.write(os.path.join(tmp, "m2.in")), FP64)
    with pytest.raises(FdfaultError, match="3D"):
        p2.set_x_range(0, 30)
