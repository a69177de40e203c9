"""x slabs against the whole domain stepped by fdf_step, bit for bit, run
after the other GPU tests:

* the planar workload at full size (two blocks of 401 x 201 x 201, FP32,
  register-window kernel) in four slabs, each a handle on the same GPU that
  updates its quarter of the x planes and swaps ghost planes after every
  stage (up to five copies of the grid at once, about 30 GB);
* STZ friction (bracketed Newton from the midpoint, FP64 and FP32) in two
  slabs."""

import os

import numpy as np
import pytest

from cases import STZ_CONST
from fdfault_b200 import problems as P
from fdfault_b200 import slabs
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [fs.FP64, fs.FP32])
def test_stz_slabs_match_whole(tmp_path, precision):
    tmp = str(tmp_path)
    p = P.planar3d(nx=48, ny=16, nz=36, h=0.25, nt=12, name="slab_stz", workdir=tmp, datadir=tmp + "/",
                   corr=1.0, region=(8.0, 6.0), nuc_half=1.0)
    itf = p.interfaces[0]
    itf.kind = "stz"
    itf.chi0 = 0.05
    itf.paramfile = "none"
    itf.perts = [P.stzparam("constant", 0., 0., 0., 0., 0., *STZ_CONST)]
    infile = p.write(os.path.join(tmp, "stz.in"))
    with fs.Problem(infile, precision=precision) as whole:
        whole.step(12)
        whole.synchronize()
        ref = {w: whole.fault(0, w) for w in (fs.U, fs.V, fs.S, fs.STATE)}
        ref_f = {c: whole.field(c) for c in range(9)}
    parts = [fs.Problem(infile, precision=precision) for _ in range(2)]
    try:
        loc = slabs.LocalSlabs(parts)
        loc.step(12)
        for w, a in ref.items():
            assert np.array_equal(loc.fault(0, w), a), w
        for c, a in ref_f.items():
            assert np.array_equal(loc.field(c), a), c
    finally:
        for q in parts:
            q.close()


def test_planar3d_full_size_four_slabs_match_whole(tmp_path):
    tmp = str(tmp_path)
    nsteps = 20
    prob = P.planar3d(nt=nsteps + 2, name="planar3d", datadir=tmp + "/", workdir=tmp, seed=1234,
                      nx=401, ny=201, nz=201, h=0.1, cfl=P.WORKLOAD_CFL_3D)
    infile = prob.write(os.path.join(tmp, "planar3d.in"))
    with fs.Problem(infile, precision=fs.FP32) as whole:
        assert whole.set_volume_kernel(3) == 3
        whole.step(nsteps)
        whole.synchronize()
        ref = {w: whole.fault(0, w) for w in (fs.U, fs.V, fs.S, fs.SN)}
        ref_f = {c: whole.field(c) for c in (0, 1, 3, 8)}
    parts = [fs.Problem(infile, precision=fs.FP32) for _ in range(4)]
    try:
        loc = slabs.LocalSlabs(parts)
        assert loc.slabs == [(0, 100), (100, 200), (200, 301), (301, 401)]
        loc.step(nsteps)
        for w, a in ref.items():
            assert np.array_equal(loc.fault(0, w), a), w
        for c, a in ref_f.items():
            assert np.array_equal(loc.field(c), a), c
    finally:
        for q in parts:
            q.close()
