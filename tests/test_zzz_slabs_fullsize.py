"""x slabs at the planar workload's full size (two blocks of 401 x 201 x 201,
FP32, register-window kernel): four slabs, each a handle on the same GPU that
updates its quarter of the x planes and swaps ghost planes after every stage,
against the whole domain stepped by fdf_step, bit for bit on the fault arrays
and field components.  Runs after the other GPU tests (it holds five copies of
the grid, about 30 GB)."""

import os

import numpy as np
import pytest

from fdfault_b200 import problems as P
from fdfault_b200 import slabs
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu


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
