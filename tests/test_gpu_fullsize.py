"""Parity at the benchmark workloads' own sizes.

* The 2D mode-II workload (two blocks of 401 x 201, FP64, 1000 RK3 steps)
  against the reference solver's output for the same input
  (tests/golden/config1_full.npz): on-fault slip, slip rate and shear stress
  every 5 steps and vx / vy snapshots, relative L2 <= 1e-10 per output unit
  (the FP64 path replays the reference's operation order, so the measured
  difference is expected to be zero).
* The reference's own example input problems/test2d.in (801 x 802 nodes,
  RK4, barrier boxcars), truncated to 100 steps, same bound
  (tests/golden/test2d.npz holds the edited input text and the outputs).
* The 3D planar workload at full size (two blocks of 401 x 201 x 201): the FP32
  path (tiled and register-window volume kernels) against the GPU's FP64 path
  (bit-identical to the reference on every small case) after 300 steps, with
  the measured relative L2 errors printed and held to FP32_FULL_RTOL.
"""

import os
import sys

import numpy as np
import pytest

import helpers
import oracle
from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

sys.path.insert(0, helpers.GOLDEN)
import make_fullsize  # noqa: E402

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-10      # the accuracy contract of the FP64 path
FP32_FULL_RTOL = 1e-5  # FP32 vs FP64 after 300 steps at full size (measured <= 1.8e-6 on every key)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    b = np.asarray(b, dtype=np.float64).reshape(-1)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def compare_units(tmp, name, gold, units):
    worst, identical = 0.0, True
    for unit, field in units:
        u = oracle.read_unit(tmp, name, unit, field)
        ref = gold["unit/" + unit]
        assert u["data"].shape == ref.shape, unit
        e = rel_l2(u["data"], ref)
        identical &= bool(np.array_equal(u["data"], ref))
        worst = max(worst, e)
        assert e <= FP64_RTOL, (unit, e)
        if "t/" + unit in gold:
            assert np.array_equal(u["t"], gold["t/" + unit]), unit
    print("%s: worst relative L2 %.3g, bit-identical %s" % (name, worst, identical))


def test_config1_full_size_fp64_matches_reference(tmp_path):
    tmp = str(tmp_path)
    prob = make_fullsize.config1_problem(tmp + "/")
    infile = prob.write(os.path.join(tmp, "config1.in"))
    with fs.Problem(infile, precision=fs.FP64) as p:
        assert p.nt == 1000 and p.nxyz == 401 * 402
        p.solve()
    compare_units(tmp, "config1", helpers.load_golden("config1_full"),
                  [(o.name, o.field) for o in prob.outputs])


def test_reference_example_test2d_fp64_matches_reference(tmp_path):
    tmp = str(tmp_path)
    gold = helpers.load_golden("test2d")
    infile = os.path.join(tmp, "test2d.in")
    with open(infile, "w") as fh:
        fh.write(str(gold["input"]).replace("@DATADIR@", tmp + "/"))
    with fs.Problem(infile, precision=fs.FP64) as p:
        assert p.nt == make_fullsize.TEST2D_STEPS and p.rkorder == 4
        p.solve()
    compare_units(tmp, "test2d", gold, [("V", "V"), ("S", "S"), ("vx", "vx")])


def test_planar3d_full_size_fp32_against_fp64(tmp_path):
    tmp = str(tmp_path)
    nsteps = 300
    prob = P.planar3d(nt=nsteps + 2, name="planar3d", datadir=tmp + "/", workdir=tmp, seed=1234,
                      nx=401, ny=201, nz=201, h=0.1, cfl=P.WORKLOAD_CFL_3D)
    infile = prob.write(os.path.join(tmp, "planar3d.in"))
    keys = (fs.U, fs.V, fs.S)

    def run(precision, kind):
        with fs.Problem(infile, precision=precision) as p:
            if kind is not None:
                assert p.set_volume_kernel(kind) == kind
            p.step(nsteps)
            p.synchronize()
            out = {w: p.fault(0, w) for w in keys}
            for c in (0, 1, 2):
                out["v%d" % c] = p.field(c)[::7]
            return out

    ref = run(fs.FP64, None)
    assert np.max(ref[fs.V]) > 0.1   # the rupture is running
    for kind in (1, 3):
        got = run(fs.FP32, kind)
        errs = {str(k): rel_l2(got[k], ref[k]) for k in ref}
        print("planar3d full size, %d steps, FP32 kind %d vs FP64: %s" % (nsteps, kind, errs))
        for k, e in errs.items():
            assert e <= FP32_FULL_RTOL, (kind, k, e)
