"""Batched ensemble: every member, advanced together with the others by the
batched launches (CUDA-graph chunks and direct remainders, any tile
configuration the autotuner may pick), is bit-identical to the same problem
run alone in FP32 with the matching volume kernel -- the tiled 2D kernel for
2D members whose blocks fit it, the one-thread-per-node kernel for the rest --
for members of different sizes (some too narrow for the tiled kernel), a 3D
member, and a member that reaches its last step early."""

import os

import numpy as np
import pytest

from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu


def members(tmp):
    files = P.ensemble_members(n=5, seed=7, workdir=tmp, nt=30, size_range=((31, 16), (121, 61)))
    short = P.mode2_rupture(nx=41, ny=21, h=0.1, nt=9, name="short", datadir=tmp + "/", nuc_half=1.0)
    files.append(short.write(os.path.join(tmp, "short.in")))
    p3 = P.planar3d(nx=25, ny=13, nz=37, h=0.25, nt=30, name="m3d", datadir=tmp + "/", workdir=tmp, corr=1.0,
                    region=(4.0, 8.0), nuc_half=0.75)
    files.append(p3.write(os.path.join(tmp, "m3d.in")))
    return files


def alone(infile, nsteps):
    with fs.Problem(infile, precision=fs.FP32) as p:
        p.set_volume_kernel(1 if p.ndim == 2 else 0)
        p.step(min(nsteps, p.nt))
        p.synchronize()
        return state(p)


def state(p):
    out = [p.field(c) for c in range(p.nfields)]
    out += [p.fault(i, w) for i in range(p.nifaces) for w in (fs.U, fs.V, fs.S, fs.SN, fs.TFRONT)]
    return out, p.step_index


def compare(ens, files, nsteps):
    for i, f in enumerate(files):
        got, gi = state(ens.member(i))
        ref, ri = alone(f, nsteps)
        assert gi == ri, (i, gi, ri)
        for k, (x, y) in enumerate(zip(got, ref)):
            assert np.array_equal(x, y, equal_nan=True), (i, k)


def test_ensemble_matches_members_alone(tmp_path):
    tmp = str(tmp_path)
    files = members(tmp)
    with fs.Ensemble(files) as ens:
        assert ens.size == len(files)
        ens.set_config(128, 1024)
        ens.run(20)   # one 16-step graph chunk and 4 direct steps
        ens.run(7)
        ens.check_status()
        compare(ens, files, 27)


def test_ensemble_autotuned(tmp_path):
    tmp = str(tmp_path)
    files = members(tmp)
    with fs.Ensemble(files) as ens:
        threads, tile = ens.autotune(1)   # six candidates, one real step each
        assert threads in (128, 256) and tile in (1024, 4096, 16384)
        ens.run(17)
        ens.check_status()
        compare(ens, files, 23)


def test_ensemble_without_graph(tmp_path):
    tmp = str(tmp_path)
    files = members(tmp)[:3]
    with fs.Ensemble(files) as ens:
        ens.use_graph(False)
        ens.run(18)
        compare(ens, files, 18)
