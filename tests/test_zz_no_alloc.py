"""fdf_get_field_noalloc -- the read-back for callers that may not allocate
device memory once running (a service that sizes its GPU memory up front, or
code under an external memory budget) -- gathers into one fixed static device
buffer and returns exactly what fdf_get_field (growable scratch buffer)
returns, on two calls in a row, for FP64 and FP32 problems, plain and
absolute stress; fields larger than the buffer are rejected.  The file is
collected last so the entry point is also exercised after every other GPU
test has run."""

import os
import tempfile

import numpy as np
import pytest

from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu

MAX_VALUES = 1 << 20   # FDF_NOALLOC_MAX_VALUES in include/fdfault_b200.h


def _compare_all(p):
    for comp in range(p.nfields):
        for absolute in (False, True):
            ref = p.field(comp, absolute)
            first = p.field_noalloc(comp, absolute)
            second = p.field_noalloc(comp, absolute)
            assert np.array_equal(first, ref), (comp, absolute)
            assert np.array_equal(second, ref), (comp, absolute)


@pytest.mark.parametrize("precision", [fs.FP64, fs.FP32])
def test_noalloc_matches_get_field_2d(precision):
    tmp = tempfile.mkdtemp(prefix="fdf_noalloc_")
    prob = P.mode2_rupture(nx=61, ny=31, h=0.1, nt=8, name="na2d", datadir=tmp + "/", nuc_half=1.0)
    infile = prob.write(os.path.join(tmp, "na2d.in"))
    with fs.Problem(infile, precision=precision) as p:
        p.step(8)
        _compare_all(p)
        p.step(2)   # state moved on: the fixed buffer must not return stale values
        _compare_all(p)


def test_noalloc_matches_get_field_3d_fp32():
    tmp = tempfile.mkdtemp(prefix="fdf_noalloc_")
    prob = P.planar3d(nx=25, ny=13, nz=37, h=0.25, nt=6, name="na3d", datadir=tmp + "/", workdir=tmp,
                      corr=1.0, region=(4.0, 2.5), nuc_half=0.75)
    infile = prob.write(os.path.join(tmp, "na3d.in"))
    with fs.Problem(infile, precision=fs.FP32) as p:
        assert p.nxyz <= MAX_VALUES
        p.step(6)
        _compare_all(p)


def test_noalloc_two_handles_in_sequence():
    """Two problems on one device use the same buffer one after the other."""
    tmp = tempfile.mkdtemp(prefix="fdf_noalloc_")
    a = P.mode2_rupture(nx=61, ny=31, h=0.1, nt=4, name="na_a", datadir=tmp + "/", nuc_half=1.0)
    b = P.mode2_rupture(nx=41, ny=21, h=0.1, nt=4, name="na_b", datadir=tmp + "/", nuc_half=1.0)
    fa = a.write(os.path.join(tmp, "na_a.in"))
    fb = b.write(os.path.join(tmp, "na_b.in"))
    with fs.Problem(fa, precision=fs.FP64) as pa, fs.Problem(fb, precision=fs.FP64) as pb:
        pa.step(4)
        pb.step(4)
        for comp in range(pa.nfields):
            ra, rb = pa.field(comp), pb.field(comp)
            assert np.array_equal(pa.field_noalloc(comp), ra)
            assert np.array_equal(pb.field_noalloc(comp), rb)
            assert np.array_equal(pa.field_noalloc(comp), ra)


def test_noalloc_rejects_oversize():
    tmp = tempfile.mkdtemp(prefix="fdf_noalloc_")
    prob = P.mode2_rupture(nx=1101, ny=501, h=0.05, nt=1, name="na_big", datadir=tmp + "/", nuc_half=1.0)
    infile = prob.write(os.path.join(tmp, "na_big.in"))
    with fs.Problem(infile, precision=fs.FP32) as p:
        assert p.nxyz > MAX_VALUES
        with pytest.raises(fs.FdfaultError, match="allocation-free buffer"):
            p.field_noalloc(0)
        # the handle stays usable after the rejection
        assert np.isfinite(p.field(0)).all()


def test_noalloc_reserves_nothing_after_set_up():
    """The static buffer is reserved when a handle is created, so the first
    allocation-free calls of a fresh handle change the device's free memory by
    nothing."""
    import torch

    tmp = tempfile.mkdtemp(prefix="fdf_noalloc_")
    prob = P.mode2_rupture(nx=61, ny=31, h=0.1, nt=4, name="na_fresh", datadir=tmp + "/", nuc_half=1.0)
    infile = prob.write(os.path.join(tmp, "na_fresh.in"))
    torch.cuda.init()
    with fs.Problem(infile, precision=fs.FP64) as p:
        p.step(2)
        p.synchronize()
        free0 = torch.cuda.mem_get_info(p.device)[0]
        for comp in range(p.nfields):
            p.field_noalloc(comp)
            p.field_noalloc(comp, True)
        p.synchronize()
        assert torch.cuda.mem_get_info(p.device)[0] == free0
