"""The device status word: conditions the reference aborts on, and the bounded
waits of the TMA-staged kernels, reach the host as a solver status from
fdf_synchronize (FDF_ERR_SOLVER, with the status bits in the message), and the
GPU stays usable afterwards.  Failures are made on the host side of the inputs
(a NaN in a side file, an STZ melting threshold below the slip rate, a wait
limit that gives up at once); nothing here faults or hangs a GPU.

Reference abort sites: src/utilities.cpp:134-137,173-176 (Newton), src/stz.cpp:
341-344 (slip rate above v1)."""

import os
import re

import numpy as np
import pytest

from cases import STZ_CONST, build_case
from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu

ERR_MELT, ERR_NONFINITE, ERR_TIMEOUT = 4, 8, 32


def status_bits(err):
    m = re.search(r"solver status (\d+)", str(err))
    assert m, str(err)
    return int(m.group(1))


@pytest.mark.parametrize("precision", [fs.FP64, fs.FP32])
def test_nan_in_load_file_is_reported_at_set_up(tmp_path, precision):
    """A NaN in a load file reaches the initial interface solve: creation fails
    with the non-finite bit in its message."""
    prob = build_case("m2_files", str(tmp_path), outputs=False)
    lf = prob.interfaces[0].loadfile
    loads = np.fromfile(lf, dtype="<f8").reshape(3, -1)
    loads[:, 30] = np.nan
    loads.astype("<f8").tofile(lf)
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    with pytest.raises(fs.FdfaultError) as ei:
        fs.Problem(infile, precision=precision)
    m = re.search(r"status (\d+)", str(ei.value))
    assert m and int(m.group(1)) & ERR_NONFINITE, str(ei.value)


@pytest.mark.parametrize("precision", [fs.FP64, fs.FP32])
def test_nan_in_fields_is_reported_by_synchronize(tmp_path, precision):
    """A NaN put into the fields after set-up is found by the interface kernel
    during stepping and reported by fdf_synchronize; the word is cleared once
    read and the handle stays usable."""
    prob = build_case("m2_sw", str(tmp_path), outputs=False)
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    with fs.Problem(infile, precision=precision) as p:
        p.step(1)
        p.synchronize()
        p.set_field(0, np.full(p.nxyz, np.nan))
        p.step(1)
        with pytest.raises(fs.FdfaultError) as ei:
            p.synchronize()
        assert status_bits(ei.value) & ERR_NONFINITE
        p.set_field(0, np.zeros(p.nxyz))
        assert np.all(p.field(0) == 0.0)
        p.synchronize()


def test_stz_slip_rate_above_v1_is_reported(tmp_path):
    prob = build_case("m2_stz", str(tmp_path), outputs=False)
    const = list(STZ_CONST)
    const[-1] = 1.0e-12   # v1 below every slip rate the fault reaches
    prob.interfaces[0].perts = [P.stzparam("constant", 0., 0., 0., 0., 0., *const)]
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    # the initial interface solve of set-up may already see it; otherwise the
    # first steps do and fdf_synchronize reports it
    with pytest.raises(fs.FdfaultError) as ei:
        with fs.Problem(infile, precision=fs.FP64) as p:
            p.step(2)
            p.synchronize()
    m = re.search(r"status (\d+)", str(ei.value))
    assert m and int(m.group(1)) & ERR_MELT, str(ei.value)


def _planar(tmp):
    prob = P.planar3d(nx=41, ny=21, nz=41, h=0.25, nt=8, name="st_planar", datadir=tmp + "/", workdir=tmp,
                      corr=1.0, region=(8.0, 6.0), nuc_half=1.0)
    return prob.write(os.path.join(tmp, "st_planar.in"))


@pytest.mark.parametrize("kind", [2, 3])
def test_staged_wait_limit_reports_timeout(tmp_path, kind):
    """With every bounded wait giving up at once, the CTAs give up: the status
    says so, each CTA first waits for its own copies in flight, and a fresh
    handle on the same GPU then gives the normal results."""
    infile = _planar(str(tmp_path))
    with fs.Problem(infile, precision=fs.FP32) as p:
        assert p.set_volume_kernel(kind) == kind
        p.use_graphs(False)
        p.set_wait_limit(-1)
        p.step(1)
        with pytest.raises(fs.FdfaultError) as ei:
            p.synchronize()
        assert status_bits(ei.value) & ERR_TIMEOUT
    out = {}
    for k in (kind, 1):
        with fs.Problem(infile, precision=fs.FP32) as q:
            assert q.set_volume_kernel(k) == k
            q.step(4)
            q.synchronize()
            out[k] = [q.field(c) for c in range(q.nfields)] + [q.fault(0, fs.V)]
    for a, b in zip(out[kind], out[1]):
        nb = np.linalg.norm(b)
        assert np.linalg.norm(a - b) / (nb if nb > 0 else 1.0) < 1e-5
