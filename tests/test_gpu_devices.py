"""Handles on different devices driven from one host thread: every C-ABI call
runs on its handle's device (made current for the call) and leaves the
caller's current device as it was, so results match each problem run alone."""

import os

import numpy as np
import pytest

from cases import build_case
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu


def _infile(tmp):
    prob = build_case("p3_sw", tmp, outputs=False)
    return prob.write(os.path.join(tmp, prob.name + ".in"))


def _state(p):
    return [p.field(c) for c in range(p.nfields)] + [p.fault(0, w) for w in (fs.U, fs.V, fs.S)]


def test_handle_keeps_callers_device(tmp_path):
    import torch

    infile = _infile(str(tmp_path))
    torch.cuda.set_device(0)
    with fs.Problem(infile, precision=fs.FP32, device=0) as p:
        p.step(2)
        p.synchronize()
        assert torch.cuda.current_device() == 0


def test_two_devices_one_thread(tmp_path):
    import torch

    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    infile = _infile(str(tmp_path))
    with fs.Problem(infile, precision=fs.FP32, device=0) as r:
        r.step(6)
        ref = _state(r)
    torch.cuda.set_device(0)
    # created on device 1 first, then device 0, and stepped interleaved
    with fs.Problem(infile, precision=fs.FP32, device=1) as a, fs.Problem(infile, precision=fs.FP32, device=0) as b:
        for _ in range(3):
            a.step(2)
            b.step(2)
        sa, sb = _state(a), _state(b)
        assert torch.cuda.current_device() == 0
    for x, y, z in zip(ref, sa, sb):
        assert np.array_equal(x, y)
        assert np.array_equal(x, z)
