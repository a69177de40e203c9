"""Stepping by CUDA-graph replay (a one-step graph per field-buffer parity,
stage time from a device step counter) gives bit-identical fields, fault
arrays and rupture times to launching every kernel from the host, for
time-dependent loads (t0 > 0), slip-weakening time weakening, plasticity, STZ
friction (plain and learned start) and the FP32 marching kernel, with even and
odd step counts and odd and even numbers of RK stages.  The fault read-back
queued behind the steps (fdf_get_fault_async) returns the values the
synchronous read returns."""

import os

import numpy as np
import pytest

from cases import build_case
from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu


def snapshot(p):
    out = [p.field(c) for c in range(p.nfields)]
    out += [p.fault(i, w) for i in range(p.nifaces) for w in (fs.U, fs.V, fs.S, fs.SN, fs.TFRONT)]
    return out


def run(infile, precision, graphs, chunks, setup=None):
    with fs.Problem(infile, precision=precision) as p:
        if setup:
            setup(p)
        p.use_graphs(graphs)
        for n in chunks:
            p.step(n)
        p.synchronize()
        return snapshot(p), p.step_index


@pytest.mark.parametrize("name,precision", [("m2_perts", fs.FP64), ("m2_sw", fs.FP64), ("m2_plastic", fs.FP64),
                                            ("p3_sw", fs.FP32), ("p3_stz_files", fs.FP64),
                                            ("p3_stz_files", fs.FP32), ("m2_s3rk2", fs.FP64),
                                            ("m2_rk1", fs.FP64), ("m2_s2rk4", fs.FP64)])
def test_graph_replay_is_bit_identical(tmp_path, name, precision):
    prob = build_case(name, str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    chunks = [5, 2, 1, 4]   # odd and even counts, starting on either field buffer
    a, ia = run(infile, precision, False, chunks)
    b, ib = run(infile, precision, True, chunks)
    assert ia == ib == sum(chunks)
    for k, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y, equal_nan=True), k


def test_graph_replay_learned_stz(tmp_path):
    tmp = str(tmp_path)
    prob = P.stz3d(nx=25, ny=13, nz=37, h=0.25, nt=12, name="g_stz", datadir=tmp + "/", workdir=tmp,
                   nuc_half=0.75, region=(4.0, 8.0))
    infile = prob.write(os.path.join(tmp, "g_stz.in"))

    def setup(p):
        p.mlp_init(5)
        p.stz_learned(True)

    a, _ = run(infile, fs.FP32, False, [12], setup)
    b, _ = run(infile, fs.FP32, True, [12], setup)
    for k, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y, equal_nan=True), k


def test_async_fault_read_matches_sync(tmp_path):
    prob = build_case("p3_sw", str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    with fs.Problem(infile, precision=fs.FP32) as p:
        outs = {w: np.full(p.fault_count(0, w), np.nan) for w in (fs.V, fs.U, fs.SX)}
        for _ in range(3):
            p.step(1)
            for w, o in outs.items():
                p.fault_async(0, w, o)
        p.synchronize()
        for w, o in outs.items():
            assert np.array_equal(o, p.fault(0, w)), w


def test_async_fault_reads_every_step_through_the_ring(tmp_path):
    # a 100,001-node fault: six 0.8 MB arrays a step wrap the 64 MB snapshot
    # ring after about 13 steps, so slots are reused while earlier copies may
    # still be in flight; every step's values must match a synchronous read
    import torch

    tmp = str(tmp_path)
    prob = P.mode2_rupture(nx=100001, ny=16, h=0.1, nt=40, name="ring", datadir=tmp + "/", nuc_half=1.0)
    infile = prob.write(os.path.join(tmp, "ring.in"))
    whichs = (fs.V, fs.U, fs.S, fs.SN, fs.VX, fs.SX)
    nsteps = 30
    with fs.Problem(infile, precision=fs.FP32) as p:
        bufs = [[torch.empty(p.fault_count(0, w), dtype=torch.float64, pin_memory=True) for w in whichs]
                for _ in range(nsteps)]
        for s in range(nsteps):
            p.step(1)
            for w, b in zip(whichs, bufs[s]):
                p.fault_async(0, w, b.numpy())
        p.synchronize()
    with fs.Problem(infile, precision=fs.FP32) as q:
        for s in range(nsteps):
            q.step(1)
            for w, b in zip(whichs, bufs[s]):
                assert np.array_equal(b.numpy(), q.fault(0, w)), (s, w)

