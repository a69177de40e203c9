"""Learned initial guess for the STZ Newton solve.

* the network's forward pass on the GPU (per-thread path and tensor-core warp
  path) against the CPU oracle (oracle/mlp.py), which emulates its BF16
  rounding and FP32 accumulation order;
* the GPU gradients against the oracle's (whose backward formulas are pinned
  by finite differences in tests/test_mlp_oracle.py);
* training on samples the solver generates lowers the held-out loss;
* a run that starts every Newton solve from the trained network's guess
  agrees with the plain (midpoint-start) run to relative L2 <= 1e-5 on slip,
  slip rate, shear stress and state, and takes fewer Newton iterations.
"""

import os
import tempfile

import numpy as np
import pytest

from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs
from oracle import mlp as M

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def stz_problem(tmp, name="stz_small", nt=20, **kw):
    # 20 steps: on this coarse 6 x 3.5 km fault the locked barrier corner grows
    # unstable after about 30 steps (the reference solver does the same)
    base = dict(nx=25, ny=13, nz=15, h=0.25, nt=nt, name=name, datadir=tmp + "/", workdir=tmp, nuc_half=0.75,
                region=(4.0, 2.5))
    base.update(kw)
    prob = P.stz3d(**base)
    return prob.write(os.path.join(tmp, name + ".in"))


@pytest.fixture(scope="module")
def small_handle():
    tmp = tempfile.mkdtemp(prefix="fdf_mlp_")
    with fs.Problem(stz_problem(tmp, nt=4), precision=fs.FP64) as p:
        yield p


def random_inputs(n, seed):
    rng = np.random.default_rng(seed)
    x = np.stack([rng.uniform(0.3, 1.0, n), rng.uniform(0.2, 0.4, n), rng.uniform(0.8, 1.2, n),
                  rng.uniform(-1.0, 1.0, n), rng.uniform(0.8, 1.1, n), rng.uniform(0.4, 1.1, n)], axis=1)
    return x.astype(np.float32)


def test_forward_matches_oracle(small_handle):
    p = small_handle
    params = M.he_init(11)
    p.mlp_set_params(params)
    assert np.array_equal(p.mlp_params(), params)
    x = random_inputs(1000, 5)   # not a multiple of 32: the last warp has idle lanes
    ref, _ = M.forward(params, x)
    y_thread = p.mlp_infer(x, force_thread=True)
    y_warp = p.mlp_infer(x, force_thread=False)
    # per-thread path: same rounding and accumulation order as the oracle
    assert np.max(np.abs(y_thread - ref)) <= 1e-6 * max(1.0, np.max(np.abs(ref)))
    # tensor-core path: FP32 accumulation in the MMA's own order; a BF16
    # rounding of a hidden activation may land on the other side
    d = np.abs(y_warp - ref)
    assert np.median(d) <= 1e-5
    assert np.max(d) <= 2e-2 * max(1.0, np.max(np.abs(ref)))


def test_gradients_match_oracle(small_handle):
    p = small_handle
    params = M.he_init(12)
    p.mlp_set_params(params)
    x = random_inputs(300, 6)
    t = np.random.default_rng(7).uniform(0.0, 1.0, 300).astype(np.float32)
    g, loss = p.mlp_gradients(x, t)
    gref, lref = M.gradients(params, x, t)
    assert abs(loss - lref) <= 1e-6 * max(lref, 1e-12) + 1e-12
    assert rel_l2(g, gref) <= 1e-5
    # and every parameter block is exercised
    for a, b in ((0, 384), (384, 448), (448, 4544), (4544, 4608), (4608, 4672), (4672, 4673)):
        assert np.linalg.norm(gref[a:b]) > 0
        assert rel_l2(g[a:b], gref[a:b]) <= 1e-4


@pytest.fixture(scope="module")
def trained():
    """Samples from a plain run of the small STZ problem, and a network trained on them."""
    tmp = tempfile.mkdtemp(prefix="fdf_stz_")
    infile = stz_problem(tmp, nt=20)
    with fs.Problem(infile, precision=fs.FP64) as p:
        p.stz_collect(1 << 20)
        p.step(20)
        samples = p.stz_samples()
        p.mlp_init(3)
        x = samples[:, :6]
        t = samples[:, 6]
        y0 = p.mlp_infer(x)
        loss0 = float(np.mean(0.5 * (y0 - t) ** 2))
        tr, va = p.mlp_train(epochs=60, batch=1024, lr=2e-3, seed=1)
        params = p.mlp_params()
    return dict(infile=infile, samples=samples, loss0=loss0, train=tr, val=va, params=params)


def test_samples_are_solver_generated(trained):
    s = trained["samples"]
    assert s.shape[0] > 5000
    assert np.all(np.isfinite(s))
    # the converged mu lies in the bracket [muy, phi/|sn|]; the target is
    # t = logit(s)/20 with s = (mu - muy)/(phi/|sn| - muy), both ends floored at 1e-16
    mh, muy = s[:, 0].astype(np.float64), s[:, 1].astype(np.float64)
    mu = s[:, 7].astype(np.float64)
    assert np.all(mu >= muy - 1e-6) and np.all(mu <= mh + 1e-6)
    t = s[:, 6]
    assert np.all(np.abs(t) <= np.log(1e16) / 20 + 1e-3)
    mid = (mu - muy > 1e-3) & (mh - mu > 1e-3)   # away from the ends, float32 mu resolves s
    sv = (mu[mid] - muy[mid]) / (mh[mid] - muy[mid])
    assert np.allclose(t[mid], np.log(sv / (1 - sv)) / 20, atol=2e-3)


def test_training_lowers_heldout_loss(trained):
    assert trained["val"] < trained["loss0"] / 20


@pytest.mark.parametrize("precision", [fs.FP64, fs.FP32])
def test_learned_start_matches_plain_and_saves_iterations(trained, precision):
    nsteps = 20
    runs = {}
    for mode in ("plain", "learned"):
        with fs.Problem(trained["infile"], precision=precision) as p:
            p.mlp_set_params(trained["params"])
            p.stz_learned(mode == "learned")
            p.stz_counting(True)
            p.step(nsteps)
            r = {w: p.fault(0, w) for w in (fs.U, fs.V, fs.S, fs.STATE)}
            r["counts"] = p.stz_counts()
            runs[mode] = r
    for w in (fs.U, fs.V, fs.S, fs.STATE):
        assert rel_l2(runs["learned"][w], runs["plain"][w]) <= 1e-5, w
    nsol_p, it_p, mid_p = runs["plain"]["counts"]
    nsol_l, it_l, mid_l = runs["learned"]["counts"]
    print("Newton iterations per solve: plain %.2f, learned %.2f (%d of %d starts rejected)"
          % (it_p / nsol_p, it_l / nsol_l, mid_l, nsol_l))
    assert nsol_p == nsol_l and nsol_p > 0
    assert mid_p == nsol_p            # the plain solve always starts at the midpoint
    assert mid_l <= 0.02 * nsol_l     # the guess is rejected rarely
    assert it_l / nsol_l < 0.85 * it_p / nsol_p


@pytest.mark.parametrize("precision", [fs.FP64, fs.FP32])
def test_judge_starts_match_plain_and_count_iterations(trained, precision):
    """The two other ways of cutting Newton iterations that judge the learned
    start: a warm start from each node's previous root, and the exact
    derivative of the slip-rate law (the reference's has the wrong sign on its
    mu_y term).  Both converge to the plain solve's roots; the iteration counts
    of all four starts are printed."""
    nsteps = 20
    modes = {"plain": fs.Problem.STZ_MIDPOINT, "learned": fs.Problem.STZ_LEARNED, "warm": fs.Problem.STZ_WARM,
             "exact derivative": fs.Problem.STZ_EXACT_DERIVATIVE}
    runs = {}
    for mode, code in modes.items():
        with fs.Problem(trained["infile"], precision=precision) as p:
            p.mlp_set_params(trained["params"])
            p.stz_start(code)
            p.stz_counting(True)
            p.step(nsteps)
            r = {w: p.fault(0, w) for w in (fs.U, fs.V, fs.S, fs.STATE)}
            r["counts"] = p.stz_counts()
            runs[mode] = r
    per = {m: runs[m]["counts"][1] / max(runs[m]["counts"][0], 1) for m in runs}
    print("Newton iterations per solve:", {m: round(v, 3) for m, v in per.items()})
    for m in ("warm", "exact derivative"):
        for w in (fs.U, fs.V, fs.S, fs.STATE):
            assert rel_l2(runs[m][w], runs["plain"][w]) <= 1e-5, (m, w)
        assert runs[m]["counts"][0] == runs["plain"]["counts"][0]
    assert per["exact derivative"] < per["plain"]
    assert per["warm"] < per["plain"]
