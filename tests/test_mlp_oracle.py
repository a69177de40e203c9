"""The CPU oracle of the learned-guess network: its analytic gradient agrees
with central finite differences (FP64, unrounded network), its BF16 rounding
is round-to-nearest-even, and its BF16/FP32 gradient stays close to the FP64
one -- this pins the backward formulas the GPU kernels are checked against."""

import numpy as np

from oracle import mlp as M


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.14159, 1e-3], dtype=np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # a tie rounds to even
    assert r[2] == np.float32(1.0078125)
    assert r[3] == -2.5
    u = r.view(np.uint32)
    assert np.all((u & 0xFFFF) == 0)
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)


def test_gradient_matches_finite_differences():
    p = M.he_init(3).astype(np.float64)
    rng = np.random.default_rng(1)
    x = rng.uniform(-1, 1, (40, 6))
    t = rng.uniform(0, 1, 40)
    g = M.grad64(p, x, t)
    idx = list(range(0, 384, 37)) + list(range(384, 448, 9)) + list(range(448, 4544, 311)) + \
        list(range(4544, 4673, 13)) + [4672]
    fd = M.grad_fd(p, x, t, idx)
    assert np.max(np.abs(fd - g[idx])) <= 1e-7 * np.max(np.abs(g[idx]))


def test_bf16_gradient_close_to_fp64():
    p = M.he_init(4)
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, (64, 6)).astype(np.float32)
    t = rng.uniform(0, 1, 64).astype(np.float32)
    g32, l32 = M.gradients(p, x, t)
    g64 = M.grad64(p, x, t)
    assert abs(l32 - M.loss64(p, x, t)) <= 0.05 * M.loss64(p, x, t)
    assert np.linalg.norm(g32 - g64) <= 0.05 * np.linalg.norm(g64)
