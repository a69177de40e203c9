"""CPU oracle for the learned STZ initial guess network (test infrastructure:
only the tests use it).

The network is 6 -> 64 -> 64 -> 1 with ReLU hidden layers.  The forward pass
rounds inputs, weights and hidden activations to BF16 (round to nearest even)
and accumulates each dot product in FP32 one term at a time with a fused
multiply-add, then adds the FP32 bias -- the order of the per-thread GPU path.
The backward pass of the mean squared error 0.5*mean((y - t)^2) is FP32 with
the same one-term-at-a-time accumulation (over inputs for the hidden deltas,
over samples for the weight gradients), from the BF16 activations and weights.

A fused multiply-add in FP32 is emulated as round32(a*b + c) computed in FP64:
the product of two FP32 numbers is exact in FP64, so this equals the hardware
result except in the rare case where the FP64 sum itself rounds.

``grad_fd`` checks the analytic gradient of the unrounded FP64 network against
central finite differences, which pins the backward formulas independently of
the GPU.  The parameter layout is the flat vector
W1[64][6], b1[64], W2[64][64], b2[64], W3[64], b3.
"""

import numpy as np

NIN, NH = 6, 64
OFF_W1, OFF_B1, OFF_W2, OFF_B2, OFF_W3, OFF_B3, NPARAM = 0, 384, 448, 4544, 4608, 4672, 4673


def bf16(x):
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    return (p[OFF_W1:OFF_B1].reshape(NH, NIN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(NH, NH),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def _fma32(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def _dot_seq(W, X):
    """Z[s, o] = sum_i W[o, i] * X[s, i], accumulated over i in order in FP32."""
    acc = np.zeros((X.shape[0], W.shape[0]), dtype=np.float32)
    for i in range(W.shape[1]):
        acc = _fma32(W[None, :, i], X[:, i:i + 1], acc)
    return acc


def forward(p, x):
    """Network outputs and the intermediate values of the BF16 forward pass."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    W1b, W2b, W3b = bf16(W1), bf16(W2), bf16(W3)
    xb = bf16(np.asarray(x, dtype=np.float32).reshape(-1, NIN))
    z1 = (_dot_seq(W1b, xb) + b1[None, :]).astype(np.float32)
    h1 = bf16(np.maximum(z1, 0.0))
    z2 = (_dot_seq(W2b, h1) + b2[None, :]).astype(np.float32)
    h2 = bf16(np.maximum(z2, 0.0))
    y = np.zeros(xb.shape[0], dtype=np.float32)
    for o in range(NH):
        y = _fma32(W3b[o], h2[:, o], y)
    y = (y + b3).astype(np.float32)
    return y, dict(xb=xb, z1=z1, h1=h1, z2=z2, h2=h2, W2b=W2b, W3b=W3b)


def gradients(p, x, t):
    """Gradient of 0.5*mean((y - t)^2) (flat, FP32) and the loss."""
    y, c = forward(p, x)
    t = np.asarray(t, dtype=np.float32).reshape(-1)
    n = y.shape[0]
    e = (y - t).astype(np.float32)
    loss = float(np.mean(0.5 * e.astype(np.float64) ** 2))
    dy = (e * np.float32(1.0 / n)).astype(np.float32)
    mask2 = (c["z2"] > 0).astype(np.float32)
    dz2 = (mask2 * (dy[:, None] * c["W3b"][None, :]).astype(np.float32)).astype(np.float32)
    dh1 = np.zeros((n, NH), dtype=np.float32)
    for o in range(NH):
        dh1 = _fma32(c["W2b"][o][None, :], dz2[:, o:o + 1], dh1)
    dz1 = np.where(c["z1"] > 0, dh1, np.float32(0.0)).astype(np.float32)

    def over_samples(a, b):
        acc = np.zeros((a.shape[1], b.shape[1]), dtype=np.float32)
        for s in range(n):
            acc = _fma32(a[s][:, None], b[s][None, :], acc)
        return acc

    def sum_samples(a):
        acc = np.zeros(a.shape[1], dtype=np.float32)
        for s in range(n):
            acc = (acc + a[s]).astype(np.float32)
        return acc

    g = np.zeros(NPARAM, dtype=np.float32)
    g[OFF_W1:OFF_B1] = over_samples(dz1, c["xb"]).reshape(-1)
    g[OFF_B1:OFF_W2] = sum_samples(dz1)
    g[OFF_W2:OFF_B2] = over_samples(dz2, c["h1"]).reshape(-1)
    g[OFF_B2:OFF_W3] = sum_samples(dz2)
    g[OFF_W3:OFF_B3] = over_samples(dy[:, None], c["h2"]).reshape(-1)
    g[OFF_B3] = sum_samples(dy[:, None])[0]
    return g, loss


def _forward64(p, x):
    p = np.asarray(p, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = (p[OFF_W1:OFF_B1].reshape(NH, NIN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(NH, NH),
                              p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3 + b3, (z1, h1, z2, h2)


def grad64(p, x, t):
    """Analytic gradient of the unrounded FP64 network."""
    p = np.asarray(p, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    W2, W3 = p[OFF_W2:OFF_B2].reshape(NH, NH), p[OFF_W3:OFF_B3]
    y, (z1, h1, z2, h2) = _forward64(p, x)
    n = x.shape[0]
    dy = (y - t) / n
    dz2 = dy[:, None] * W3[None, :] * (z2 > 0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    g = np.zeros(NPARAM)
    g[OFF_W1:OFF_B1] = (dz1.T @ x).reshape(-1)
    g[OFF_B1:OFF_W2] = dz1.sum(0)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).reshape(-1)
    g[OFF_B2:OFF_W3] = dz2.sum(0)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    return g


def loss64(p, x, t):
    y, _ = _forward64(p, x)
    return 0.5 * np.mean((y - np.asarray(t, dtype=np.float64)) ** 2)


def grad_fd(p, x, t, idx, h=1e-6):
    """Central finite differences of loss64 for the parameters in idx."""
    p = np.asarray(p, dtype=np.float64).copy()
    out = []
    for q in idx:
        a = p.copy()
        a[q] += h
        b = p.copy()
        b[q] -= h
        out.append((loss64(a, x, t) - loss64(b, x, t)) / (2 * h))
    return np.array(out)


def he_init(seed):
    """A seeded parameter vector with the scale the solver's initialisation uses."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM, dtype=np.float32)
    p[OFF_W1:OFF_B1] = rng.standard_normal(NH * NIN) * np.sqrt(2.0 / NIN)
    p[OFF_W2:OFF_B2] = rng.standard_normal(NH * NH) * np.sqrt(2.0 / NH)
    p[OFF_W3:OFF_B3] = rng.standard_normal(NH) * np.sqrt(1.0 / NH)
    p[OFF_B1:OFF_W2] = rng.standard_normal(NH) * 0.1
    p[OFF_B2:OFF_W3] = rng.standard_normal(NH) * 0.1
    p[OFF_B3] = 0.5
    return p
