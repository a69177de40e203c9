"""FP64 energy diagnostics (fdf_energy).

* The device reductions (kinetic and strain energy in the SBP norm, their rate
  along the semi-discrete operator's L(f)) equal the same sums done here in
  numpy from the fields, the rates the call leaves in the rate register (dt
  L(f)) and
  the Jacobian; the norm used here is re-derived from the closure rows of the
  reference's operator (src/fd.cpp:53-120) by the SBP property
  H D + D^T H = diag(-1, 0, ..., 0, 1) starting from its h0.
* Energy stability of the semi-discretisation: from random states without
  initial stress or loads, dE/dt <= 0 for absorbing, free and rigid outer
  faces, locked, frictionless and slip-weakening interfaces, SBP orders 2-4,
  2D (modes II and III) and 3D, homogeneous and heterogeneous material.
* Over one RK step of a running rupture the energy change matches the
  trapezoidal rule on the computed rates.
* The FP32 path's energies against the FP64 path's after a rupture.
"""

import os

import numpy as np
import pytest

from cases import build_case
from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu

CLOSURE = {
    2: [[-0.5, 0., 0.5], [-1., 1., 0.], [-0.5, 0., 0.5]],
    3: [[1. / 12., -2. / 3., 0., 2. / 3., -1. / 12.], [-24. / 17., 59. / 34., -4. / 17., -3. / 34., 0., 0.],
        [-0.5, 0., 0.5, 0., 0., 0.], [4. / 43., -59. / 86., 0., 59. / 86., -4. / 43., 0.],
        [3. / 98., 0., -59. / 98., 0., 32. / 49., -4. / 49.]],
    4: [[-1. / 60., 3. / 20., -3. / 4., 0., 3. / 4., -3. / 20., 1. / 60.],
        [-1.582533518939116, 2.033378678700676, -0.141512858744873, -0.450398306578272, 0.104488069284042,
         0.036577936277544, 0., 0., 0.],
        [-0.462059195631158, 0., 0.287258622978251, 0.258816087376832, -0.069112065532624, -0.014903449191300,
         0., 0., 0.],
        [0.071247104721830, -0.636451095137907, 0., 0.606235523609147, -0.022902190275815, -0.018129342917256,
         0., 0., 0.],
        [0.114713313798970, -0.290087484386815, -0.306681191361148, 0., 0.520262285050482, -0.051642265516119,
         0.013435342414630, 0., 0.],
        [-0.036210680656541, 0.105400944933782, 0.015764336127392, -0.707905442575989, 0., 0.769199413962647,
         -0.164529643265203, 0.018281071473911, 0.],
        [-0.011398193015050, 0.020437334208704, 0.011220896474665, 0.063183694641876, -0.691649024426814, 0.,
         0.739709139060752, -0.147941827812150, 0.016437980868017]],
}
H0 = {2: 0.5, 3: 17. / 48., 4: 13649. / 43200.}


def derivative_matrix(order, n):
    C = CLOSURE[order]
    h, nb = (len(C[0]) - 1) // 2, len(C) - 1
    D = np.zeros((n, n))
    for p in range(n):
        if p < nb:
            D[p, :len(C[p + 1])] = C[p + 1]
        elif p >= n - nb:
            q = n - 1 - p
            D[p, n - len(C[q + 1]):] = -np.array(C[q + 1])[::-1]
        else:
            D[p, p - h:p + h + 1] = C[0]
    return D


def norm_1d(order, n):
    """Diagonal SBP norm of an n-point block from h0 and the closure rows."""
    D = derivative_matrix(order, n)
    nb = len(CLOSURE[order]) - 1
    w = np.ones(n)
    w[0] = w[-1] = H0[order]
    for i in range(1, nb):
        w[i] = w[n - 1 - i] = -w[0] * D[0, i] / D[i, 0]
    B = np.zeros((n, n))
    B[0, 0], B[-1, -1] = -1., 1.
    assert np.abs(np.diag(w) @ D + D.T @ np.diag(w) - B).max() < 1e-12
    return w


def node_weights(prob):
    per_dir = []
    for d in range(prob.ndim):
        parts = [norm_1d(prob.sbporder, n) / (n - 1) for n in prob.nx_block[d]]
        per_dir.append(np.concatenate(parts))
    w = per_dir[0][:, None] * per_dir[1][None, :]
    if prob.ndim == 3:
        w = w[:, :, None] * per_dir[2][None, None, :]
    return w.reshape(-1)


def energy_numpy(prob, J, F, R):
    rho, lam, g = P.RHO, P.LAM, P.G
    if prob.matfile != "none":   # per-node material
        rho, lam, g = np.fromfile(prob.matfile, dtype="<f8").reshape(3, -1)
    w = node_weights(prob) * J
    z = np.zeros_like(F[0])
    if prob.ndim == 3:
        v, rv = F[:3], R[:3]
        s, rs = list(F[3:9]), list(R[3:9])
    elif prob.mode == 2:
        nu = 0.5 * lam / (lam + g)
        v, rv = F[:2], R[:2]
        s = [F[2], F[3], z, F[4], z, nu * (F[2] + F[4])]
        rs = [R[2], R[3], z, R[4], z, nu * (R[2] + R[4])]
    else:
        v, rv = F[:1], R[:1]
        s, rs = [z, z, F[1], z, F[2], z], [z, z, R[1], z, R[2], z]
    c = lam / (3 * lam + 2 * g)
    tr, trr = s[0] + s[3] + s[5], rs[0] + rs[3] + rs[5]
    ss = s[0] ** 2 + s[3] ** 2 + s[5] ** 2 + 2 * (s[1] ** 2 + s[2] ** 2 + s[4] ** 2)
    sr = s[0] * rs[0] + s[3] * rs[3] + s[5] * rs[5] + 2 * (s[1] * rs[1] + s[2] * rs[2] + s[4] * rs[4])
    kin = 0.5 * rho * sum(a * a for a in v)
    kr = rho * sum(a * b for a, b in zip(v, rv))
    wr = 0.5 / g * (sr - c * tr * trr)
    return (np.sum(w * kin), np.sum(w * 0.25 / g * (ss - c * tr * tr)), np.sum(w * (kr + wr)),
            np.sum(w * (np.abs(kr) + np.abs(wr))))


def write(prob, tmp):
    return prob.write(os.path.join(tmp, prob.name + ".in"))


@pytest.mark.parametrize("name", ["m2_sw", "m3", "p3_sw", "m2_s2rk4", "m2_s3rk2", "m2_hetmat", "p3_hetmat"])
def test_energy_reductions_match_numpy(tmp_path, name):
    prob = build_case(name, str(tmp_path), outputs=False)
    with fs.Problem(write(prob, str(tmp_path)), precision=fs.FP64) as p:
        p.step(6)
        e = p.energy(rate=True)
        F = np.array([p.field(c) for c in range(p.nfields)])
        R = np.array([p.rate(c) for c in range(p.nfields)]) / p.dt   # the register holds dt L(f)
        J = p.geometry(2)
    k, s, r, scale = energy_numpy(prob, J, F, R)
    assert abs(e["kinetic"] - k) <= 1e-12 * abs(k)
    assert abs(e["strain"] - s) <= 1e-12 * abs(s)
    assert abs(e["rate"] - r) <= 1e-12 * scale
    assert abs(e["rate_scale"] - scale) <= 1e-12 * scale


def _unloaded(name, tmp):
    """A test case with its initial stress and fault loads removed, so the
    elastic energy has no source."""
    prob = build_case(name, tmp, outputs=False)
    prob.s0 = (0., 0., 0., 0., 0., 0.)
    prob.loadfile = "none"
    for itf in prob.interfaces:
        itf.loads = []
        itf.loadfile = "none"
    return prob


@pytest.mark.parametrize("name", ["m2_sw", "m2_freerigid", "m2_locked", "m2_frictionless", "m3", "p3_sw",
                                  "p3_rk4", "m2_s2rk4", "m2_s3rk2", "m2_hetmat", "p3_hetmat"])
def test_energy_rate_nonpositive_without_sources(tmp_path, name):
    prob = _unloaded(name, str(tmp_path))
    rng = np.random.default_rng(17)
    with fs.Problem(write(prob, str(tmp_path)), precision=fs.FP64) as p:
        for c in range(p.nfields):
            p.set_field(c, rng.uniform(-1., 1., p.nxyz))
        e = p.energy(rate=True)
    assert e["total"] > 0.
    print(name, "dE/dt %.6g, scale %.6g" % (e["rate"], e["rate_scale"]))
    assert e["rate"] <= 1e-12 * e["rate_scale"]


def test_energy_step_follows_trapezoidal_rule(tmp_path):
    prob = build_case("m2_sw", str(tmp_path), outputs=False)
    with fs.Problem(write(prob, str(tmp_path)), precision=fs.FP64) as p:
        p.step(20)
        e0 = p.energy(rate=True)
        p.step(1)
        e1 = p.energy(rate=True)
        dt = p.dt
    de = e1["total"] - e0["total"]
    trap = 0.5 * dt * (e0["rate"] + e1["rate"])
    print("energy change %.6g, trapezoidal rule %.6g" % (de, trap))
    assert abs(de - trap) <= 0.02 * abs(trap)
    assert e0["friction_power"] > 0. and e1["friction_power"] > 0.


def test_fp32_energies_close_to_fp64(tmp_path):
    prob = build_case("p3_sw", str(tmp_path), outputs=False)
    infile = write(prob, str(tmp_path))
    out = {}
    for prec in (fs.FP64, fs.FP32):
        with fs.Problem(infile, precision=prec) as p:
            p.step(12)
            out[prec] = p.energy(rate=True)
    rel = {k: abs(out[fs.FP32][k] - out[fs.FP64][k]) / abs(out[fs.FP64][k])
           for k in ("kinetic", "strain", "total", "rate", "friction_power")}
    print("FP32 vs FP64 energy diagnostics, relative difference:", rel)
    assert rel["total"] <= 1e-5 and rel["kinetic"] <= 1e-5 and rel["strain"] <= 1e-5
    assert rel["friction_power"] <= 1e-4
