"""Parity cases: small fdfault problems covering every branch of the hot path.

Each case is built with ``fdfault_b200.problems`` (no dependency on the
reference's Python package) from fixed seeds, so the same ``.in`` file and
side files can be regenerated on any machine.  ``tests/golden/make_golden.py``
runs the reference solver on them; the tests compare the oracle and the GPU
path against those outputs and against each other.
"""

from __future__ import annotations

import os
from typing import Callable, Dict, List

import numpy as np

from fdfault_b200 import problems as P

STZ_CONST = (1.e-6, 0.55, 0.02, 0.3, 500.0, 1.e-3, 1.0, 0.2, 1.e4)


def _m2(name, **kw):
    base = dict(nx=61, ny=31, h=0.1, nt=40, name=name, nuc_half=1.0)
    base.update(kw)
    return P.mode2_rupture(**base)


def _plastic(p, tensor=False):
    p.material = "plastic"
    p.plastic_tensor = tensor
    for b in p.blocks.values():
        b.plastic = (0.6, 5.0, 0.2, 0.01 * b.g)
    return p


def c_m2_sw(tmp):
    return _m2("m2_sw")


def c_m2_s2rk4(tmp):
    return _m2("m2_s2rk4", sbporder=2, rkorder=4)


def c_m2_s3rk2(tmp):
    return _m2("m2_s3rk2", sbporder=3, rkorder=2)


def c_m2_rk1(tmp):
    return _m2("m2_rk1", rkorder=1, cfl=0.1)


def c_m2_freerigid(tmp):
    p = _m2("m2_freerigid")
    p.blocks[(0, 0, 0)].bounds = ["free", "rigid", "absorbing", "none"]
    p.blocks[(0, 1, 0)].bounds = ["rigid", "free", "none", "free"]
    return p


def c_m2_locked(tmp):
    p = _m2("m2_locked")
    p.interfaces[0].kind = "locked"
    p.s0 = (-5., 3., 0., -7., 0., 0.)
    p.blocks[(0, 0, 0)].bounds = ["absorbing", "free", "absorbing", "none"]
    # an unbalanced initial stress field launches waves across the locked interface
    nx, ny, nz = p.nx
    rng = np.random.default_rng(6)
    hf = os.path.join(tmp, "m2_locked.stress")
    rng.uniform(-1, 1, (3, nx, ny, nz)).astype("<f8").tofile(hf)
    p.loadfile = hf
    return p


def c_m2_frictionless(tmp):
    p = _m2("m2_frictionless")
    p.interfaces[0].kind = "frictionless"
    return p


def c_m2_diss(tmp):
    p = _m2("m2_diss")
    p.cdiss = 0.1
    return p


def c_m2_perts(tmp):
    p = _m2("m2_perts")
    itf = p.interfaces[0]
    itf.loads.append(P.load("gaussian", 0.05, 3.0, 0.8, 0.0, 0.0, -2.0, 3.0, 0.0))
    itf.loads.append(P.load("ellipse", 0.0, 2.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0))
    itf.perts.append(P.swparam("linear", 0.0, 0.1, 30.0, 0.0, 0.0, 0.0, 0.01, 0.0))
    itf.perts.append(P.swparam("boxcar", 0.0, 1.0, 0.5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.5, 0.05, 0.1))
    return p


def c_m2_files(tmp):
    p = _m2("m2_files")
    itf = p.interfaces[0]
    n0 = 61
    rng = np.random.default_rng(3)
    lf = os.path.join(tmp, "m2_files.load")
    np.stack([rng.uniform(-1, 1, n0), rng.uniform(-1, 1, n0), np.zeros(n0)]).astype("<f8").tofile(lf)
    itf.loadfile = lf
    pf = os.path.join(tmp, "m2_files.swp")
    np.stack([np.zeros(n0), rng.uniform(0, 0.05, n0), np.zeros(n0), np.zeros(n0), np.zeros(n0),
              np.zeros(n0)]).astype("<f8").tofile(pf)
    itf.paramfile = pf
    return p


def c_m2_het(tmp):
    p = _m2("m2_het")
    nx, ny, nz = p.nx
    rng = np.random.default_rng(4)
    hf = os.path.join(tmp, "m2_het.stress")
    rng.uniform(-1, 1, (3, nx, ny, nz)).astype("<f8").tofile(hf)
    p.loadfile = hf
    return p


def c_m2_hetmat(tmp):
    p = _m2("m2_hetmat")
    P.layered_material(p, os.path.join(tmp, "m2_hetmat.mat"), seed=11)
    return p


def _yielding(p, mu, tensor):
    """Plastic problem that yields: a uniform initial shear stress of 60 MPa
    under 120 MPa compression puts the volume at the Drucker-Prager limit for
    mu = 0.5 (no cohesion); the fault carries 10 MPa more shear."""
    p = _plastic(p, tensor)
    for b in p.blocks.values():
        b.plastic = (mu, 0.0, 0.2, 0.01 * b.g)
    p.s0 = (-120., 60., 0., -120., 0., -120.)
    p.interfaces[0].loads[0] = P.load("constant", 0., 0., 0., 0., 0., 0., 10., 0.)
    return p


def c_m2_hetmat_plastic(tmp):
    # yields at most nodes
    p = _yielding(_m2("m2_hetmat_plastic"), 0.5, False)
    P.layered_material(p, os.path.join(tmp, "m2_hetmat_plastic.mat"), seed=12)
    return p


def c_m2_plastic_yield(tmp):
    # yields at a few nodes near the rupture front
    return _yielding(_m2("m2_plastic_yield"), 0.51, True)


def c_m2_plastic(tmp):
    p = _plastic(_m2("m2_plastic"))
    p.s0 = (-120., 0., 0., -120., 0., -120.)
    p.interfaces[0].loads[0] = P.load("constant", 0., 0., 0., 0., 0., 0., 70., 0.)
    return p


def c_m2_plastic_tensor(tmp):
    p = _plastic(_m2("m2_plastic_tensor"), tensor=True)
    p.s0 = (-120., 0., 0., -120., 0., -120.)
    p.interfaces[0].loads[0] = P.load("constant", 0., 0., 0., 0., 0., 0., 70., 0.)
    return p


def c_m2_curve(tmp):
    p = _m2("m2_curve")
    nx, ny, h = 61, 31, 0.1
    x = np.arange(nx) * h
    yf = 3.0 + 0.15 * np.sin(2 * np.pi * x / 6.0)

    def surf(name, xs, ys):
        fn = os.path.join(tmp, name)
        np.stack([xs, ys]).astype("<f8").tofile(fn)
        return fn

    sf = surf("m2c_fault", x, yf)
    yb0, yb1 = np.linspace(0, yf[0], ny), np.linspace(0, yf[-1], ny)
    p.blocks[(0, 0, 0)].surfaces = [surf("m2c_b0x0", np.zeros(ny), yb0), surf("m2c_b0x1", np.full(ny, x[-1]), yb1),
                                    surf("m2c_b0y0", x, np.zeros(nx)), sf]
    yt0, yt1 = np.linspace(yf[0], 6.0, ny), np.linspace(yf[-1], 6.0, ny)
    p.blocks[(0, 1, 0)].surfaces = [surf("m2c_b1x0", np.zeros(ny), yt0), surf("m2c_b1x1", np.full(ny, x[-1]), yt1),
                                    sf, surf("m2c_b1y1", x, np.full(nx, 6.0))]
    return p


def c_m3(tmp):
    p = _m2("m3")
    p.mode = 3
    p.interfaces[0].loads = [P.load("constant", 0., 0., 0., 0., 0., -120., 0., 70.),
                             P.load("boxcar", 0., 3.0, 1.0, 0., 0., 0., 0., 11.6)]
    return p


def c_m3_plastic(tmp):
    p = _plastic(_m2("m3_plastic"))
    p.mode = 3
    p.s0 = (-120., 0., 10., -120., 0., -120.)
    p.interfaces[0].loads = [P.load("constant", 0., 0., 0., 0., 0., 0., 0., 60.),
                             P.load("boxcar", 0., 3.0, 1.0, 0., 0., 0., 0., 21.6)]
    return p


def c_m2_stz(tmp):
    p = _m2("m2_stz")
    itf = p.interfaces[0]
    itf.kind = "stz"
    itf.chi0 = 0.05
    itf.perts = [P.stzparam("constant", 0., 0., 0., 0., 0., *STZ_CONST)]
    return p


def _p3(name, tmp, **kw):
    base = dict(nx=25, ny=13, nz=15, h=0.25, nt=20, name=name, workdir=tmp, corr=1.0, region=(4.0, 2.5),
                nuc_half=0.75)
    base.update(kw)
    return P.planar3d(**base)


def c_p3_sw(tmp):
    return _p3("p3_sw", tmp)


def c_p3_rk4(tmp):
    p = _p3("p3_rk4", tmp, nt=12, rkorder=4, sbporder=3)
    p.blocks[(0, 0, 0)].bounds = ["rigid", "free", "absorbing", "none", "free", "absorbing"]
    p.cdiss = 0.05
    return p


def c_p3_plastic(tmp):
    p = _plastic(_p3("p3_plastic", tmp, nt=10), tensor=True)
    p.s0 = (-100., 0., 0., -120., 0., -110.)
    p.interfaces[0].loads[0] = P.load("constant", 0., 0., 0., 0., 0., 0., 70., 0.)
    nx, ny, nz = p.nx
    rng = np.random.default_rng(5)
    hf = os.path.join(tmp, "p3_plastic.stress")
    rng.uniform(-1, 1, (6, nx, ny, nz)).astype("<f8").tofile(hf)
    p.loadfile = hf
    return p


def c_p3_hetmat(tmp):
    p = _p3("p3_hetmat", tmp)
    p.blocks[(0, 0, 0)].bounds = ["absorbing", "free", "absorbing", "none", "free", "absorbing"]
    P.layered_material(p, os.path.join(tmp, "p3_hetmat.mat"), seed=13)
    return p


def c_p3_plastic_yield(tmp):
    return _yielding(_p3("p3_plastic_yield", tmp, nt=10), 0.5, True)


def c_p3_hetmat_visits(tmp):
    # a soft bottom plane (lambda + 2/3 G = 5.5): the reference's return-map
    # loop, whose z index takes the bulk modulus (block.cpp:451-524), visits
    # k = 0 and then k = trunc(5.5) + 1 = 6 of every column, where the usual
    # moduli (53.4) send it past the block
    p = _yielding(_p3("p3_hetmat_visits", tmp, nt=10), 0.5, True)
    nx, ny, nz = p.nx
    b = next(iter(p.blocks.values()))
    rho, lam, g = (np.full((nx, ny, nz), v) for v in (b.rho, b.lam, b.g))
    lam[:, :, 0] = 2.0
    g[:, :, 0] = 5.25
    p.matfile = P.write_material(os.path.join(tmp, "p3_hetmat_visits.mat"), rho, lam, g)
    return p


def c_p3_stz(tmp):
    p = _p3("p3_stz", tmp, nt=12)
    itf = p.interfaces[0]
    itf.kind = "stz"
    itf.chi0 = 0.05
    itf.paramfile = "none"
    itf.perts = [P.stzparam("constant", 0., 0., 0., 0., 0., *STZ_CONST)]
    return p


def c_p3_stz_files(tmp):
    """STZ with per-node f0 (parameter file) and chi0 (state file), the planar STZ workload's set-up."""
    return P.stz3d(nx=25, ny=13, nz=15, h=0.25, nt=12, name="p3_stz_files", workdir=tmp, nuc_half=0.75,
                   region=(4.0, 2.5))


def c_p3_rough(tmp):
    """Rough fault from surface files, Drucker-Prager plasticity, depth-dependent stress file
    (the rough-fault workload's set-up at small size)."""
    return P.rough3d(nx=25, ny=13, nz=15, h=0.25, nt=10, name="p3_rough", workdir=tmp, nuc_half=0.75)


def c_p3_xfault(tmp):
    p = P.Problem(name="p3_xfault", ndim=3, nx_block=([13, 13], [15], [14]), nt=10)
    p.blocks[(0, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (0., 0., 0.), (3., 3.5, 3.25),
                                  ["absorbing", "none", "absorbing", "absorbing", "absorbing", "free"])
    p.blocks[(1, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (3., 0., 0.), (3., 3.5, 3.25),
                                  ["none", "absorbing", "absorbing", "absorbing", "absorbing", "free"])
    itf = P.Interface("x", (0, 0, 0), (1, 0, 0), "slipweak")
    itf.loads = [P.load("constant", 0., 0., 0., 0., 0., -120., 40., 50.),
                 P.load("boxcar", 0., 1.75, 0.6, 1.6, 0.6, 0., 20., 20.)]
    itf.perts = [P.swparam("constant", 0., 0., 0., 0., 0., 0.4, 0.677, 0.525)]
    p.interfaces.append(itf)
    return p


def c_p3_zfault(tmp):
    p = P.Problem(name="p3_zfault", ndim=3, nx_block=([14], [15], [13, 13]), nt=10)
    p.blocks[(0, 0, 0)] = P.Block(P.RHO, P.LAM, P.G, (0., 0., 0.), (3.25, 3.5, 3.),
                                  ["absorbing", "absorbing", "absorbing", "absorbing", "absorbing", "none"])
    p.blocks[(0, 0, 1)] = P.Block(P.RHO, P.LAM, P.G, (0., 0., 3.), (3.25, 3.5, 3.),
                                  ["absorbing", "absorbing", "absorbing", "absorbing", "none", "free"])
    itf = P.Interface("z", (0, 0, 0), (0, 0, 1), "slipweak")
    itf.loads = [P.load("constant", 0., 0., 0., 0., 0., -120., 40., 50.),
                 P.load("boxcar", 0., 1.6, 0.6, 1.75, 0.6, 0., 20., 20.)]
    itf.perts = [P.swparam("constant", 0., 0., 0., 0., 0., 0.4, 0.677, 0.525)]
    p.interfaces.append(itf)
    return p


def _with_material(p, name, tmp, seed):
    p.name = name
    P.layered_material(p, os.path.join(tmp, name + ".mat"), seed=seed)
    return p


def c_p3_hetmat_xfault(tmp):
    return _with_material(c_p3_xfault(tmp), "p3_hetmat_xfault", tmp, 14)


def c_p3_hetmat_stz(tmp):
    return _with_material(c_p3_stz(tmp), "p3_hetmat_stz", tmp, 15)


def c_m2_hetmat_locked(tmp):
    return _with_material(c_m2_locked(tmp), "m2_hetmat_locked", tmp, 16)


def c_m2_four_blocks(tmp):
    """Four blocks, four interfaces meeting at a corner node (shared finalisation)."""
    h = 0.1
    p = P.Problem(name="m2_four_blocks", ndim=2, mode=2, nx_block=([31, 31], [21, 21], [1]), nt=30)
    for i in range(2):
        for j in range(2):
            bounds = ["absorbing" if i == 0 else "none", "none" if i == 0 else "absorbing",
                      "absorbing" if j == 0 else "none", "none" if j == 0 else "absorbing"]
            p.blocks[(i, j, 0)] = P.Block(P.RHO, P.LAM, P.G, (i * 3.0, j * 2.0), (3.0, 2.0), bounds)
    specs = [("x", (0, 0, 0), (1, 0, 0), "locked"), ("x", (0, 1, 0), (1, 1, 0), "locked"),
             ("y", (0, 0, 0), (0, 1, 0), "slipweak"), ("y", (1, 0, 0), (1, 1, 0), "slipweak")]
    for d, a, b, k in specs:
        itf = P.Interface(d, a, b, k)
        if k == "slipweak":
            itf.loads = [P.load("constant", 0., 0., 0., 0., 0., -120., 70., 0.),
                         P.load("boxcar", 0., 3.0, 0.8, 0., 0., 0., 11.6, 0.)]
            itf.perts = [P.swparam("constant", 0., 0., 0., 0., 0., 0.4, 0.677, 0.525)]
        p.interfaces.append(itf)
    return p


CASES: Dict[str, Callable] = {
    "m2_sw": c_m2_sw, "m2_s2rk4": c_m2_s2rk4, "m2_s3rk2": c_m2_s3rk2, "m2_rk1": c_m2_rk1,
    "m2_freerigid": c_m2_freerigid, "m2_locked": c_m2_locked, "m2_frictionless": c_m2_frictionless,
    "m2_diss": c_m2_diss, "m2_perts": c_m2_perts, "m2_files": c_m2_files, "m2_het": c_m2_het,
    "m2_plastic": c_m2_plastic, "m2_plastic_tensor": c_m2_plastic_tensor, "m2_curve": c_m2_curve,
    "m3": c_m3, "m3_plastic": c_m3_plastic, "m2_stz": c_m2_stz, "m2_four_blocks": c_m2_four_blocks,
    "p3_sw": c_p3_sw, "p3_rk4": c_p3_rk4, "p3_plastic": c_p3_plastic, "p3_stz": c_p3_stz,
    "p3_xfault": c_p3_xfault, "p3_zfault": c_p3_zfault, "p3_stz_files": c_p3_stz_files,
    "p3_rough": c_p3_rough, "m2_hetmat": c_m2_hetmat, "m2_hetmat_plastic": c_m2_hetmat_plastic,
    "p3_hetmat": c_p3_hetmat, "m2_plastic_yield": c_m2_plastic_yield, "p3_plastic_yield": c_p3_plastic_yield,
    "p3_hetmat_visits": c_p3_hetmat_visits, "p3_hetmat_xfault": c_p3_hetmat_xfault,
    "p3_hetmat_stz": c_p3_hetmat_stz, "m2_hetmat_locked": c_m2_hetmat_locked,
}

# cases whose friction law calls exp/log inside the per-stage solve (STZ);
# device and host libm differ in the last bit there
LIBM_CASES = {"m2_stz", "p3_stz", "p3_stz_files", "p3_hetmat_stz"}


def fault_fields(prob: P.Problem, iface: int = 0):
    """Output-unit fields valid for interface `iface` of `prob` (reference numbering rules)."""
    itf = prob.interfaces[iface]
    D = {"x": 0, "y": 1, "z": 2}[itf.direction]
    base = ["V", "U", "S", "Sn"] + (["state"] if itf.kind == "stz" else [])
    if prob.ndim == 2:
        tang = ["z"] if prob.mode == 3 else (["x"] if D == 1 else ["y"])
    else:
        tang = [c for i, c in enumerate("xyz") if i != D]
    comp = []
    for k, c in enumerate(tang):
        for q in ("V", "U", "S"):
            comp.append((q + c, k))
    return base, comp


def volume_fields(prob: P.Problem) -> List[str]:
    if prob.ndim == 3:
        f = ["vx", "vy", "vz", "sxx", "sxy", "sxz", "syy", "syz", "szz"]
    elif prob.mode == 2:
        f = ["vx", "vy", "sxx", "sxy", "syy"] + (["szz"] if prob.material == "plastic" else [])
    else:
        f = ["vz", "sxz", "syz"]
    if prob.material == "plastic":
        f += ["lambda", "gammap"]
        if prob.plastic_tensor:
            f += ["epxx", "epxy", "epxz", "epyy", "epyz", "epzz"]
    return f


def add_outputs(prob: P.Problem, every: int = 0) -> None:
    """Fault fields every step, a front, and volume snapshots: every `every`
    steps, or only at the last step when `every` is 0 (strided by 2 in 3D)."""
    nx, ny, nz = prob.nx
    nt = prob.nt
    xs = (2, 2, 2) if prob.ndim == 3 else (1, 1, 1)
    tm, ts = (nt, 1) if every <= 0 else (0, every)
    outs = [P.Output("vol_" + f, f, tm, nt, ts, (0, 0, 0), (nx - 1, ny - 1, nz - 1), xs)
            for f in volume_fields(prob)]
    for n, itf in enumerate(prob.interfaces):
        if itf.kind == "locked":
            continue
        D = {"x": 0, "y": 1, "z": 2}[itf.direction]
        start = prob.block_start(itf.idx2)
        b2 = prob.nx_block
        xm = list(start)
        xp = [start[d] + b2[d][itf.idx2[d]] - 1 for d in range(3)]
        xp[D] = start[D]
        base, comp = fault_fields(prob, n)
        for f in base + [c for c, _ in comp]:
            outs.append(P.Output("f%d_%s" % (n, f), f, 0, nt, 1, tuple(xm), tuple(xp), (1, 1, 1)))
    prob.front = ("V", 0.001) if any(i.kind != "locked" for i in prob.interfaces) else None
    prob.outputs = outs


def build_case(name: str, tmp: str, outputs: bool = True, every: int = 0) -> P.Problem:
    prob = CASES[name](tmp)
    prob.datadir = tmp.rstrip("/") + "/"
    if outputs:
        add_outputs(prob, every)
    return prob
