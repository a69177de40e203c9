"""Writer for fdfault ``.in`` problem files and their binary side files.

The solver reads the sectioned text format that the fdfault Python module
writes (``python/fdfault/problem.py:1449-1512`` and the per-section writers it
calls).  This module produces the same format from a small in-memory
description, so problems can be built without the reference's Python package
(which is not installed on GPU hosts).  Section layout and value order follow
the readers in the reference solver:

* ``[fdfault.problem]``   src/problem.cpp:24-50
* ``[fdfault.domain]``    src/domain.cpp:35-76
* ``[fdfault.fields]``    src/fields.cpp:24-47
* ``[fdfault.blockIJK]``  src/block.cpp:52-86
* ``[fdfault.operator]``  src/block.cpp:87-107
* ``[fdfault.interfaceN]`` src/interface.cpp:28-54
* ``[fdfault.friction]``  src/friction.cpp:76-129
* ``[fdfault.slipweak]``  src/slipweak.cpp:42-96
* ``[fdfault.stz]``       src/stz.cpp:51-113
* ``[fdfault.outputlist]`` src/outputlist.cpp:28-72
* ``[fdfault.frontlist]`` src/frontlist.cpp:20-40

Floating-point values are written with ``repr`` so that the solver's decimal
to binary conversion reproduces exactly the double held here.
"""

from __future__ import annotations

import dataclasses
import os
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np


def _f(x: float) -> str:
    return repr(float(x))


@dataclasses.dataclass
class Pert:
    """One parametric perturbation line: shape, time ramp t0, x0, dx, y0, dy, values."""

    kind: str
    t0: float
    x0: float
    dx: float
    y0: float
    dy: float
    values: Tuple[float, ...]

    def line(self) -> str:
        return " ".join([self.kind] + [_f(v) for v in (self.t0, self.x0, self.dx, self.y0, self.dy)]
                        + [_f(v) for v in self.values])


def load(kind, t0, x0, dx, y0, dy, sn, s2, s3) -> Pert:
    return Pert(kind, t0, x0, dx, y0, dy, (sn, s2, s3))


def swparam(kind, t0, x0, dx, y0, dy, dc, mus, mud, c0=0.0, trup=0.0, tc=0.0) -> Pert:
    return Pert(kind, t0, x0, dx, y0, dy, (dc, mus, mud, c0, trup, tc))


def stzparam(kind, t0, x0, dx, y0, dy, v0, f0, a, muy, c0, R, beta, chiw, v1) -> Pert:
    return Pert(kind, t0, x0, dx, y0, dy, (v0, f0, a, muy, c0, R, beta, chiw, v1))


@dataclasses.dataclass
class Block:
    rho: float
    lam: float
    g: float
    xb: Sequence[float]
    lb: Sequence[float]
    bounds: Sequence[str]
    surfaces: Sequence[str] = ()
    plastic: Tuple[float, float, float, float] = (0.5735, 0.0, 0.2867, 0.2775)  # mu, c, beta, eta


@dataclasses.dataclass
class Interface:
    direction: str
    idx1: Tuple[int, int, int]
    idx2: Tuple[int, int, int]
    kind: str
    loads: List[Pert] = dataclasses.field(default_factory=list)
    loadfile: str = "none"
    perts: List[Pert] = dataclasses.field(default_factory=list)
    paramfile: str = "none"
    chi0: float = 0.0
    statefile: str = "none"


@dataclasses.dataclass
class Output:
    name: str
    field: str
    tm: int
    tp: int
    ts: int
    xm: Tuple[int, int, int]
    xp: Tuple[int, int, int]
    xs: Tuple[int, int, int]


@dataclasses.dataclass
class Problem:
    name: str
    ndim: int
    nx_block: Tuple[List[int], List[int], List[int]]
    mode: int = 2
    datadir: str = "data/"
    nt: int = 0
    dt: float = 0.0
    ttot: float = 0.0
    cfl: float = 0.3
    ninfo: int = 1000000
    rkorder: int = 3
    sbporder: int = 4
    material: str = "elastic"
    s0: Tuple[float, ...] = (0.0,) * 6
    loadfile: str = "none"
    matfile: str = "none"
    plastic_tensor: bool = False
    cdiss: float = 0.0
    blocks: Dict[Tuple[int, int, int], Block] = dataclasses.field(default_factory=dict)
    interfaces: List[Interface] = dataclasses.field(default_factory=list)
    outputs: List[Output] = dataclasses.field(default_factory=list)
    front: Optional[Tuple[str, float]] = None

    @property
    def nblocks(self) -> Tuple[int, int, int]:
        return tuple(len(v) for v in self.nx_block)  # type: ignore

    @property
    def nx(self) -> Tuple[int, int, int]:
        return tuple(sum(v) for v in self.nx_block)  # type: ignore

    def block_start(self, coords) -> Tuple[int, int, int]:
        return tuple(sum(self.nx_block[d][: coords[d]]) for d in range(3))  # type: ignore

    def text(self) -> str:
        L: List[str] = []
        L += ["[fdfault.problem]", self.name, self.datadir, str(self.nt), _f(self.dt), _f(self.ttot),
              _f(self.cfl), str(self.ninfo), str(self.rkorder), ""]
        nb = self.nblocks
        L += ["[fdfault.domain]", str(self.ndim), str(self.mode), " ".join(str(v) for v in self.nx),
              " ".join(str(v) for v in nb)]
        for d in range(3):
            L.append(" ".join(str(v) for v in self.nx_block[d]))
        L += [str(len(self.interfaces))]
        L += [" ".join(i.kind for i in self.interfaces)] if self.interfaces else [""]
        L += [str(self.sbporder), self.material, ""]
        L += ["[fdfault.fields]", " ".join(_f(v) for v in self.s0), self.loadfile, self.matfile,
              str(int(self.plastic_tensor)), ""]
        for i in range(nb[0]):
            for j in range(nb[1]):
                for k in range(nb[2]):
                    b = self.blocks[(i, j, k)]
                    L.append("[fdfault.block%d%d%d]" % (i, j, k))
                    mat = [b.rho, b.lam, b.g]
                    if self.material == "plastic":
                        mat += list(b.plastic)
                    L.append(" ".join(_f(v) for v in mat))
                    L.append(" ".join(_f(v) for v in b.xb[: self.ndim]))
                    L.append(" ".join(_f(v) for v in b.lb[: self.ndim]))
                    L += list(b.bounds)
                    surfs = list(b.surfaces) if b.surfaces else ["none"] * (2 * self.ndim)
                    L += surfs
                    L.append("")
        if self.cdiss > 0.0:
            L += ["[fdfault.operator]", _f(self.cdiss), ""]
        for n, itf in enumerate(self.interfaces):
            L += ["[fdfault.interface%d]" % n, itf.direction, " ".join(str(v) for v in itf.idx1),
                  " ".join(str(v) for v in itf.idx2), ""]
            if itf.kind != "locked":
                L += ["[fdfault.friction]", str(len(itf.loads))] + [p.line() for p in itf.loads]
                L += [itf.loadfile, ""]
            if itf.kind == "slipweak":
                L += ["[fdfault.slipweak]", str(len(itf.perts))] + [p.line() for p in itf.perts]
                L += [itf.paramfile, ""]
            elif itf.kind == "stz":
                L += ["[fdfault.stz]", _f(itf.chi0), itf.statefile, str(len(itf.perts))]
                L += [p.line() for p in itf.perts] + [itf.paramfile, ""]
        L.append("[fdfault.outputlist]")
        for o in self.outputs:
            L += [o.name, o.field, "%d %d %d" % (o.tm, o.tp, o.ts)]
            for d in range(3):
                L.append("%d %d %d" % (o.xm[d], o.xp[d], o.xs[d]))
        L += ["", ""]
        L.append("[fdfault.frontlist]")
        if self.front is None:
            L.append("0")
        else:
            L += ["1", self.front[0], _f(self.front[1])]
        L.append("")
        return "\n".join(L) + "\n"

    def write(self, path: str) -> str:
        with open(path, "w") as fh:
            fh.write(self.text())
        return path


# ---------------------------------------------------------------------------
# workload builders (seeded synthetic inputs with the shapes of the benchmark
# configurations)

RHO, CS, CP = 2.67, 3.464, 6.0
LAM = RHO * (CP ** 2 - 2.0 * CS ** 2)
G = RHO * CS ** 2


def mode2_rupture(nx: int = 401, ny: int = 201, h: float = 0.1, nt: int = 1000, name: str = "mode2",
                  datadir: str = "data/", rkorder: int = 3, sbporder: int = 4, cfl: float = 0.3,
                  mus: float = 0.677, mud: float = 0.525, dc: float = 0.4, sn: float = -120.0,
                  s2: float = 70.0, nuc_dtau: float = 11.6, nuc_half: float = 1.5,
                  barriers: bool = False, outputs: Sequence[Output] = ()) -> Problem:
    """2D plane-strain mode-II rupture on a flat horizontal fault.

    Two blocks of nx by ny nodes (grid spacing h km) meet on the y-normal
    fault; slip-weakening friction; uniform normal and shear load plus a
    centred nucleation patch of half-width nuc_half km where the shear load
    is raised by ``nuc_dtau`` (70 + 11.6 = 81.6 MPa by default); absorbing
    outer boundaries.
    """
    lx, ly = (nx - 1) * h, (ny - 1) * h
    p = Problem(name=name, ndim=2, mode=2, nx_block=([nx], [ny, ny], [1]), datadir=datadir, nt=nt,
                cfl=cfl, rkorder=rkorder, sbporder=sbporder)
    p.blocks[(0, 0, 0)] = Block(RHO, LAM, G, (0.0, 0.0), (lx, ly),
                                ["absorbing", "absorbing", "absorbing", "none"])
    p.blocks[(0, 1, 0)] = Block(RHO, LAM, G, (0.0, ly), (lx, ly),
                                ["absorbing", "absorbing", "none", "absorbing"])
    itf = Interface("y", (0, 0, 0), (0, 1, 0), "slipweak")
    itf.loads = [load("constant", 0.0, 0.0, 0.0, 0.0, 0.0, sn, s2, 0.0),
                 load("boxcar", 0.0, 0.5 * lx, nuc_half, 0.0, 0.0, 0.0, nuc_dtau, 0.0)]
    itf.perts = [swparam("constant", 0.0, 0.0, 0.0, 0.0, 0.0, dc, mus, mud)]
    if barriers:
        itf.perts += [swparam("boxcar", 0.0, 0.0625 * lx, 0.0625 * lx, 0.0, 0.0, 0.0, 10000.0, 0.0),
                      swparam("boxcar", 0.0, 0.9375 * lx, 0.0625 * lx, 0.0, 0.0, 0.0, 10000.0, 0.0)]
    p.interfaces.append(itf)
    p.outputs = list(outputs)
    return p


def lognormal_field(n0: int, n1: int, h: float, mean: float, sd: float, corr: float,
                    seed: int) -> np.ndarray:
    """Seeded log-normal random field with a Gaussian correlation length.

    White Gaussian noise is filtered in Fourier space by a Gaussian kernel of
    correlation length ``corr`` (same units as the grid spacing ``h``), scaled
    to unit variance, and mapped to a log-normal field with the requested
    arithmetic mean and standard deviation.
    """
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n0, n1))
    k0 = np.fft.fftfreq(n0, d=h)
    k1 = np.fft.fftfreq(n1, d=h)
    kk = k0[:, None] ** 2 + k1[None, :] ** 2
    filt = np.exp(-0.5 * (2.0 * np.pi) ** 2 * kk * (corr ** 2) / 2.0)
    g = np.real(np.fft.ifft2(np.fft.fft2(w) * filt))
    g = (g - g.mean()) / (g.std() + 1e-300)
    s2 = np.log1p((sd / mean) ** 2)
    mu_ln = np.log(mean) - 0.5 * s2
    return np.exp(mu_ln + np.sqrt(s2) * g)


def write_material(path: str, rho: np.ndarray, lam: np.ndarray, g: np.ndarray) -> str:
    """Heterogeneous material file (fields.cpp:582-711): density, Lame's first
    parameter and shear modulus over the whole grid, each an (nx, ny, nz) array
    in C order (nz = 1 in 2D), written one after the other as little-endian
    FP64.  Every value must be positive.  Set the problem's ``matfile`` to the
    returned path; the blocks' own (rho, lam, g) are then not used by the
    time stepping."""
    arrs = [np.asarray(a, dtype="<f8") for a in (rho, lam, g)]
    if not all(a.shape == arrs[0].shape for a in arrs):
        raise ValueError("material arrays differ in shape")
    if not all(np.all(a > 0.) and np.all(np.isfinite(a)) for a in arrs):
        raise ValueError("material properties must be positive and finite")
    np.concatenate([a.reshape(-1) for a in arrs]).tofile(path)
    return path


def layered_material(prob: "Problem", path: str, seed: int, contrast: float = 0.2,
                     noise: float = 0.05) -> str:
    """Write a seeded heterogeneous material for ``prob`` and point its
    ``matfile`` at it: each of rho, lambda and G is the first block's value
    times (1 + contrast * (y - 1/2) + noise * U[-1, 1]) with y the node's
    relative position across the grid in y, so a fault normal to y sees a
    different material on each side and every node its own."""
    nx, ny, nz = prob.nx
    b = next(iter(prob.blocks.values()))
    rng = np.random.default_rng(seed)
    y = (np.arange(ny) / max(ny - 1, 1))[None, :, None]
    arrs = [base * (1. + contrast * (y - 0.5) + noise * rng.uniform(-1., 1., (nx, ny, nz)))
            for base in (b.rho, b.lam, b.g)]
    prob.matfile = write_material(path, *arrs)
    return path


# CFL number of the full-size 3D workloads (two blocks of 401 x 201 x 201 at
# h = 0.1 km, RK3).  At CFL 0.3 and 0.25 both precisions grow without bound at
# the corners where the fault meets the absorbing x and z- faces after about
# 180 and 450 steps (the SAT terms of three faces stack there and RK3's
# stability interval is exceeded); at 0.2 and 0.15 1500 steps stay bounded.
WORKLOAD_CFL_3D = 0.2


def planar3d(nx: int = 401, ny: int = 201, nz: int = 201, h: float = 0.1, nt: int = 1500,
             name: str = "planar3d", datadir: str = "data/", workdir: str = ".", seed: int = 1234,
             rkorder: int = 3, sbporder: int = 4, cfl: float = 0.3, mus_mean: float = 0.677,
             mus_sd: float = 0.03, corr: float = 2.0, region: Tuple[float, float] = (20.0, 15.0),
             nuc_half: float = 1.0, mud: float = 0.525, dc: float = 0.4, sn: float = -120.0,
             s2: float = 70.0, nuc_dtau: float = 11.6, outputs: Sequence[Output] = ()) -> Problem:
    """3D vertical strike-slip fault: two blocks of nx*ny*nz nodes split in y.

    Static friction per fault node comes from a seeded log-normal field
    (written to a slip-weakening parameter file); outside a frictional region
    of ``region`` km (along strike, along dip) static friction is 10000; a
    square nucleation patch of half-width ``nuc_half`` km sits at the centre.
    The free surface is the z+ face; the other outer faces absorb.
    """
    lx, ly, lz = (nx - 1) * h, (ny - 1) * h, (nz - 1) * h
    p = Problem(name=name, ndim=3, mode=2, nx_block=([nx], [ny, ny], [nz]), datadir=datadir, nt=nt,
                cfl=cfl, rkorder=rkorder, sbporder=sbporder)
    p.blocks[(0, 0, 0)] = Block(RHO, LAM, G, (0.0, 0.0, 0.0), (lx, ly, lz),
                                ["absorbing", "absorbing", "absorbing", "none", "absorbing", "free"])
    p.blocks[(0, 1, 0)] = Block(RHO, LAM, G, (0.0, ly, 0.0), (lx, ly, lz),
                                ["absorbing", "absorbing", "none", "absorbing", "absorbing", "free"])
    itf = Interface("y", (0, 0, 0), (0, 1, 0), "slipweak")
    xc, zc = 0.5 * lx, 0.5 * lz
    itf.loads = [load("constant", 0.0, 0.0, 0.0, 0.0, 0.0, sn, s2, 0.0),
                 load("boxcar", 0.0, xc, nuc_half, zc, nuc_half, 0.0, nuc_dtau, 0.0)]
    itf.perts = [swparam("constant", 0.0, 0.0, 0.0, 0.0, 0.0, dc, 0.0, mud)]
    # per-node static friction: log-normal inside the frictional region, barrier outside
    xs = np.arange(nx) * h
    zs = np.arange(nz) * h
    mus = lognormal_field(nx, nz, h, mus_mean, mus_sd, corr, seed)
    inside = (np.abs(xs[:, None] - xc) <= 0.5 * region[0]) & (np.abs(zs[None, :] - zc) <= 0.5 * region[1])
    mus = np.where(inside, mus, 10000.0)
    zero = np.zeros((nx, nz))
    pfile = os.path.join(workdir, name + ".swparam")
    np.stack([zero, mus, zero, zero, zero, zero]).astype("<f8").tofile(pfile)
    itf.paramfile = pfile
    p.interfaces.append(itf)
    p.outputs = list(outputs)
    return p


# STZ constants of the planar STZ workload: a, muy, c0, R, beta, chiw, v1 are not
# given by the workload's description and are chosen here (v0 and the ranges
# of f0 and chi0 are given).  With chi0 spread over [0.05, 0.1] the initial
# slip rate at one stress spans a factor e^10; a = 0.03 keeps the fault
# creeping (up to a few cm/s outside the nucleation patch, dm/s inside) where
# smaller a (0.02) starts the chi0 = 0.1 nodes at tens of m/s and the run
# diverges.
# chiw = 0.2 keeps the steady-state effective temperature below chi0 for all
# slip rates below v1, so every node strengthens as it slips: with larger chiw
# (1.2) single grid nodes heat up, run away and the run diverges.
STZ_V0 = 1.0e-6
STZ_CONSTANTS = dict(a=0.03, muy=0.3, c0=500.0, R=1.0e-3, beta=1.0, chiw=0.2, v1=1.0e4)


def stz3d(nx: int = 401, ny: int = 201, nz: int = 201, h: float = 0.1, nt: int = 1500,
          name: str = "stz3d", datadir: str = "data/", workdir: str = ".", seed: int = 4321,
          rkorder: int = 3, sbporder: int = 4, cfl: float = 0.3, f0_range: Tuple[float, float] = (0.5, 0.6),
          chi0_range: Tuple[float, float] = (0.05, 0.1), region: Tuple[float, float] = (20.0, 15.0),
          muy_barrier: float = 10000.0, nuc_half: float = 1.0, sn: float = -120.0, s2: float = 70.0,
          nuc_dtau: float = 11.6, outputs: Sequence[Output] = ()) -> Problem:
    """3D vertical strike-slip fault with STZ friction: the planar geometry of
    ``planar3d`` (two blocks of nx*ny*nz nodes split in y) with per-node STZ
    parameters drawn from a seeded uniform distribution: f0 in ``f0_range``
    (STZ parameter file) and the initial effective temperature chi0 in
    ``chi0_range`` (state file); v0 = 1e-6 m/s and the other STZ constants
    are STZ_CONSTANTS.  Outside a central region of ``region`` km (along
    strike, along dip) the jamming friction muy is raised by ``muy_barrier``,
    which locks the fault edges without a Newton solve (muy above the
    traction ratio takes the solver's locked branch) -- the counterpart of
    ``planar3d``'s static-friction barrier.  Loads and nucleation patch as in
    ``planar3d``."""
    lx, ly, lz = (nx - 1) * h, (ny - 1) * h, (nz - 1) * h
    p = Problem(name=name, ndim=3, mode=2, nx_block=([nx], [ny, ny], [nz]), datadir=datadir, nt=nt,
                cfl=cfl, rkorder=rkorder, sbporder=sbporder)
    p.blocks[(0, 0, 0)] = Block(RHO, LAM, G, (0.0, 0.0, 0.0), (lx, ly, lz),
                                ["absorbing", "absorbing", "absorbing", "none", "absorbing", "free"])
    p.blocks[(0, 1, 0)] = Block(RHO, LAM, G, (0.0, ly, 0.0), (lx, ly, lz),
                                ["absorbing", "absorbing", "none", "absorbing", "absorbing", "free"])
    itf = Interface("y", (0, 0, 0), (0, 1, 0), "stz")
    xc, zc = 0.5 * lx, 0.5 * lz
    itf.loads = [load("constant", 0.0, 0.0, 0.0, 0.0, 0.0, sn, s2, 0.0),
                 load("boxcar", 0.0, xc, nuc_half, zc, nuc_half, 0.0, nuc_dtau, 0.0)]
    c = STZ_CONSTANTS
    itf.perts = [stzparam("constant", 0.0, 0.0, 0.0, 0.0, 0.0, STZ_V0, 0.0, c["a"], c["muy"], c["c0"], c["R"],
                          c["beta"], c["chiw"], c["v1"])]
    rng = np.random.default_rng(seed)
    f0 = rng.uniform(f0_range[0], f0_range[1], (nx, nz))
    chi0 = rng.uniform(chi0_range[0], chi0_range[1], (nx, nz))
    xs = np.arange(nx) * h
    zs = np.arange(nz) * h
    inside = (np.abs(xs[:, None] - xc) <= 0.5 * region[0]) & (np.abs(zs[None, :] - zc) <= 0.5 * region[1])
    muy = np.where(inside, 0.0, muy_barrier)
    zero = np.zeros((nx, nz))
    pfile = os.path.join(workdir, name + ".stzparam")
    np.stack([zero, f0, zero, muy, zero, zero, zero, zero, zero]).astype("<f8").tofile(pfile)
    sfile = os.path.join(workdir, name + ".state")
    chi0.astype("<f8").tofile(sfile)
    itf.paramfile = pfile
    itf.statefile = sfile
    itf.chi0 = 0.0
    p.interfaces.append(itf)
    p.outputs = list(outputs)
    return p


def ensemble_members(n: int = 256, seed: int = 2024, workdir: str = ".", nt: int = 400,
                     size_range: Tuple[Tuple[int, int], Tuple[int, int]] = ((101, 51), (801, 401)),
                     h: float = 0.1) -> List[str]:
    """``n`` 2D mode-II slip-weakening ruptures of uneven sizes, written as .in
    files under ``workdir`` (returned in order).

    Member i has two blocks of nx by ny nodes with nx drawn log-uniform in
    the range of ``size_range`` (ny = nx // 2 + 1, so 101x51 ... 801x401) at a
    common grid spacing ``h`` (so every member has the same time step and runs
    ``nt`` steps); static and dynamic friction, slip-weakening distance and
    the nucleation shear load are drawn uniformly per member: mus in [0.6,
    0.75], mud in [0.45, 0.55], dc in [0.2, 0.6] m and the nucleation patch's
    shear load 2 to 8 MPa above the static strength (mus * 120 MPa)."""
    rng = np.random.default_rng(seed)
    (lo, _), (hi, _) = size_range
    files = []
    for i in range(n):
        nx = int(round(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        ny = nx // 2 + 1
        mus = float(rng.uniform(0.6, 0.75))
        mud = float(rng.uniform(0.45, 0.55))
        dc = float(rng.uniform(0.2, 0.6))
        over = float(rng.uniform(2.0, 8.0))
        nuc_dtau = mus * 120.0 + over - 70.0
        name = "member%03d" % i
        p = mode2_rupture(nx=nx, ny=ny, h=h, nt=nt, name=name, datadir=workdir.rstrip("/") + "/",
                          mus=mus, mud=mud, dc=dc, nuc_dtau=nuc_dtau, nuc_half=min(1.5, 0.1 * (nx - 1) * h))
        files.append(p.write(os.path.join(workdir, name + ".in")))
    return files


def rough_surface(nx: int, nz: int, h: float, alpha: float = 1e-3, lmin: float = 0.2, lmax: float = 20.0,
                  seed: int = 99) -> np.ndarray:
    """Band-limited self-similar roughness r(x, z) in km on an nx by nz grid of spacing h.

    Random Fourier phases from ``seed``, amplitude spectrum proportional to
    |k|^-2 (power spectral density |k|^-4, the 2D self-similar case) for
    wavelengths between ``lmin`` and ``lmax`` (and at least two grid
    spacings), and root-mean-square height ``alpha`` times the longest
    wavelength present (the domain length when that is shorter than lmax)."""
    rng = np.random.default_rng(seed)
    kx = np.fft.fftfreq(nx, d=h)
    kz = np.fft.rfftfreq(nz, d=h)
    kk = np.sqrt(kx[:, None] ** 2 + kz[None, :] ** 2)
    lo = 1.0 / min(lmax, max((nx - 1) * h, (nz - 1) * h))
    hi = 1.0 / max(lmin, 2.0 * h)
    band = (kk >= lo) & (kk <= hi)
    amp = np.where(band, 1.0 / np.maximum(kk, 1e-30) ** 2, 0.0)
    phase = rng.uniform(0.0, 2.0 * np.pi, amp.shape)
    surf = np.fft.irfft2(amp * np.exp(1j * phase), s=(nx, nz))
    rms = float(np.sqrt(np.mean(surf ** 2)))
    target = alpha / lo
    return surf * (target / rms) if rms > 0 else surf


def rough3d(nx: int = 601, ny: int = 301, nz: int = 301, h: float = 0.1, nt: int = 1000, name: str = "rough3d",
            datadir: str = "data/", workdir: str = ".", seed: int = 99, alpha: float = 1e-3,
            lmin: float = 0.2, lmax: float = 20.0, grad: float = 16.7, shear_ratio: float = 0.6,
            cohesion: float = 5.0, friction: float = 0.6, tvisc: float = 0.01, nuc_half: float = 1.5,
            nuc_dtau: float = 0.0, rkorder: int = 3, sbporder: int = 4, cfl: float = 0.3,
            outputs: Sequence[Output] = ()) -> Problem:
    """3D rough-fault rupture with Drucker-Prager plasticity.

    Two blocks of nx*ny*nz nodes meet on a vertical fault y = ly + r(x, z),
    r from ``rough_surface``; the side faces follow the fault edges so the
    transfinite grids conform.  The free surface is the z+ face (depth
    d = lz - z, km).  Initial volume stress (heterogeneous stress file):
    sxx = syy = szz = -grad*d and sxy = shear_ratio*grad*d MPa, so the fault
    normal stress is -grad*d MPa/km.  Plasticity: cohesion ``cohesion`` MPa,
    internal friction ``friction``, viscosity ``tvisc`` * G (the viscoplastic
    time times the shear modulus).  Slip-weakening friction (0.677, 0.525,
    0.4 m) with a nucleation patch at mid-depth whose shear load is raised to
    ``nuc_dtau`` MPa above the static strength there (0: just above it)."""
    lx, ly, lz = (nx - 1) * h, (ny - 1) * h, (nz - 1) * h
    p = Problem(name=name, ndim=3, mode=2, nx_block=([nx], [ny, ny], [nz]), datadir=datadir, nt=nt,
                cfl=cfl, rkorder=rkorder, sbporder=sbporder)
    p.material = "plastic"
    xs = np.arange(nx) * h
    zs = np.arange(nz) * h
    r = rough_surface(nx, nz, h, alpha, lmin, lmax, seed)
    yf = ly + r   # fault y(x, z)

    def write(tag, arrs):
        fn = os.path.join(workdir, "%s_%s.surf" % (name, tag))
        np.stack(arrs).astype("<f8").tofile(fn)
        return fn

    X2, Z2 = np.meshgrid(xs, zs, indexing="ij")            # (nx, nz)
    fault = write("fault", [X2, yf, Z2])
    sides = {}
    t = np.linspace(0.0, 1.0, ny)
    for b, (y0, y1) in enumerate([(np.zeros_like(yf), yf), (yf, np.full_like(yf, 2 * ly))]):
        # x faces: arrays over (y index, z)
        xm = [np.zeros((ny, nz)), y0[0][None, :] + t[:, None] * (y1[0] - y0[0])[None, :], np.tile(zs, (ny, 1))]
        xp = [np.full((ny, nz), lx), y0[-1][None, :] + t[:, None] * (y1[-1] - y0[-1])[None, :], np.tile(zs, (ny, 1))]
        # z faces: arrays over (x, y index)
        zm = [np.tile(xs[:, None], (1, ny)), y0[:, 0][:, None] + t[None, :] * (y1[:, 0] - y0[:, 0])[:, None],
              np.zeros((nx, ny))]
        zp = [np.tile(xs[:, None], (1, ny)), y0[:, -1][:, None] + t[None, :] * (y1[:, -1] - y0[:, -1])[:, None],
              np.full((nx, ny), lz)]
        youter = np.zeros_like(yf) if b == 0 else np.full_like(yf, 2 * ly)
        outer = write("b%d_y%d" % (b, 0 if b == 0 else 1), [X2, youter, Z2])
        ysurf = [outer, fault] if b == 0 else [fault, outer]
        sides[b] = [write("b%d_x0" % b, xm), write("b%d_x1" % b, xp)] + ysurf + \
                   [write("b%d_z0" % b, zm), write("b%d_z1" % b, zp)]
    eta = tvisc * G
    for b, key in enumerate([(0, 0, 0), (0, 1, 0)]):
        bounds = ["absorbing", "absorbing", "absorbing", "none", "absorbing", "free"] if b == 0 else \
                 ["absorbing", "absorbing", "none", "absorbing", "absorbing", "free"]
        p.blocks[key] = Block(RHO, LAM, G, (0.0, b * ly, 0.0), (lx, ly, lz), bounds, surfaces=sides[b],
                              plastic=(friction, cohesion, 0.0, eta))
    # depth-dependent initial stress, node order (i, j, k) over the whole domain,
    # written one x-plane at a time (the full-size file is several GB)
    dplane = np.broadcast_to((lz - zs)[None, :], (2 * ny, nz))
    planes = {"n": np.ascontiguousarray(-grad * dplane, dtype="<f8"),
              "s": np.ascontiguousarray(shear_ratio * grad * dplane, dtype="<f8"),
              "0": np.zeros((2 * ny, nz), dtype="<f8")}
    sfile = os.path.join(workdir, name + ".stress")
    with open(sfile, "wb") as fh:
        for comp in "ns0n0n":   # sxx, sxy, sxz, syy, syz, szz
            for _ in range(nx):
                planes[comp].tofile(fh)
    p.loadfile = sfile
    itf = Interface("y", (0, 0, 0), (0, 1, 0), "slipweak")
    xc, zc = 0.5 * lx, 0.5 * lz
    dnuc = lz - zc
    extra = (0.677 - shear_ratio) * grad * dnuc + nuc_dtau + 0.5
    itf.loads = [load("boxcar", 0.0, xc, nuc_half, zc, nuc_half, 0.0, extra, 0.0)]
    itf.perts = [swparam("constant", 0.0, 0.0, 0.0, 0.0, 0.0, 0.4, 0.677, 0.525)]
    p.interfaces.append(itf)
    p.outputs = list(outputs)
    return p
