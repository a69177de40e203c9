"""x-slab host logic on CPU: the slab plan, and gloo ranks that step slabs of
a stand-in problem with a ghost exchange after every stage, against the
same problem stepped whole.

The stand-in has the data dependencies of the solver's stage: two field
buffers swapped every stage, an x stencil that reads `ghosts` planes on each
side, and updates written only inside the slab, so that a missing, stale or
misplaced ghost plane changes the result."""

import ctypes
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from fdfault_b200 import slabs


class StandIn:
    """Duck-typed stand-in for ``solver.Problem`` on host memory."""

    nstages = 3
    ghosts = 2

    def __init__(self, nx=53, m=6, nfields=3, seed=7):
        self.nx = (nx, m, 1)
        self.nblocks = (1, 1, 1)
        self.device = 0
        self.torch_device = torch.device("cpu")
        rng = np.random.default_rng(seed)
        self.F = [rng.standard_normal((nfields, nx, m)), np.zeros((nfields, nx, m))]
        self.cur = 0
        self.x0, self.x1 = 0, nx
        self.step_index = 0
        self.next = 0

    def block(self, b):
        return (0, 0, 0), self.nx

    def set_x_range(self, x0, x1):
        self.x0, self.x1 = x0, x1

    def ghost_info(self):
        nf, _, m = self.F[0].shape
        return self.ghosts, nf * self.ghosts * m, 8

    def step_stage(self, st):
        assert st == self.next
        old, new = self.F[self.cur], self.F[1 - self.cur]
        nx = self.nx[0]
        for i in range(self.x0, self.x1):
            acc = old[:, i].copy()
            for d in range(1, self.ghosts + 1):
                acc += (0.11 * d) * (old[:, min(i + d, nx - 1)] - old[:, max(i - d, 0)])
            new[:, i] = np.tanh(acc) + 0.01 * (st + 1)
        self.cur = 1 - self.cur
        self.next = (st + 1) % self.nstages
        if self.next == 0:
            self.step_index += 1

    def _planes(self, side, ghost):
        g = self.ghosts
        if ghost:
            return slice(self.x0 - g, self.x0) if side == 0 else slice(self.x1, self.x1 + g)
        return slice(self.x0, self.x0 + g) if side == 0 else slice(self.x1 - g, self.x1)

    def pack_ghosts(self, side, ptr):
        a = np.ascontiguousarray(self.F[self.cur][:, self._planes(side, False)])
        ctypes.memmove(ptr, a.ctypes.data, a.nbytes)

    def unpack_ghosts(self, side, ptr):
        sl = self._planes(side, True)
        shape = self.F[self.cur][:, sl].shape
        buf = (ctypes.c_double * int(np.prod(shape))).from_address(ptr)
        self.F[self.cur][:, sl] = np.frombuffer(buf, dtype=np.float64).reshape(shape)

    def field(self, comp, absolute=False):
        return self.F[self.cur][comp].reshape(-1).copy()

    # a fault: direction 1 spans every x plane (row a at x = a), direction 0
    # lies on plane `xplane` (rows along the other axis); two components
    fault_dir = 1
    xplane = 31

    def interface(self, i):
        nx, m, _ = self.nx
        if self.fault_dir == 1:
            return 1, (0, 0, 0), (nx, m)
        return 0, (self.xplane, 0, 0), (m, 1)

    def fault(self, i, which):
        f = self.F[self.cur]
        if self.fault_dir == 1:
            return np.concatenate([f[0], f[1] * which]).reshape(-1)
        return np.concatenate([f[0, self.xplane], f[1, self.xplane] * which]).reshape(-1)

    def energy(self, rate=True):
        f = self.F[self.cur][:, self.x0:self.x1]
        return {"kinetic": float(np.sum(f[0] ** 2)), "strain": float(np.sum(f[1] ** 2)),
                "rate": float(np.sum(f[2])), "rate_scale": 1.0, "friction_power": float(np.sum(f[0] * f[1]))}


ENERGY_KEYS = ("kinetic", "strain", "total", "rate", "friction_power")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir, nsteps):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = StandIn()
        run = slabs.SlabRun(p, rank, world, transport=slabs.DistTransport(rank, world), use_current_stream=False)
        run.step(nsteps)
        for comp in range(3):
            f = run.gather_field(comp)
            if rank == 0:
                np.save(os.path.join(outdir, "f%d.npy" % comp), f)
        for d in (1, 0):
            p.fault_dir = d
            f = run.gather_fault(0, 3)
            if rank == 0:
                np.save(os.path.join(outdir, "fault%d.npy" % d), f)
        e = run.energy()
        if rank == 0:
            np.save(os.path.join(outdir, "energy.npy"), np.array([e[k] for k in ENERGY_KEYS]))
        with open(os.path.join(outdir, "r%d.txt" % rank), "w") as fh:
            fh.write("%d %d %d %d\n" % (run.x0, run.x1, run.exchanges, p.step_index))
    finally:
        dist.destroy_process_group()


def test_plan_balanced_and_inside_blocks():
    plan = slabs.plan_slabs([(0, 401)], 8)
    assert plan[0][0] == 0 and plan[-1][1] == 401
    assert all(a[1] == b[0] for a, b in zip(plan, plan[1:]))
    widths = [b - a for a, b in plan]
    assert max(widths) - min(widths) <= 1
    # two x blocks: no cut within 16 planes of a block face
    plan = slabs.plan_slabs([(0, 100), (100, 60)], 4)
    for a, _ in plan[1:]:
        assert 16 <= a <= 84 or 116 <= a <= 144
    assert slabs.plan_slabs([(0, 30)], 1) == [(0, 30)]
    with pytest.raises(ValueError):
        slabs.plan_slabs([(0, 40)], 3)
    assert slabs.neighbours(0, 3) == {1: 1} and slabs.neighbours(1, 3) == {0: 0, 1: 2}


def test_plan_properties_on_random_block_layouts():
    # any x block layout and rank count: either a plan whose slabs tile
    # [0, nx), each at least 16 planes wide with every cut at least 16 planes
    # inside a block, or ValueError when no such plan exists for that count
    rng = np.random.default_rng(11)
    for _ in range(300):
        sizes = rng.integers(20, 300, size=rng.integers(1, 4))
        blocks, lo = [], 0
        for n in sizes:
            blocks.append((lo, int(n)))
            lo += int(n)
        nx = lo
        world = int(rng.integers(1, 12))
        try:
            plan = slabs.plan_slabs(blocks, world)
        except ValueError:
            # one block of n planes has a plan exactly when n >= 16 * world
            assert len(blocks) > 1 or nx < 16 * world
            continue
        assert len(blocks) > 1 or nx >= 16 * world or world == 1
        assert len(plan) == world and plan[0][0] == 0 and plan[-1][1] == nx
        assert all(a[1] == b[0] for a, b in zip(plan, plan[1:]))
        assert all(b - a >= 16 for a, b in plan) or world == 1
        for a, _ in plan[1:]:
            assert any(lo0 + 16 <= a <= lo0 + n - 16 for lo0, n in blocks)
        if len(blocks) == 1 and world > 1:   # one block: within a plane of the equal share
            assert max(b - a for a, b in plan) - min(b - a for a, b in plan) <= 1


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_slabs_match_whole_domain(world):
    nsteps = 4
    whole = StandIn()
    for _ in range(nsteps):
        for st in range(whole.nstages):
            whole.step_stage(st)
    out = tempfile.mkdtemp(prefix="fdf_slab_")
    mp.start_processes(_rank, args=(world, _free_port(), out, nsteps), nprocs=world, join=True,
                       start_method="spawn")
    for comp in range(3):
        got = np.load(os.path.join(out, "f%d.npy" % comp))
        assert np.array_equal(got, whole.field(comp))
    for d in (1, 0):
        whole.fault_dir = d
        assert np.array_equal(np.load(os.path.join(out, "fault%d.npy" % d)), whole.fault(0, 3))
    e = whole.energy()
    e["total"] = e["kinetic"] + e["strain"]
    np.testing.assert_allclose(np.load(os.path.join(out, "energy.npy")), [e[k] for k in ENERGY_KEYS],
                               rtol=1e-13)
    rows = [open(os.path.join(out, "r%d.txt" % r)).read().split() for r in range(world)]
    assert [int(r[0]) for r in rows][0] == 0 and int(rows[-1][1]) == whole.nx[0]
    for r in rows:
        assert int(r[2]) == nsteps * whole.nstages and int(r[3]) == nsteps


def test_missing_exchange_is_detected():
    # the stand-in is sensitive to its ghosts: slabs stepped without the
    # exchange differ from the whole run
    whole, a, b = StandIn(), StandIn(), StandIn()
    a.set_x_range(0, 26)
    b.set_x_range(26, 53)
    for st in range(whole.nstages):
        for p in (whole, a, b):
            p.step_stage(st)
    merged = np.concatenate([a.F[a.cur][0, :26], b.F[b.cur][0, 26:]])
    assert not np.array_equal(merged, whole.F[whole.cur][0])
