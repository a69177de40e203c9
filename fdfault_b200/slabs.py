"""Host logic of x-slab runs: one problem split along x across GPUs.

The reference runs one MPI rank per subdomain: ``cartesian::cartesian``
(src/cartesian.cpp:88-165) picks the split and ``fields::exchange_neighbors``
(src/fields.cpp:276-291) swaps ghost planes with the neighbours after every
Runge-Kutta stage (called from ``domain::do_rk_stage``, src/domain.cpp:228-305).
Here one process per GPU holds the whole grid on its device and updates the x
planes of its own slab (``Problem.set_x_range``); after every stage it packs
the planes next to each of its cuts into a contiguous device buffer
(``fdf_pack_ghosts``), exchanges the buffers with its neighbours and unpacks
what it receives into its ghost planes (``fdf_unpack_ghosts``).  The exchange
is the only collective on the data path: point-to-point sends between
neighbouring ranks (NCCL over NVLink on GPUs, gloo on CPU), queued on the
stream the solver launches on, so a stage needs no host synchronisation.

Slabs split the work, not the memory: every rank keeps the whole grid and its
geometry (set up identically on every rank, so the time step needs no
reduction), which the 180 GB of a B200 holds for every problem this path runs.

Cuts lie at least ``MARGIN`` planes inside an x block, so that the SBP
closure rows, the x faces and any x-normal interface stay with one slab and
each slab is wider than its ghost planes.  Output units and ``solve`` belong to
whole-domain runs; ``gather_field``/``gather_fault`` assemble the slabs'
values on rank 0 and ``energy`` sums the diagnostics over ranks.
"""

from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

MARGIN = 16   # planes between a cut and the nearest x block face (the solver checks the same)


def x_blocks(problem) -> List[Tuple[int, int]]:
    """Distinct (first x node, x node count) of the problem's blocks, in x order."""
    nb = problem.nblocks[0] * problem.nblocks[1] * problem.nblocks[2]
    out = sorted({(lo[0], n[0]) for lo, n in (problem.block(b) for b in range(nb))})
    return out


def valid_cuts(blocks: Sequence[Tuple[int, int]], margin: int = MARGIN) -> List[int]:
    """Global x positions where a slab may start: at least ``margin`` planes inside a block."""
    cuts: List[int] = []
    for lo, n in blocks:
        cuts.extend(range(lo + margin, lo + n - margin + 1))
    return cuts


def plan_slabs(blocks: Sequence[Tuple[int, int]], world: int, margin: int = MARGIN) -> List[Tuple[int, int]]:
    """Split the x planes of ``blocks`` into ``world`` slabs [x0, x1) of nearly equal width.

    Each cut is the valid position nearest the equal-share one that keeps every
    slab at least ``margin`` planes wide.  Raises ValueError when the grid is
    too narrow for ``world`` slabs."""
    if world < 1:
        raise ValueError("world must be at least 1")
    nx = max(lo + n for lo, n in blocks)
    if world == 1:
        return [(0, nx)]
    cand = np.array(valid_cuts(blocks, margin), dtype=np.int64)
    cuts: List[int] = []
    prev = 0
    for r in range(1, world):
        target = r * nx / world
        # room for this slab (>= margin) and for the slabs after it
        ok = cand[(cand >= prev + margin) & (cand <= nx - (world - r) * margin)]
        if ok.size == 0:
            raise ValueError("x extent %d is too small for %d slabs %d planes from block faces" % (nx, world, margin))
        c = int(ok[np.argmin(np.abs(ok - target))])
        cuts.append(c)
        prev = c
    edges = [0] + cuts + [nx]
    slabs = [(edges[r], edges[r + 1]) for r in range(world)]
    if any(b - a < margin for a, b in slabs):
        raise ValueError("x extent %d is too small for %d slabs" % (nx, world))
    return slabs


def neighbours(rank: int, world: int) -> Dict[int, int]:
    """Side -> neighbouring rank: side 0 the slab below (rank - 1), side 1 the one above."""
    out = {}
    if rank > 0:
        out[0] = rank - 1
    if rank < world - 1:
        out[1] = rank + 1
    return out


class DistTransport:
    """Ghost exchange with the neighbouring ranks over ``torch.distributed``.

    ``exchange(send, recv)`` sends ``send[side]`` to the neighbour on that side
    and receives ``recv[side]`` from it (side 0 below, side 1 above), all
    posted at once; with NCCL the transfers are ordered after the work queued
    on the current stream and the current stream waits for them."""

    def __init__(self, rank: int, world: int, group=None):
        self.rank, self.world, self.group = rank, world, group
        self.peers = neighbours(rank, world)

    def exchange(self, send: Dict[int, "object"], recv: Dict[int, "object"]) -> None:
        import torch.distributed as dist

        ops = []
        for side, peer in self.peers.items():
            ops.append(dist.P2POp(dist.irecv, recv[side], peer, self.group))
            ops.append(dist.P2POp(dist.isend, send[side], peer, self.group))
        if not ops:
            return
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class SlabRun:
    """One rank's slab of a problem, stepped stage by stage with a ghost exchange after each.

    ``problem`` is this rank's ``fdfault_b200.solver.Problem`` (the whole
    grid); ``slabs`` the plan of every rank (``plan_slabs``), by default
    computed from the problem's blocks.  ``transport`` is a ``DistTransport``
    (or None for a single slab).  With ``use_current_stream`` the solver
    launches on torch's current stream of its device, the stream the NCCL
    transfers are ordered against."""

    def __init__(self, problem, rank: int, world: int, transport=None,
                 slabs: Optional[Sequence[Tuple[int, int]]] = None, use_current_stream: bool = True):
        import torch

        self.problem = problem
        self.rank, self.world = rank, world
        self.slabs = list(slabs) if slabs is not None else plan_slabs(x_blocks(problem), world)
        if len(self.slabs) != world:
            raise ValueError("one slab per rank")
        self.x0, self.x1 = self.slabs[rank]
        self.transport = transport
        self.device = problem.torch_device
        problem.set_x_range(self.x0, self.x1)
        self.ghosts, count, elem = problem.ghost_info()
        dtype = torch.float64 if elem == 8 else torch.float32
        self.sides = sorted(neighbours(rank, world))
        self.send = {s: torch.empty(count, dtype=dtype, device=self.device) for s in self.sides}
        self.recv = {s: torch.empty(count, dtype=dtype, device=self.device) for s in self.sides}
        if use_current_stream:
            problem.set_stream(torch.cuda.current_stream(self.device).cuda_stream)
        self.exchanges = 0

    @property
    def ghost_bytes_per_exchange(self) -> int:
        """Bytes this rank sends per exchange (both sides)."""
        return sum(t.numel() * t.element_size() for t in self.send.values())

    def pack(self) -> None:
        for s in self.sides:
            self.problem.pack_ghosts(s, self.send[s].data_ptr())

    def unpack(self) -> None:
        for s in self.sides:
            self.problem.unpack_ghosts(s, self.recv[s].data_ptr())

    def exchange(self) -> None:
        if not self.sides:
            return
        self.pack()
        self.transport.exchange(self.send, self.recv)
        self.unpack()
        self.exchanges += 1

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            for st in range(self.problem.nstages):
                self.problem.step_stage(st)
                self.exchange()

    def release(self) -> None:
        """Back to the whole domain on the problem's own stream."""
        self.problem.set_stream(None)
        self.problem.set_x_range(0, self.problem.nx[0])

    # --- results on rank 0 ---------------------------------------------
    def _gather_rows(self, full: np.ndarray, rows_of) -> Optional[np.ndarray]:
        """Rank 0: ``full`` with every rank's own rows (``rows_of(x0, x1)``, an index array) filled in."""
        import torch
        import torch.distributed as dist

        if self.world == 1:
            return full
        dev = self.device if dist.get_backend() == "nccl" else torch.device("cpu")
        if self.rank != 0:
            idx = rows_of(self.x0, self.x1)
            if idx.size:   # every rank knows which ranks own no rows
                dist.send(torch.from_numpy(np.ascontiguousarray(full[idx])).to(dev), 0)
            return None
        out = full.copy()
        for r in range(1, self.world):
            idx = rows_of(*self.slabs[r])
            if not idx.size:
                continue
            buf = torch.empty(full[idx].shape, dtype=torch.float64, device=dev)
            dist.recv(buf, r)
            out[idx] = buf.cpu().numpy()
        return out

    def gather_field(self, comp: int, absolute: bool = False) -> Optional[np.ndarray]:
        """Field component ``comp`` of the whole domain on rank 0 (None elsewhere)."""
        nx, ny, nz = self.problem.nx
        full = self.problem.field(comp, absolute).reshape(nx, ny * nz)
        out = self._gather_rows(full, lambda a, b: np.arange(a, b))
        return None if out is None else out.reshape(-1)

    def gather_fault(self, iface: int, which: int) -> Optional[np.ndarray]:
        """Fault array ``which`` of interface ``iface`` on rank 0 (None elsewhere)."""
        full = self.problem.fault(iface, which)
        d, lo, (n0, n1) = self.problem.interface(iface)
        ncomp = full.size // (n0 * n1)
        rows = full.reshape(ncomp * n0, n1)
        if d == 0:   # an x-normal fault lies on one plane: its slab's rank has all of it
            def rows_of(a, b):
                return np.arange(ncomp * n0) if a <= lo[0] < b else np.arange(0)
        else:
            def rows_of(a, b):
                xs = np.arange(n0) + lo[0]
                mine = np.nonzero((xs >= a) & (xs < b))[0]
                return (np.arange(ncomp)[:, None] * n0 + mine[None, :]).reshape(-1)
        out = self._gather_rows(rows, rows_of)
        return None if out is None else out.reshape(-1)

    def energy(self, rate: bool = True) -> Dict[str, float]:
        """The energy diagnostics of the whole domain on every rank (sums over the slabs)."""
        import torch
        import torch.distributed as dist

        e = self.problem.energy(rate)
        if self.world == 1:
            return e
        keys = ["kinetic", "strain", "rate", "rate_scale", "friction_power"]
        dev = self.device if dist.get_backend() == "nccl" else torch.device("cpu")
        t = torch.tensor([e[k] for k in keys], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        out = dict(zip(keys, t.cpu().tolist()))
        out["total"] = out["kinetic"] + out["strain"]
        return out


class LocalSlabs:
    """Several slabs of one problem in one process, each a separate ``Problem``
    on the same device, exchanging ghost planes by device copies.

    The same pack and unpack calls as ``SlabRun`` with the transport replaced
    by a copy between the slabs' buffers, for checking a split against the
    whole-domain run on one GPU.  The slabs run one after another (no kernel
    waits on another slab's kernel)."""

    def __init__(self, problems: Sequence, slabs: Optional[Sequence[Tuple[int, int]]] = None, stream=None):
        """``stream``: a ``torch.cuda.Stream`` on which every slab launches
        (``Problem.set_stream``, as a rank of a multi-GPU run launches on the
        stream its NCCL transfers are ordered against), with the copies queued
        on it too; None keeps each slab on its own stream and synchronises
        around the copies."""
        import torch

        self.problems = list(problems)
        world = len(self.problems)
        self.slabs = list(slabs) if slabs is not None else plan_slabs(x_blocks(self.problems[0]), world)
        self.stream = stream
        self.runs = []
        for r, p in enumerate(self.problems):
            if stream is None:
                self.runs.append(SlabRun(p, r, world, transport=None, slabs=self.slabs, use_current_stream=False))
            else:
                with torch.cuda.stream(stream):
                    self.runs.append(SlabRun(p, r, world, transport=None, slabs=self.slabs))
        self.torch = torch

    def _copies(self) -> None:
        runs = self.runs
        for i, r in enumerate(runs):
            if 0 in r.sides:
                r.recv[0].copy_(runs[i - 1].send[1])
            if 1 in r.sides:
                r.recv[1].copy_(runs[i + 1].send[0])

    def exchange(self) -> None:
        runs = self.runs
        if self.stream is not None:   # one stream orders everything
            with self.torch.cuda.stream(self.stream):
                for r in runs:
                    r.pack()
                self._copies()
                for r in runs:
                    r.unpack()
            return
        for r in runs:
            r.pack()
        for r in runs:
            r.problem.synchronize()
        self._copies()
        self.torch.cuda.synchronize(runs[0].device)
        for r in runs:
            r.unpack()

    def step(self, nsteps: int = 1) -> None:
        nst = self.problems[0].nstages
        for _ in range(nsteps):
            for st in range(nst):
                for r in self.runs:
                    r.problem.step_stage(st)
                self.exchange()
        for r in self.runs:
            r.problem.synchronize()

    def field(self, comp: int, absolute: bool = False) -> np.ndarray:
        nx, ny, nz = self.problems[0].nx
        out = np.empty((nx, ny * nz))
        for r in self.runs:
            out[r.x0:r.x1] = r.problem.field(comp, absolute).reshape(nx, ny * nz)[r.x0:r.x1]
        return out.reshape(-1)

    def fault(self, iface: int, which: int) -> np.ndarray:
        p0 = self.problems[0]
        d, lo, (n0, n1) = p0.interface(iface)
        parts = [r.problem.fault(iface, which) for r in self.runs]
        ncomp = parts[0].size // (n0 * n1)
        out = np.empty((ncomp, n0, n1))
        for r, part in zip(self.runs, parts):
            a = part.reshape(ncomp, n0, n1)
            if d == 0:
                if r.x0 <= lo[0] < r.x1:
                    out[:] = a
            else:
                xs = np.arange(n0) + lo[0]
                m = (xs >= r.x0) & (xs < r.x1)
                out[:, m] = a[:, m]
        return out.reshape(-1)
