"""Multi-GPU host logic on CPU: two gloo ranks split a list of ensemble members
(disjoint, covering, balanced) and reduce their reported work (sum) and
device time (max), as bench.py does over NCCL with one rank per GPU."""

import os
import socket
import tempfile

import pytest
import torch.multiprocessing as mp

from fdfault_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, outdir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        items = ["member%03d" % i for i in range(11)]
        mine = replicas.partition(items, rank, world)
        work = 100.0 * len(mine)
        ms = 10.0 + rank
        tot, slow = replicas.reduce_totals(work, ms)
        with open(os.path.join(outdir, "r%d.txt" % rank), "w") as fh:
            fh.write("%s\n%r %r\n" % (",".join(mine), tot, slow))
    finally:
        dist.destroy_process_group()


def test_partition_is_disjoint_covering_balanced():
    items = list(range(257))
    parts = [replicas.partition(items, r, 4) for r in range(4)]
    flat = sorted(x for p in parts for x in p)
    assert flat == items
    assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        replicas.partition(items, 4, 4)


def test_reduce_without_process_group_is_identity():
    assert replicas.reduce_totals(3.0, 2.5) == (3.0, 2.5)


def test_two_gloo_ranks():
    out = tempfile.mkdtemp(prefix="fdf_gloo_")
    port = _free_port()
    mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = [open(os.path.join(out, "r%d.txt" % r)).read().split("\n") for r in range(2)]
    mine = [g[0].split(",") for g in got]
    assert set(mine[0]).isdisjoint(mine[1])
    assert len(mine[0]) + len(mine[1]) == 11
    for g in got:
        tot, slow = (float(v) for v in g[1].split())
        assert tot == 1100.0 and slow == 11.0
