"""Multi-GPU form on CPU: two gloo ranks each classify their shard of the reads against their
own index replica (the CPU restatement stands in for the device here) and the gathered results
equal the single-process results."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from mirage_b200.shard import shard_batch, shard_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, mhm, bases, offs, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle as O

    b, o, lo = shard_batch(bases, offs, rank, world)
    res = O.Index(mhm).classify(b, o)
    got = [None] * world
    dist.all_gather_object(got, (lo, res.merged))
    if rank == 0:
        merged = []
        for lo_r, m in sorted(got, key=lambda x: x[0]):
            merged += [(lo_r + i, s, h, t) for (i, s, h, t) in m]
        out.put(merged)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_ranges_cover_all():
    for n in (0, 1, 7, 100, 101):
        for w in (1, 2, 3, 8):
            rs = [shard_range(n, r, w) for r in range(w)]
            assert rs[0][0] == 0 and rs[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            assert max(h - l for l, h in rs) - min(h - l for l, h in rs) <= 1


def test_two_rank_replicas_match_single(golden):
    from oracle import oracle as O

    g = golden("uneven_small")
    bases, offs = g.reads.data, g.reads.offs
    full = O.Index(g.mhm_path).classify(bases, offs).merged
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, g.mhm_path, bases, offs, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=300)
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert merged == full
