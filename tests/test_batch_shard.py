"""The batched path across GPUs shards with no communication (independent
graphs): every rank computes the same greedy edge-balanced assignment of
the 4096-graph mix.  Checked with two gloo ranks on the CPU: the shards are
disjoint, cover the mix, agree between ranks, and their loads differ by at
most the largest graph."""
from __future__ import annotations

import os

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

import kaspan_b200 as K
import kaspan_b200.graphs as KG


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n, d = K.batch_shape(4096, 5)
    work = n.astype(np.float64) + d.astype(np.float64)
    parts = KG.batch_partition(work, world)
    got = [None] * world
    dist.all_gather_object(got, [p.tolist() for p in parts])
    if rank == 0:
        q.put((got, work.tolist()))
    dist.destroy_process_group()


def test_two_ranks_agree_and_balance():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got, work = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    work = np.array(work)
    assert got[0] == got[1]
    shards = [np.array(s) for s in got[0]]
    allg = np.concatenate(shards)
    assert len(allg) == 4096 and len(np.unique(allg)) == 4096
    loads = [work[s].sum() for s in shards]
    assert abs(loads[0] - loads[1]) <= work.max()
