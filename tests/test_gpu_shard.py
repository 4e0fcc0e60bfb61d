"""GPU: the sharded decomposition (kaspan_b200/shard.py) with the CUDA
steps (kspn_shard_* and, for the residual, the single-GPU pipeline),
compared with the oracle Tarjan of the whole graph.  One rank in-process;
then two ranks as two processes on the one GPU of this run, exchanging
through gloo on the host (their kernels never wait on one another: every
exchange is a host collective between launches).  Between GPUs the same
loop runs its exchanges over NCCL."""
from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest

import oracle as O
from kaspan_b200 import shard as SH

pytestmark = pytest.mark.gpu

GRAPHS = {
    "rmat12": lambda: O.rmat(12, 8, 3),
    "rgg12": lambda: O.rgg(1 << 12, 6),
    "gnm": lambda: O.gnm(3000, 9000, 9),
    "fuzzy": lambda: O.fuzzy(777, 280, 1.0)[0],
}


def _shard(G, rank, world):
    import torch

    bounds = SH.partition_bounds(G.n, G.fwh, world)
    lo, hi = bounds[rank], bounds[rank + 1]
    fwh, fwc = SH.slice_rows(G.fwh, G.fwc[: G.m], lo, hi)
    bwh, bwc = SH.slice_rows(G.bwh, G.bwc[: G.m], lo, hi)
    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a).view(dt).copy() if a.size else np.zeros(1, dt)).cuda()  # noqa: E731
    return SH.Shard(G.n, rank, world, bounds, t(fwh, np.int64), t(fwc, np.int32), t(bwh, np.int64), t(bwc, np.int32))


def _run_rank(ctx, G, rank, world):
    S = _shard(G, rank, world)
    st = SH.ShardStats()
    ids = SH.scc_sharded(SH.CudaShardOps(ctx, S), SH.Exchange(), S, stats=st)
    return S.lo, ids.cpu().numpy().view(np.uint32).copy(), st


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_sharded_one_rank(ctx, name):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("gloo", rank=0, world_size=1, timeout=datetime.timedelta(seconds=90))
    try:
        G = GRAPHS[name]()
        lo, ids, st = _run_rank(ctx, G, 0, 1)
        assert np.array_equal(ids, O.tarjan(G))
        assert st.decided_trim + st.decided_fwbw + st.decided_residual == G.n
    finally:
        dist.destroy_process_group()


def _rank_main(rank, world, port, name, q):
    import torch
    import torch.distributed as dist

    import kaspan_b200 as K

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=90))
    try:
        with K.Context(0) as ctx:
            G = GRAPHS[name]()
            lo, ids, st = _run_rank(ctx, G, rank, world)
            q.put((rank, lo, ids.tolist(), st.exchanged, st.rounds))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", sorted(GRAPHS))
def test_sharded_two_ranks_one_gpu(name):
    import multiprocessing as mp

    c = mp.get_context("spawn")
    q = c.Queue()
    port = _free_port()
    procs = [c.Process(target=_rank_main, args=(r, 2, port, name, q), daemon=True) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = [q.get(timeout=240) for _ in range(2)]
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
    finally:
        for p in procs:
            if p.is_alive():
                p.terminate()
                p.join(timeout=30)
    G = GRAPHS[name]()
    ids = np.full(G.n, 0xFFFFFFFF, np.uint32)
    for rank, lo, part, exchanged, rounds in got:
        ids[lo: lo + len(part)] = part
    assert np.array_equal(ids, O.tarjan(G))
    assert sum(g[3] for g in got) > 0, "ids should cross the two shards"
