"""CPU: the sharded decomposition's host loop (kaspan_b200/shard.py) over
gloo ranks, world sizes 2 and 3, each rank holding one contiguous vertex
range of the graph.  The device steps are replaced by HostShardOps below, a
plain restatement of what each kspn_shard_* entry point computes (test
infrastructure only), so the partition, the frontier exchange (counts, then
ids, all-to-all), the all-reduces and the residual gather are checked
without a GPU; the union of the ranks' ids must equal the oracle Tarjan of
the whole graph.  The GPU test (test_gpu_shard.py) runs the same loop with
the CUDA steps."""
from __future__ import annotations

import datetime
import os
import socket

import numpy as np
import pytest

import oracle as O
from kaspan_b200 import shard as SH

UNDECIDED = SH.UNDECIDED


class HostShardOps:
    """The kspn_shard_* steps restated on the host (torch CPU tensors)."""

    def __init__(self, S: SH.Shard):
        self.S = S
        self.fwh, self.fwc = np.asarray(S.fwh, np.int64), np.asarray(S.fwc, np.int64)
        self.bwh, self.bwc = np.asarray(S.bwh, np.int64), np.asarray(S.bwc, np.int64)
        self.und = np.zeros(S.n_loc, bool)
        self.ids = np.full(S.n_loc, UNDECIDED, np.int64)
        self.front = [[], []]
        self.next = [[], []]

    def _deg(self, v):
        return (self.fwh[v + 1] - self.fwh[v]) * (self.bwh[v + 1] - self.bwh[v])

    def _best(self, mask):
        best, vid = 0, UNDECIDED
        for v in np.nonzero(mask)[0]:
            p = int(self._deg(v))
            if p > best:
                best, vid = p, self.S.lo + int(v)
        return best, vid

    def trim_first(self):  # kaspan/scc/trim_1_local.hpp:12-46 on the local rows
        out = self.fwh[1:] - self.fwh[:-1]
        inn = self.bwh[1:] - self.bwh[:-1]
        self.und = (out > 0) & (inn > 0)
        dec = np.nonzero(~self.und)[0]
        self.ids[dec] = self.S.lo + dec
        best, vid = self._best(self.und)
        return int(dec.size), best, vid

    def pivot(self):
        return self._best(self.und)

    def search_begin(self):
        self.cand = [self.und.copy(), self.und.copy()]
        self.vis = [np.zeros(self.S.n_loc, bool), np.zeros(self.S.n_loc, bool)]
        self.sent = [set(), set()]
        self.front = [[], []]
        self.next = [[], []]

    def receive(self, d, ids):
        for u in (int(x) for x in ids):
            lu = u - self.S.lo
            assert 0 <= lu < self.S.n_loc, "an id sent to the wrong shard"
            if self.cand[d][lu]:
                self.cand[d][lu] = False
                self.vis[d][lu] = True
                self.next[d].append(lu)

    def expand(self, d):
        import torch

        head, adj = (self.fwh, self.fwc) if d == 0 else (self.bwh, self.bwc)
        S = self.S
        remote = []
        for v in self.front[d]:
            for u in adj[head[v]: head[v + 1]]:
                u = int(u)
                if S.lo <= u < S.hi:
                    self.receive(d, [u])
                elif u not in self.sent[d]:
                    self.sent[d].add(u)
                    remote.append(u)
        owner = np.searchsorted(np.asarray(S.bounds), np.asarray(remote, np.int64), side="right") - 1
        order = np.argsort(owner, kind="stable")
        counts = [int((owner == r).sum()) for r in range(S.parts)]
        return torch.tensor(np.asarray(remote, np.int64)[order], dtype=torch.int32), counts

    def advance(self, d):
        self.front[d], self.next[d] = self.next[d], []
        return len(self.front[d])

    def scc_min(self):
        both = np.nonzero(self.vis[0] & self.vis[1])[0]
        return self.S.lo + int(both[0]) if both.size else UNDECIDED

    def finalize(self, scc):
        both = np.nonzero(self.vis[0] & self.vis[1] & self.und)[0]
        self.und[both] = False
        self.ids[both] = scc
        return int(both.size)

    def und_words(self):
        import torch

        bits = np.zeros(((self.S.n_loc + 31) // 32) * 32, np.uint32)
        bits[: self.S.n_loc] = self.und
        w = (bits.reshape(-1, 32) << np.arange(32, dtype=np.uint32)).sum(axis=1, dtype=np.uint64).astype(np.uint32)
        return torch.from_numpy(w.view(np.int32).copy())

    def residual_edges(self, gund):
        import torch

        g = gund.numpy().view(np.uint32)
        src, dst = [], []
        for v in np.nonzero(self.und)[0]:
            for u in self.fwc[self.fwh[v]: self.fwh[v + 1]]:
                if (g[u >> 5] >> (u & 31)) & 1:
                    src.append(self.S.lo + int(v))
                    dst.append(int(u))
        return torch.tensor(src, dtype=torch.int32), torch.tensor(dst, dtype=torch.int32)

    def solve_residual(self, k, src, dst):
        import torch

        G = O.from_edges(k, src.numpy().astype(np.uint32), dst.numpy().astype(np.uint32))
        return torch.from_numpy(O.tarjan(G).astype(np.int64))

    def set_ids(self, pos, values):
        self.ids[pos.numpy()] = values.numpy()

    def local_ids(self):
        return self.ids


def _graphs():
    fz, _ = O.fuzzy(4242, 300, 1.0)
    # chains of cycles joined one way (many SCCs, FW and BW both cross shards)
    src, dst, base = [], [], 0
    for ln in range(1, 40):
        src += [base + i for i in range(ln)]
        dst += [base + (i + 1) % ln for i in range(ln)]
        if base:
            src.append(base - 1), dst.append(base)
        base += ln
    chains = O.from_edges(base, np.asarray(src, np.uint32), np.asarray(dst, np.uint32))
    return {"rmat10": O.rmat(10, 8, 3), "gnm": O.gnm(1500, 4000, 9), "fuzzy": fz, "chains": chains, "kat": None}


def _rank_main(rank, world, port, name, q):
    import torch.distributed as dist

    from kspn_testlib import kat_graph

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=90))
    try:
        G = _graphs()[name] or kat_graph()
        bounds = SH.partition_bounds(G.n, G.fwh, world, align=64)
        lo, hi = bounds[rank], bounds[rank + 1]
        fwh, fwc = SH.slice_rows(G.fwh, G.fwc[: G.m], lo, hi)
        bwh, bwc = SH.slice_rows(G.bwh, G.bwc[: G.m], lo, hi)
        S = SH.Shard(G.n, rank, world, bounds, fwh, fwc, bwh, bwc)
        st = SH.ShardStats()
        ids = SH.scc_sharded(HostShardOps(S), SH.Exchange(), S, stats=st)
        q.put((rank, lo, [int(x) for x in ids], st.rounds, st.exchanged))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("name", ["rmat10", "gnm", "fuzzy", "chains", "kat"])
def test_sharded_loop_matches_tarjan(world, name):
    import multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, name, q), daemon=True) for r in range(world)]
    for p in procs:
        p.start()
    try:
        got = [q.get(timeout=240) for _ in range(world)]
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
    finally:
        for p in procs:
            if p.is_alive():
                p.terminate()
                p.join(timeout=30)
    from kspn_testlib import kat_graph

    G = _graphs()[name] or kat_graph()
    ids = np.full(G.n, UNDECIDED, np.int64)
    for rank, lo, part, rounds, exchanged in got:
        ids[lo: lo + len(part)] = part
    assert np.array_equal(ids.astype(np.uint32), O.tarjan(G))
    # the ranges really were split (more than one rank owns vertices) and ids crossed ranks
    if G.n >= 64 * world:
        assert sum(1 for r in got if len(r[2]) > 0) > 1
        assert sum(r[4] for r in got) > 0


def test_partition_bounds_balance_and_alignment():
    G = O.rmat(12, 8, 5)
    for parts in (1, 2, 3, 8):
        b = SH.partition_bounds(G.n, G.fwh, parts)
        assert b[0] == 0 and b[-1] == G.n and all(x <= y for x, y in zip(b, b[1:]))
        assert all(x % 64 == 0 for x in b[:-1])
        cost = [(b[r + 1] - b[r]) + int(G.fwh[b[r + 1]] - G.fwh[b[r]]) for r in range(parts)]
        assert max(cost) <= (G.n + G.m) / parts + 64 + G.fwh[-1] / G.n * 64 * 4
