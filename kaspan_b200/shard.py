"""One graph over several GPUs: the sharded decomposition (one process per GPU).

Reference: the distributed ``kaspan::scc`` (kaspan/scc/scc.hpp:21-87) on a 1D
vertex partition.  Rank r owns the contiguous vertex range [lo, hi) and its
rows of the forward CSR and of the transpose, with global neighbour ids
(kaspan/graph/bidi_graph_part.hpp:12-28); the searches exchange frontier
messages every iteration (``frontier::comm``, kaspan/scc/frontier.hpp:237-282:
an all-to-all of the counts, then of the payload) and phases end with an
all-reduce of the decided count (kaspan/util/mpi_basic.hpp).

Here every rank runs, in lockstep:

1. ``trim_1_first`` on its rows (kaspan/scc/trim_1_local.hpp:12-46) and an
   all-gather of the ranks' best (in * out, id): the pivot is the largest
   product, smallest id on ties (the reference's rule at one rank);
2. rounds of FW-BW from the pivot: both searches top-down, one level at a
   time; a level expands the local frontier, sends the remote finds to their
   owners (counts, then ids: ``all_to_all_single`` twice), takes the
   received ids as local finds; the searches end when an all-reduce of the
   frontier sizes is 0.  The SCC is FW & BW, named after its smallest
   member (an all-reduce MIN); a round that decides less than 1/64 of the
   remaining vertices ends the rounds (the next pivot: the largest in * out
   of the undecided vertices, all-gathered);
3. the residual: the undecided vertices (an all-gather of the ranks'
   bitmap words) and the edges between them (an all-gather of each rank's
   part, the local half of ``allgather_fw_sub_graph``,
   kaspan/scc/allgather_sub_graph.hpp:253-301) form one graph that every rank
   decomposes whole; each keeps its own vertices' ids.

The device steps are the library's ``kspn_shard_*`` entry points
(``CudaShardOps``); torch.distributed carries the exchanges -- NCCL between
GPUs, gloo (on host copies) when the ranks share a device or run on CPU.
The loop only sees the ``ops`` interface, so the tests drive the same loop
with a CPU stand-in of the steps over gloo ranks.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

UNDECIDED = 0xFFFFFFFF
WORD_ALIGN = 64  # shard boundaries: whole u64 words of the reference's bitset layout


def partition_bounds(n: int, fw_head: np.ndarray, parts: int, align: int = WORD_ALIGN) -> list[int]:
    """Contiguous ranges balanced by rows + edges: bounds[r] is the first
    vertex whose cost (its id + its first edge's offset) reaches r / parts
    of the total, rounded down to a multiple of `align` (a shard's bitmap
    words are then whole words of the global one).  bounds[0] = 0,
    bounds[parts] = n; ranges may be empty on tiny graphs."""
    fw_head = np.asarray(fw_head, dtype=np.uint64)
    total = float(n) + float(fw_head[n])
    cost = np.arange(n + 1, dtype=np.float64) + fw_head[: n + 1].astype(np.float64)
    bounds = [0]
    for r in range(1, parts):
        v = int(np.searchsorted(cost, total * r / parts, side="left"))
        v = min(n, (v // align) * align)
        bounds.append(max(v, bounds[-1]))
    bounds.append(n)
    return bounds


@dataclass
class Shard:
    """One rank's part of the graph: vertices [lo, hi) of n; heads with
    local offsets (hi - lo + 1 entries), rows with global ids."""

    n: int
    rank: int
    parts: int
    bounds: list
    fwh: object
    fwc: object
    bwh: object
    bwc: object

    @property
    def lo(self) -> int:
        return self.bounds[self.rank]

    @property
    def hi(self) -> int:
        return self.bounds[self.rank + 1]

    @property
    def n_loc(self) -> int:
        return self.hi - self.lo


def slice_rows(head: np.ndarray, csr: np.ndarray, lo: int, hi: int):
    """Rows [lo, hi) of a host CSR: (local head, rows)."""
    b, e = int(head[lo]), int(head[hi])
    return (head[lo: hi + 1] - head[lo]).astype(np.uint64), np.ascontiguousarray(csr[b:e], dtype=np.uint32)


class Exchange:
    """The collectives of the sharded loop over a torch.distributed group.
    With the gloo backend device tensors travel through host copies."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.host = dist.get_backend(group) == "gloo"

    def _to(self, t):
        return t.cpu() if self.host and t.is_cuda else t

    def sum(self, values) -> list:
        import torch

        dev = "cpu" if self.host else "cuda"
        t = torch.tensor([int(v) for v in values], dtype=torch.int64, device=dev)
        self.dist.all_reduce(t, group=self.group)
        return [int(x) for x in t.tolist()]

    def min(self, value: int) -> int:
        import torch

        dev = "cpu" if self.host else "cuda"
        t = torch.tensor([int(value)], dtype=torch.int64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MIN, group=self.group)
        return int(t.item())

    def pivot(self, prod: int, vid: int) -> int:
        """The ranks' (in * out, id) candidates -> the largest product,
        smallest id on ties; UNDECIDED when every product is 0."""
        import torch

        dev = "cpu" if self.host else "cuda"
        mine = torch.tensor([prod >> 32, prod & 0xFFFFFFFF, vid], dtype=torch.int64, device=dev)
        got = [torch.zeros_like(mine) for _ in range(self.world)]
        self.dist.all_gather(got, mine, group=self.group)
        best = None
        for g in got:
            p, v = (int(g[0]) << 32) | int(g[1]), int(g[2])
            if p and (best is None or p > best[0] or (p == best[0] and v < best[1])):
                best = (p, v)
        return UNDECIDED if best is None else best[1]

    def all_to_all(self, send, counts: list):
        """Payload `send` (grouped by destination, counts[r] ids for rank r)
        -> the ids the other ranks sent here (same dtype and device)."""
        import torch

        dev = "cpu" if self.host else send.device
        c = torch.tensor(counts, dtype=torch.int64, device=dev)
        rc = torch.empty_like(c)
        self.dist.all_to_all_single(rc, c, group=self.group)
        rcl = [int(x) for x in rc.tolist()]
        payload = self._to(send[: sum(counts)])
        recv = torch.empty(sum(rcl), dtype=payload.dtype, device=payload.device)
        self.dist.all_to_all_single(recv, payload, rcl, list(counts), group=self.group)
        return recv.to(send.device) if recv.device != send.device else recv

    def all_gather_var(self, t):
        """Every rank's 1-D tensor `t` (lengths may differ), concatenated in
        rank order, on t's device."""
        import torch

        dev = "cpu" if self.host else t.device
        n = torch.tensor([t.numel()], dtype=torch.int64, device=dev)
        ns = [torch.zeros_like(n) for _ in range(self.world)]
        self.dist.all_gather(ns, n, group=self.group)
        lens = [int(x.item()) for x in ns]
        width = max(max(lens), 1)
        pad = torch.zeros(width, dtype=t.dtype, device=dev)
        pad[: t.numel()] = self._to(t)
        got = [torch.zeros_like(pad) for _ in range(self.world)]
        self.dist.all_gather(got, pad, group=self.group)
        out = torch.cat([g[:k] for g, k in zip(got, lens)])
        return out.to(t.device) if out.device != t.device else out


class CudaShardOps:
    """One rank's device steps through libkspn (kspn_shard_* and, for the
    residual, kspn_build_csr + kspn_scc_device).  Buffers are torch CUDA
    tensors owned here."""

    def __init__(self, ctx, shard: Shard):
        import torch

        from . import lib

        self.L = lib()
        self.ctx = ctx
        self.S = shard
        n_loc, n = shard.n_loc, shard.n
        words, gwords = (n_loc + 31) // 32 + 1, (n + 31) // 32 + 1
        z = lambda k: torch.zeros(max(k, 1), dtype=torch.int32, device="cuda")  # noqa: E731
        self.und = z(words)
        self.ids = z(n_loc)
        self.cand = [z(words), z(words)]
        self.vis = [z(words), z(words)]
        self.sent = [z(gwords), z(gwords)]
        self.front = [z(n_loc), z(n_loc)]
        self.next = [z(n_loc), z(n_loc)]
        self.front_n = [0, 0]
        self.next_n = [0, 0]
        self.remote = z(n)
        self.send = z(n)
        self.counts = z(2 * shard.parts)
        self.bounds = torch.tensor(shard.bounds, dtype=torch.int64).to(torch.int32).cuda()
        self.rows = [(shard.fwh, shard.fwc), (shard.bwh, shard.bwc)]  # FW expands out-rows, BW in-rows

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr())

    @staticmethod
    def _torch_done():
        """Inputs made by torch (on its current stream) are complete before a
        library step reads them on the context's stream."""
        import torch

        torch.cuda.current_stream().synchronize()

    def _ok(self, rc):
        from . import KspnError

        if rc != 0:
            raise KspnError(rc, (self.L.kspn_last_error(self.ctx.h) or b"").decode())

    def trim_first(self):
        S = self.S
        prod, vid, dec = C.c_uint64(), C.c_uint32(), C.c_uint32()
        self._ok(self.L.kspn_shard_trim_first(self.ctx.h, S.n_loc, S.lo, self._p(S.fwh), self._p(S.bwh), self._p(self.und), self._p(self.ids),
                                              C.byref(prod), C.byref(vid), C.byref(dec)))
        return dec.value, prod.value, vid.value

    def pivot(self):
        S = self.S
        prod, vid = C.c_uint64(), C.c_uint32()
        self._ok(self.L.kspn_shard_pivot(self.ctx.h, S.n_loc, S.lo, self._p(S.fwh), self._p(S.bwh), self._p(self.und), C.byref(prod), C.byref(vid)))
        return prod.value, vid.value

    def search_begin(self):
        S = self.S
        self._ok(self.L.kspn_shard_search_begin(self.ctx.h, S.n_loc, S.n, self._p(self.und), self._p(self.cand[0]), self._p(self.cand[1]),
                                                self._p(self.vis[0]), self._p(self.vis[1]), self._p(self.sent[0]), self._p(self.sent[1])))
        self.front_n = [0, 0]
        self.next_n = [0, 0]

    def receive(self, d: int, ids):
        """Global ids (this shard's) taken as finds of search d."""
        import torch

        S = self.S
        ids = ids.to(device="cuda", dtype=torch.int32).contiguous()
        self._torch_done()
        nn = C.c_uint32(self.next_n[d])
        self._ok(self.L.kspn_shard_receive(self.ctx.h, S.n_loc, S.lo, self._p(ids), ids.numel(), self._p(self.cand[d]), self._p(self.vis[d]),
                                           self._p(self.next[d]), S.n_loc, C.byref(nn)))
        self.next_n[d] = nn.value

    def expand(self, d: int):
        """Expands search d's frontier: local finds to its next list; returns
        (ids for the other ranks grouped by owner, counts per rank)."""
        S = self.S
        head, adj = self.rows[d]
        nn = C.c_uint32(self.next_n[d])
        counts = (C.c_uint32 * S.parts)()
        self._ok(self.L.kspn_shard_expand(self.ctx.h, S.n_loc, S.lo, self._p(head), self._p(adj), self._p(self.front[d]), self.front_n[d],
                                          self._p(self.cand[d]), self._p(self.vis[d]), self._p(self.sent[d]), self._p(self.next[d]), S.n_loc, C.byref(nn),
                                          self._p(self.remote), S.n, S.parts, self._p(self.bounds), self._p(self.send), self._p(self.counts), counts))
        self.next_n[d] = nn.value
        return self.send, list(counts)

    def advance(self, d: int) -> int:
        self.front[d], self.next[d] = self.next[d], self.front[d]
        self.front_n[d], self.next_n[d] = self.next_n[d], 0
        return self.front_n[d]

    def scc_min(self) -> int:
        S = self.S
        m = C.c_uint32()
        self._ok(self.L.kspn_shard_scc_min(self.ctx.h, S.n_loc, S.lo, self._p(self.vis[0]), self._p(self.vis[1]), C.byref(m)))
        return m.value

    def finalize(self, scc: int) -> int:
        S = self.S
        dec = C.c_uint32()
        self._ok(self.L.kspn_shard_finalize(self.ctx.h, S.n_loc, self._p(self.vis[0]), self._p(self.vis[1]), self._p(self.und), self._p(self.ids),
                                            scc, C.byref(dec)))
        return dec.value

    def und_words(self):
        return self.und[: (self.S.n_loc + 31) // 32]

    def residual_edges(self, gund):
        import torch

        S = self.S
        gund = gund.to(device="cuda", dtype=torch.int32).contiguous()
        self._torch_done()
        cnt = C.c_uint64()
        self._ok(self.L.kspn_shard_residual(self.ctx.h, S.n_loc, S.lo, self._p(S.fwh), self._p(S.fwc), self._p(self.und), self._p(gund),
                                            None, None, 0, C.byref(cnt)))
        k = cnt.value
        src = torch.empty(max(k, 1), dtype=torch.int32, device="cuda")
        dst = torch.empty(max(k, 1), dtype=torch.int32, device="cuda")
        if k:
            self._ok(self.L.kspn_shard_residual(self.ctx.h, S.n_loc, S.lo, self._p(S.fwh), self._p(S.fwc), self._p(self.und), self._p(gund),
                                                self._p(src), self._p(dst), k, C.byref(cnt)))
        return src[:k], dst[:k]

    def solve_residual(self, k: int, src, dst):
        """SCCs of the k-vertex residual graph (compact ids, edges src ->
        dst): the smallest member per vertex, by the single-GPU pipeline."""
        import torch

        from . import default_options
        from .graphs import from_edges

        src, dst = src.to(torch.int32).contiguous().clone(), dst.to(torch.int32).contiguous().clone()
        self._torch_done()
        G = from_edges(self.ctx, k, src, dst)
        out = torch.empty(max(k, 1), dtype=torch.int32, device="cuda")
        self.ctx.scc_device(k, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, default_options(validate=0))
        return out[:k]

    def set_ids(self, local_pos, values):
        import torch

        self.ids[local_pos.to(device="cuda", dtype=torch.int64)] = values.to(device="cuda", dtype=torch.int32)

    def local_ids(self):
        return self.ids[: self.S.n_loc]


def _bits_to_ids(words, n: int, xp):
    """Vertex ids < n whose bit is set in u32 bitmap words."""
    w = words.to(xp.int64) & 0xFFFFFFFF if hasattr(words, "to") else words.astype(np.int64) & 0xFFFFFFFF
    if hasattr(w, "device"):
        import torch

        bits = (w.unsqueeze(1) >> torch.arange(32, device=w.device)) & 1
        return torch.nonzero(bits.reshape(-1)[:n]).reshape(-1)
    bits = (w[:, None] >> np.arange(32)) & 1
    return np.nonzero(bits.reshape(-1)[:n])[0]


@dataclass
class ShardStats:
    decided_trim: int = 0
    decided_fwbw: int = 0
    decided_residual: int = 0
    rounds: int = 0
    levels: int = 0
    exchanged: int = 0  # ids sent between ranks, all levels, this rank


def scc_sharded(ops, ex: Exchange, S: Shard, max_rounds: int = 8, stats: ShardStats | None = None):
    """The sharded decomposition; returns this rank's ids (smallest member
    of each vertex's SCC, global ids) as the ops' array type."""
    import torch

    st = stats if stats is not None else ShardStats()
    dec, prod, vid = ops.trim_first()
    decided = ex.sum([dec])[0]
    st.decided_trim = decided
    pivot = ex.pivot(prod, vid)
    while decided < S.n and pivot != UNDECIDED and st.rounds < max_rounds:
        # ---- FW-BW from the pivot, both searches a level at a time
        ops.search_begin()
        seed = torch.tensor([pivot], dtype=torch.int64) if S.lo <= pivot < S.hi else torch.zeros(0, dtype=torch.int64)
        for d in (0, 1):
            ops.receive(d, seed)
        live = ex.sum([ops.advance(0), ops.advance(1)])
        while live[0] or live[1]:
            for d in (0, 1):
                if live[d]:
                    send, counts = ops.expand(d)
                    st.exchanged += sum(counts)
                    ops.receive(d, ex.all_to_all(send, counts))
            live = ex.sum([ops.advance(0) if live[0] else 0, ops.advance(1) if live[1] else 0])
            st.levels += 1
        scc = ex.min(ops.scc_min())
        got = ex.sum([ops.finalize(scc)])[0] if scc != UNDECIDED else 0
        st.decided_fwbw += got
        st.rounds += 1
        left = S.n - decided
        decided += got
        if got * 64 < left:
            break
        prod, vid = ops.pivot()
        pivot = ex.pivot(prod, vid)
    if decided < S.n:
        # ---- the residual, decomposed whole on every rank
        gund = ex.all_gather_var(ops.und_words())
        verts = _bits_to_ids(gund, S.n, torch)
        k = int(verts.numel())
        src, dst = ops.residual_edges(gund)
        src, dst = ex.all_gather_var(src), ex.all_gather_var(dst)
        verts = verts.to(src.device)
        cs = torch.searchsorted(verts, src.to(torch.int64))
        cd = torch.searchsorted(verts, dst.to(torch.int64))
        low = ops.solve_residual(k, cs, cd)  # compact ids; order-preserving, so the smallest member maps to the smallest global id
        mine = (verts >= S.lo) & (verts < S.hi)
        ops.set_ids(verts[mine] - S.lo, verts[low.to(torch.int64)][mine])
        st.decided_residual = k
    return ops.local_ids()
