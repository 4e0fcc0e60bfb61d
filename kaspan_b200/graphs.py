"""Device-resident graphs and the seeded synthetic inputs, built with libkspn.

The generators stand in for the KaGen inputs the reference benchmarks with
(experiment/horeka/bootstrap.py:35-39): directed G(n, m), R-MAT with a
seeded id permutation, and a 2D random geometric graph (each pair within
the radius becomes u->v, v->u, both or neither).  Every step runs on the GPU through the C ABI:
draw the edge list (kspn_gen_*), sort + dedupe into a CSR (kspn_build_csr),
build the transpose (kspn_transpose).  torch provides the device buffers.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import Context


@dataclass
class DeviceGraph:
    n: int
    m: int
    fwh: "torch.Tensor"  # int64[n+1] holding u64 offsets
    fwc: "torch.Tensor"  # int32[m]   holding u32 ids
    bwh: "torch.Tensor"
    bwc: "torch.Tensor"

    def nbytes(self) -> int:
        return 2 * 8 * (self.n + 1) + 2 * 4 * self.m

    def to_host(self):
        """(fwh, fwc, bwh, bwc) as numpy u64/u32 arrays."""
        return (self.fwh.cpu().numpy().view(np.uint64), self.fwc.cpu().numpy().view(np.uint32),
                self.bwh.cpu().numpy().view(np.uint64), self.bwc.cpu().numpy().view(np.uint32))


def rmat_thresholds(a: float, b: float, c: float):
    s = float(1 << 32)
    return int(math.floor(a * s)), int(math.floor((a + b) * s)), int(math.floor((a + b + c) * s))


def from_edges(ctx: Context, n: int, src, dst, device="cuda") -> DeviceGraph:
    """Edge list (device int32 tensors, consumed) -> DeviceGraph."""
    import torch

    m_raw = src.numel()
    head = torch.empty(n + 1, dtype=torch.int64, device=device)
    csr = torch.empty(max(m_raw, 1), dtype=torch.int32, device=device)
    m = ctx.build_csr(n, m_raw, src, dst, head, csr)
    del src, dst
    csr = csr[:m].clone() if m < csr.numel() else csr
    bwh = torch.empty(n + 1, dtype=torch.int64, device=device)
    bwc = torch.empty(max(m, 1), dtype=torch.int32, device=device)
    ctx.transpose(n, m, head, csr, bwh, bwc)
    return DeviceGraph(n, m, head, csr, bwh, bwc)


def from_host_csr(n: int, fwh, fwc, bwh, bwc, device="cuda") -> DeviceGraph:
    import torch

    def t(a, dt):
        a = np.ascontiguousarray(a)
        return torch.from_numpy(a.view(dt).copy()).to(device)

    m = int(fwh[n]) if n else 0
    return DeviceGraph(n, m, t(fwh, np.int64), t(fwc[: max(m, 1)], np.int32), t(bwh, np.int64), t(bwc[: max(m, 1)], np.int32))


def gnm(ctx: Context, n: int, draws: int, seed: int, device="cuda") -> DeviceGraph:
    import torch

    src = torch.empty(max(draws, 1), dtype=torch.int32, device=device)
    dst = torch.empty(max(draws, 1), dtype=torch.int32, device=device)
    ctx.gen_gnm(n, draws, seed, src, dst)
    return from_edges(ctx, n, src[:draws], dst[:draws], device)


def rmat(ctx: Context, scale: int, edge_factor: int, seed: int, a=0.57, b=0.19, c=0.19, permute=True, device="cuda") -> DeviceGraph:
    import torch

    draws = edge_factor << scale
    ta, tab, tabc = rmat_thresholds(a, b, c)
    src = torch.empty(max(draws, 1), dtype=torch.int32, device=device)
    dst = torch.empty(max(draws, 1), dtype=torch.int32, device=device)
    ctx.gen_rmat(scale, draws, seed, ta, tab, tabc, permute, src, dst)
    return from_edges(ctx, 1 << scale, src[:draws], dst[:draws], device)


def rgg_params(n: int, mean_undirected_degree: float = 8.0):
    """Cells per side g = floor(1/r) and r^2 in units of 2^-60 for radius
    r = sqrt(deg / (pi n)) (mean undirected degree deg, boundary effects
    ignored)."""
    r2 = mean_undirected_degree / (math.pi * n)
    g = max(1, int(math.floor(1.0 / math.sqrt(r2))))
    return g, int(math.floor(r2 * float(1 << 60)))


def rgg(ctx: Context, n: int, seed: int, mean_undirected_degree: float = 8.0, device="cuda") -> DeviceGraph:
    import torch

    g, r2 = rgg_params(n, mean_undirected_degree)
    m_raw = ctx.gen_rgg(n, seed, g, r2)
    src = torch.empty(max(m_raw, 1), dtype=torch.int32, device=device)
    dst = torch.empty(max(m_raw, 1), dtype=torch.int32, device=device)
    ctx.gen_rgg(n, seed, g, r2, src, dst, m_raw)
    return from_edges(ctx, n, src[:m_raw], dst[:m_raw], device)


@dataclass
class DeviceBatch:
    """Many graphs in one concatenated CSR/CSC (heads: global edge
    positions, rows: local ids), as kspn_scc_batched takes them."""
    count: int
    n: int  # total vertices
    m: int  # total edges
    vtx_off: "torch.Tensor"  # int64[count+1]
    fwh: "torch.Tensor"
    fwc: "torch.Tensor"
    bwh: "torch.Tensor"
    bwc: "torch.Tensor"
    sizes: np.ndarray  # vertices per graph

    def graph(self, g: int):
        """Graph g as host CSR/CSC with local offsets (for checking)."""
        vo = np.concatenate([[0], np.cumsum(self.sizes, dtype=np.uint64)])
        a, b = int(vo[g]), int(vo[g + 1])
        fwh = self.fwh[a: b + 1].cpu().numpy().view(np.uint64)
        bwh = self.bwh[a: b + 1].cpu().numpy().view(np.uint64)
        fwc = self.fwc[int(fwh[0]): int(fwh[-1])].cpu().numpy().view(np.uint32)
        bwc = self.bwc[int(bwh[0]): int(bwh[-1])].cpu().numpy().view(np.uint32)
        return b - a, fwh - fwh[0], fwc, bwh - bwh[0], bwc


def batch_partition(work: np.ndarray, parts: int) -> list[np.ndarray]:
    """Greedy longest-processing-time bin packing of graphs (by `work`, e.g.
    n + edge draws) onto `parts` GPUs: largest first, each to the least
    loaded part (ties: lowest part).  Deterministic; every rank computes the
    same assignment.  Returns each part's graph indices, ascending."""
    order = np.argsort(-np.asarray(work, np.float64), kind="stable")
    load = np.zeros(parts, np.float64)
    owner = np.empty(len(order), np.int64)
    for g in order:
        p = int(np.argmin(load))
        owner[g] = p
        load[p] += float(work[g])
    return [np.nonzero(owner == p)[0] for p in range(parts)]


def batch(ctx: Context, count: int = 4096, seed: int = 5, log2_min: int = 8, log2_max: int = 18, deg_min: float = 0.8, deg_max: float = 6.0,
          device="cuda", graphs: "np.ndarray | None" = None) -> DeviceBatch:
    """The uneven G(n, m) mix: graph i has round(2^U[log2_min, log2_max])
    vertices and round(n * U[deg_min, deg_max]) edge draws (self-loops and
    duplicates removed); all on the device.  `graphs`: only these graphs of
    the mix (a shard; each is the same graph the whole mix holds)."""
    import torch

    from . import batch_shape

    sizes, draws = batch_shape(count, seed, log2_min, log2_max, deg_min, deg_max)
    ids = None
    if graphs is not None:
        graphs = np.asarray(graphs, np.int64)
        sizes, draws = sizes[graphs], draws[graphs]
        ids = torch.from_numpy(graphs.astype(np.int32)).to(device)
        count = len(graphs)
    vtx_off = np.concatenate([[0], np.cumsum(sizes, dtype=np.uint64)]).astype(np.uint64)
    draw_off = np.concatenate([[0], np.cumsum(draws, dtype=np.uint64)]).astype(np.uint64)
    N, D = int(vtx_off[-1]), int(draw_off[-1])
    d_vo = torch.from_numpy(vtx_off.view(np.int64).copy()).to(device)
    d_do = torch.from_numpy(draw_off.view(np.int64).copy()).to(device)
    src = torch.empty(max(D, 1), dtype=torch.int32, device=device)
    dst = torch.empty(max(D, 1), dtype=torch.int32, device=device)
    torch.cuda.synchronize()
    ctx.gen_batch(count, seed, d_vo, d_do, src, dst, ids)
    G = from_edges(ctx, N, src[:D], dst[:D], device)
    del src, dst
    ctx.batch_localize(count, N, d_vo, G.fwh, G.fwc)
    ctx.batch_localize(count, N, d_vo, G.bwh, G.bwc)
    return DeviceBatch(count, N, G.m, d_vo, G.fwh, G.fwc, G.bwh, G.bwc, sizes)


def from_manifest(ctx: Context, path: str, device="cuda") -> DeviceGraph:
    """A graph in the reference's manifest format, loaded onto the device
    (kspn_manifest_read + kspn_manifest_load)."""
    import torch

    from . import manifest_read

    mf = manifest_read(path)
    n, m = int(mf.node_count), int(mf.edge_count)
    fwh = torch.empty(n + 1, dtype=torch.int64, device=device)
    bwh = torch.empty(n + 1, dtype=torch.int64, device=device)
    fwc = torch.empty(max(m, 1), dtype=torch.int32, device=device)
    bwc = torch.empty(max(m, 1), dtype=torch.int32, device=device)
    torch.cuda.synchronize()
    ctx.manifest_load(mf, fwh, fwc, bwh, bwc)
    return DeviceGraph(n, m, fwh, fwc, bwh, bwc)
