"""The batched path (kspn_scc_batched; no reference counterpart): many
independent G(n, m) graphs of uneven size in one call, each checked against
the oracle's Tarjan of that graph (bit-exact, smallest-member ids), through
every route a large graph can take (trim + FW-BW rounds, the shared-memory
Tarjan of the remainder, one thread's Tarjan after the round cap)."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import kaspan_b200.graphs as KG
import oracle as O

pytestmark = pytest.mark.gpu


def _oracle_ids(B) -> np.ndarray:
    """Tarjan of the batch as one graph with global ids, back to local ids."""
    fwh = B.fwh.cpu().numpy().view(np.uint64)
    fwc = B.fwc.cpu().numpy().view(np.uint32)[: B.m].astype(np.uint64)
    vo = np.concatenate([[0], np.cumsum(B.sizes, dtype=np.uint64)]).astype(np.uint64)
    row_graph = np.repeat(np.arange(B.count), B.sizes)
    row_of_edge = np.repeat(np.arange(B.n), np.diff(fwh).astype(np.int64))
    glob = (fwc + vo[row_graph[row_of_edge]]).astype(np.uint32)
    ids = O.tarjan(O.from_csr(B.n, fwh, glob))
    return (ids.astype(np.uint64) - vo[row_graph]).astype(np.uint32)


def _run(ctx, B, **opt):
    import torch

    o = K.BatchOptions()
    lib = K.lib()
    lib.kspn_batch_options_default(__import__("ctypes").byref(o))
    for k, v in opt.items():
        setattr(o, k, v)
    out = torch.empty(B.n, dtype=torch.int32, device="cuda")
    st = ctx.scc_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out, o)
    return out.cpu().numpy().view(np.uint32).copy(), st


@pytest.fixture(scope="module")
def mix(ctx):
    # 300 graphs, 2^4 .. 2^13 vertices, mean out-degree 0.8 .. 6 (both sides
    # of the giant-component threshold): small graphs for the warp path and
    # larger ones for the block path
    B = KG.batch(ctx, 300, 11, 4, 13, 0.8, 6.0)
    return B, _oracle_ids(B)


def test_batch_shape_is_deterministic():
    n1, d1 = K.batch_shape(64, 5)
    n2, d2 = K.batch_shape(64, 5)
    assert np.array_equal(n1, n2) and np.array_equal(d1, d2)
    assert n1.min() >= 2**8 and n1.max() <= 2**18
    ratio = d1 / n1
    assert ratio.min() >= 0.8 - 1e-3 and ratio.max() <= 6.0 + 1e-2


def test_batched_matches_tarjan(ctx, mix):
    B, want = mix
    got, st = _run(ctx, B)
    assert np.array_equal(got, want)
    assert st.graphs_small > 0 and st.graphs_large > 0 and st.graphs_small + st.graphs_large == B.count
    # the replayed CUDA graph gives the same output
    got2, st2 = _run(ctx, B)
    assert np.array_equal(got2, want)
    assert st2.fwbw_rounds == st.fwbw_rounds


@pytest.mark.parametrize("search", [1, 2])
@pytest.mark.parametrize("cluster_size", [1, 2, 8])
@pytest.mark.parametrize("max_rounds,rem_tarjan", [(1, 1), (1000, 1), (2, 512), (64, 64)])
def test_batched_routes(ctx, mix, max_rounds, rem_tarjan, cluster_size, search):
    """(1, 1): one FW-BW round, then one thread's Tarjan; (1000, 1): FW-BW
    rounds until nothing is left; the others mix in the shared-memory
    Tarjan of the remainder.  With cluster_size > 1, graphs of n + m >=
    2000 go to thread-block clusters of that many blocks; search 1 runs FW
    and BW at the same time, 2 one after the other."""
    B, want = mix
    got, st = _run(ctx, B, max_rounds=max_rounds, rem_tarjan=rem_tarjan, cluster_size=cluster_size, cluster_min=2000, search=search)
    assert np.array_equal(got, want)
    assert st.cluster_size == cluster_size
    assert (st.graphs_cluster > 0) == (cluster_size > 1)  # size 1: every larger graph gets a block
    if (max_rounds, rem_tarjan) == (1, 1):
        assert st.tarjan_serial > 0
    if (max_rounds, rem_tarjan) == (1000, 1):
        assert st.tarjan_serial == 0


def test_batched_edge_cases(ctx):
    """Graphs of one vertex, self-loops only, a long cycle, a long path and
    two cycles joined by a path, concatenated with local ids."""
    import torch

    graphs = []
    graphs.append((1, []))
    graphs.append((3, [(0, 0), (1, 1), (2, 2)]))
    k = 3000
    graphs.append((k, [(i, (i + 1) % k) for i in range(k)]))
    graphs.append((k, [(i, i + 1) for i in range(k - 1)]))
    graphs.append((700, [(i, (i + 1) % 300) for i in range(300)] + [(299, 300)] + [(300 + i, 300 + (i + 1) % 400) for i in range(400)]))
    sizes = np.array([g[0] for g in graphs], np.uint32)
    vo = np.concatenate([[0], np.cumsum(sizes, dtype=np.uint64)])
    N = int(vo[-1])
    src = np.concatenate([np.array([e[0] for e in es], np.uint64) + vo[i] for i, (n, es) in enumerate(graphs)]).astype(np.uint32)
    dst = np.concatenate([np.array([e[1] for e in es], np.uint64) + vo[i] for i, (n, es) in enumerate(graphs)]).astype(np.uint32)
    G = KG.from_edges(ctx, N, torch.from_numpy(src.view(np.int32)).cuda(), torch.from_numpy(dst.view(np.int32)).cuda())
    d_vo = torch.from_numpy(vo.astype(np.int64)).cuda()
    ctx.batch_localize(len(graphs), N, d_vo, G.fwh, G.fwc)
    ctx.batch_localize(len(graphs), N, d_vo, G.bwh, G.bwc)
    B = KG.DeviceBatch(len(graphs), N, G.m, d_vo, G.fwh, G.fwc, G.bwh, G.bwc, sizes)
    want = _oracle_ids(B)
    for opt in ({}, {"max_rounds": 1, "rem_tarjan": 1}, {"cluster_min": 100}, {"cluster_min": 100, "cluster_size": 4, "rem_tarjan": 1},
                {"search": 2}, {"search": 2, "rem_tarjan": 1}):
        got, _ = _run(ctx, B, **opt)
        assert np.array_equal(got, want)
    # spot checks: the cycle is one SCC named 0, the path all singletons
    assert np.all(want[int(vo[2]): int(vo[3])] == 0)
    assert np.array_equal(want[int(vo[3]): int(vo[4])], np.arange(k, dtype=np.uint32))


def test_batched_union_route(ctx, mix):
    """route 1: the mix as one graph with a super-source linked to every
    graph's pivot, through the single-graph pipeline; the same ids as the
    per-graph route and as Tarjan, on a repeated call too."""
    B, want = mix
    for _ in range(2):
        got, st = _run(ctx, B, route=1)
        assert np.array_equal(got, want)
        assert st.graphs_large == B.count and st.graphs_small == 0  # the union route ran


def test_batched_union_route_edge_cases(ctx):
    """The union route on a graph of one vertex (no pivot), self-loops only,
    a long cycle, a long path and two cycles joined by a path."""
    import torch

    graphs = [(1, []), (3, [(0, 0), (1, 1), (2, 2)])]
    k = 3000
    graphs.append((k, [(i, (i + 1) % k) for i in range(k)]))
    graphs.append((k, [(i, i + 1) for i in range(k - 1)]))
    graphs.append((700, [(i, (i + 1) % 300) for i in range(300)] + [(299, 300)] + [(300 + i, 300 + (i + 1) % 400) for i in range(400)]))
    sizes = np.array([g[0] for g in graphs], np.uint32)
    vo = np.concatenate([[0], np.cumsum(sizes, dtype=np.uint64)])
    N = int(vo[-1])
    src = np.concatenate([np.array([e[0] for e in es], np.uint64) + vo[i] for i, (n, es) in enumerate(graphs)]).astype(np.uint32)
    dst = np.concatenate([np.array([e[1] for e in es], np.uint64) + vo[i] for i, (n, es) in enumerate(graphs)]).astype(np.uint32)
    G = KG.from_edges(ctx, N, torch.from_numpy(src.view(np.int32)).cuda(), torch.from_numpy(dst.view(np.int32)).cuda())
    d_vo = torch.from_numpy(vo.astype(np.int64)).cuda()
    ctx.batch_localize(len(graphs), N, d_vo, G.fwh, G.fwc)
    ctx.batch_localize(len(graphs), N, d_vo, G.bwh, G.bwc)
    B = KG.DeviceBatch(len(graphs), N, G.m, d_vo, G.fwh, G.fwc, G.bwh, G.bwc, sizes)
    want = _oracle_ids(B)
    got, st = _run(ctx, B, route=1)
    assert np.array_equal(got, want)
    assert st.graphs_large == len(graphs)
