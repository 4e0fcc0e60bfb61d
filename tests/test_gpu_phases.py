"""GPU parity of every phase on the path against the reference's own code
(oracle/_ref, compiled from its sources) or, where the reference has no
one-call counterpart, the C restatement (oracle/kspn_oracle.c).

Each phase starts from the same vertex state on both sides and must leave
the same undecided bitset and the same member ids -- bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O
from kspn_testlib import (bits_equal, bits_to_dev, dev_to_bits, dev_to_u32, device, edge_case_graphs, full_bits,
                          fuzzy_cases, kat_graph, u32_to_dev)

pytestmark = pytest.mark.gpu


def graphs():
    out = [("kat", kat_graph())]
    out += [(f"edge_{n}", G) for n, G in edge_case_graphs()]
    for key, G, _ in fuzzy_cases((6, 33, 64, 150, 299), seeds=(0, 1), degrees=(0.5, 1.0, 4.0)):
        out.append((f"fuzzy{key}", G))
    out.append(("gnm12", O.gnm(1 << 12, 1 << 15, 1)))
    out.append(("rmat12", O.rmat(12, 16, 2)))
    out.append(("rmat14", O.rmat(14, 8, 7)))
    out.append(("rgg12", O.rgg(1 << 12, 3)))
    out.append(("rgg14", O.rgg(1 << 14, 5)))
    return out


GRAPHS = graphs()


def ref():
    R = O.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref not built")
    return R


def state_after(G, steps):
    """Reference state (bits, scc_id, pivot) after the listed reference phases."""
    R = ref()
    bits = full_bits(G.n)
    sid = np.full(max(G.n, 1), O.UNDECIDED, np.uint32)
    pivot = R.kref_trim_1_first(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid)
    if "fwbw" in steps and pivot < G.n:
        R.kref_fw_bw(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid, pivot)
    if "normal" in steps:
        R.kref_trim_1_normal(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid)
    return bits, sid, pivot


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_trim_1_first(ctx, name, G):
    R = ref()
    bits = full_bits(G.n)
    sid = np.full(max(G.n, 1), O.UNDECIDED, np.uint32)
    pivot = R.kref_trim_1_first(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid)
    fwh, fwc, bwh, bwc = device(G)
    d_bits = bits_to_dev(full_bits(G.n))
    d_sid = u32_to_dev(np.full(max(G.n, 1), O.UNDECIDED, np.uint32))
    gp = ctx.trim_1_first(G.n, G.m, fwh, bwh, d_bits, d_sid)
    assert gp == pivot
    assert bits_equal(dev_to_bits(d_bits), bits, G.n)
    und = O.bytes_from_bits(bits, G.n)
    assert np.array_equal(dev_to_u32(d_sid)[: G.n][und == 0], sid[: G.n][und == 0])


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_forward_backward_search(ctx, name, G):
    R = ref()
    bits, sid, pivot = state_after(G, ())
    fwh, fwc, bwh, bwc = device(G)
    if pivot >= G.n:
        # trim_1_first decided every vertex: no pivot; the phase call rejects
        # a pivot >= n with KSPN_ERR_INVALID_ARGUMENT and changes nothing
        d_bits, d_sid = bits_to_dev(bits), u32_to_dev(sid)
        with pytest.raises(K.KspnError) as e:
            ctx.forward_backward_search(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid, G.n)
        assert e.value.status == 1
        assert bits_equal(dev_to_bits(d_bits), bits, G.n)
        return
    d_bits, d_sid = bits_to_dev(bits), u32_to_dev(sid)
    before = O.bytes_from_bits(bits, G.n).sum()
    R.kref_fw_bw(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid, pivot)
    dec = ctx.forward_backward_search(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid, pivot)
    assert dec == before - O.bytes_from_bits(bits, G.n).sum()
    assert bits_equal(dev_to_bits(d_bits), bits, G.n)
    assert np.array_equal(dev_to_u32(d_sid)[: G.n], sid[: G.n])


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_trim_1_normal(ctx, name, G):
    R = ref()
    bits, sid, _ = state_after(G, ("fwbw",))
    fwh, fwc, bwh, bwc = device(G)
    d_bits, d_sid = bits_to_dev(bits), u32_to_dev(sid)
    R.kref_trim_1_normal(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid)
    ctx.trim_1_normal(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid)
    assert bits_equal(dev_to_bits(d_bits), bits, G.n)
    assert np.array_equal(dev_to_u32(d_sid)[: G.n], sid[: G.n])


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_label_search_chain(ctx, name, G):
    """Rotations 1, 2, 3, ... as kaspan::scc issues them, call by call,
    until every vertex is decided (at most 12 calls checked)."""
    R = ref()
    bits, sid, _ = state_after(G, ("fwbw", "normal"))
    fwh, fwc, bwh, bwc = device(G)
    d_bits, d_sid = bits_to_dev(bits), u32_to_dev(sid)
    import torch

    d_label = torch.empty(max(G.n, 1), dtype=torch.int32, device="cuda")
    for rot in range(1, 13):
        if not O.bytes_from_bits(bits, G.n).any():
            break
        R.kref_label_search_pull(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid, rot)
        ctx.label_search(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid, rot, d_label)
        assert bits_equal(dev_to_bits(d_bits), bits, G.n), rot
        assert np.array_equal(dev_to_u32(d_sid)[: G.n], sid[: G.n]), rot


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_trim_1_exhaustive_first(ctx, name, G):
    R = ref()
    bits = full_bits(G.n)
    sid = np.full(max(G.n, 1), O.UNDECIDED, np.uint32)
    outd = np.zeros(max(G.n, 1), np.uint32)
    ind = np.zeros(max(G.n, 1), np.uint32)
    R.kref_trim_1_exhaustive_first(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid, outd, ind)
    fwh, fwc, bwh, bwc = device(G)
    d_bits = bits_to_dev(full_bits(G.n))
    d_sid = u32_to_dev(np.full(max(G.n, 1), O.UNDECIDED, np.uint32))
    d_out = u32_to_dev(np.zeros(max(G.n, 1), np.uint32))
    d_in = u32_to_dev(np.zeros(max(G.n, 1), np.uint32))
    ctx.trim_1_exhaustive_first(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid, d_out, d_in)
    assert bits_equal(dev_to_bits(d_bits), bits, G.n)
    und = O.bytes_from_bits(bits, G.n).astype(bool)
    assert np.array_equal(dev_to_u32(d_sid)[: G.n][~und], sid[: G.n][~und])
    # live degrees of the survivors are the reference's
    assert np.array_equal(dev_to_u32(d_out)[: G.n][und], outd[: G.n][und])
    assert np.array_equal(dev_to_u32(d_in)[: G.n][und], ind[: G.n][und])


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_trim_1_fixpoint(ctx, name, G):
    bits, sid, _ = state_after(G, ())
    und = O.bytes_from_bits(bits, G.n).copy()
    osid = sid.copy()
    if G.n:
        O.lib().orc_trim_1_fixpoint(G.n, G.fwh, G.fwc, G.bwh, G.bwc, und, osid)
    fwh, fwc, bwh, bwc = device(G)
    d_bits, d_sid = bits_to_dev(bits), u32_to_dev(sid)
    ctx.trim_1_fixpoint(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid)
    assert np.array_equal(O.bytes_from_bits(dev_to_bits(d_bits), G.n), und[: G.n])
    assert np.array_equal(dev_to_u32(d_sid)[: G.n], osid[: G.n])


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_trim_2_exact(ctx, name, G):
    """Every pair trim-2 decides is a size-2 SCC (per Tarjan), and every
    pair matching the rule on the CPU is decided."""
    bits, sid, _ = state_after(G, ())
    fwh, fwc, bwh, bwc = device(G)
    d_bits, d_sid = bits_to_dev(bits), u32_to_dev(sid)
    ctx.trim_1_fixpoint(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid)
    before = O.bytes_from_bits(dev_to_bits(d_bits), G.n)
    ctx.trim_2(G.n, G.m, fwh, fwc, bwh, bwc, d_bits, d_sid)
    after = O.bytes_from_bits(dev_to_bits(d_bits), G.n)
    ids = dev_to_u32(d_sid)[: G.n]
    truth = O.tarjan(G)
    newly = np.nonzero((before == 1) & (after == 0))[0]
    for v in newly:
        comp = np.nonzero(truth == truth[v])[0]
        assert len(comp) == 2 and ids[v] == comp.min(), (v, comp)

    # CPU restatement of the rule on the pre-trim-2 state
    def one(head, adj, v):
        s = {int(w) for w in adj[head[v]:head[v + 1]] if before[w]}
        return s.pop() if len(s) == 1 else None

    expect = set()
    for u in np.nonzero(before)[0]:
        for head, adj in ((G.fwh, G.fwc), (G.bwh, G.bwc)):
            v = one(head, adj, u)
            if v is not None and v != u and one(head, adj, v) == u:
                expect |= {int(u), v}
    assert expect == set(int(x) for x in newly)


def test_normalise(ctx):
    rng = np.random.default_rng(5)
    for n in (1, 7, 1000, 100_000):
        ids = rng.integers(0, n, n).astype(np.uint32)
        d = u32_to_dev(ids)
        ctx.normalise(n, d)
        assert np.array_equal(dev_to_u32(d)[:n], O.normalise(ids))


@pytest.mark.parametrize("name,G", GRAPHS[:12] + GRAPHS[-5:], ids=[g[0] for g in GRAPHS[:12] + GRAPHS[-5:]])
def test_transpose(ctx, name, G):
    import torch

    fwh, fwc, _, _ = device(G)
    bwh = torch.empty(G.n + 1, dtype=torch.int64, device="cuda")
    bwc = torch.empty(max(G.m, 1), dtype=torch.int32, device="cuda")
    ctx.transpose(G.n, G.m, fwh, fwc, bwh, bwc)
    assert np.array_equal(bwh.cpu().numpy().view(np.uint64), G.bwh)
    assert np.array_equal(bwc.cpu().numpy().view(np.uint32)[: G.m], G.bwc[: G.m])


@pytest.mark.parametrize("kind", ["gnm", "rmat", "rmat_noperm", "rmat_odd"])
def test_generators_and_csr_build(ctx, kind):
    import torch

    import kaspan_b200.graphs as KG

    if kind == "gnm":
        n, draws = 1 << 13, 1 << 16
        es, ed = O.gnm_edges(n, draws, 21)
        src = torch.empty(draws, dtype=torch.int32, device="cuda")
        dst = torch.empty(draws, dtype=torch.int32, device="cuda")
        ctx.gen_gnm(n, draws, 21, src, dst)
    else:
        scale = 13 if kind != "rmat_odd" else 11
        perm = kind != "rmat_noperm"
        n, draws = 1 << scale, 8 << scale
        es, ed = O.rmat_edges(scale, 8, 22, permute=perm)
        ta, tab, tabc = KG.rmat_thresholds(0.57, 0.19, 0.19)
        src = torch.empty(draws, dtype=torch.int32, device="cuda")
        dst = torch.empty(draws, dtype=torch.int32, device="cuda")
        ctx.gen_rmat(scale, draws, 22, ta, tab, tabc, perm, src, dst)
    assert np.array_equal(src.cpu().numpy().view(np.uint32), es)
    assert np.array_equal(dst.cpu().numpy().view(np.uint32), ed)
    G = O.from_edges(n, es, ed)
    DG = KG.from_edges(ctx, n, src, dst)
    assert DG.m == G.m
    fwh, fwc, bwh, bwc = DG.to_host()
    assert np.array_equal(fwh, G.fwh) and np.array_equal(fwc[: G.m], G.fwc[: G.m])
    assert np.array_equal(bwh, G.bwh) and np.array_equal(bwc[: G.m], G.bwc[: G.m])


@pytest.mark.parametrize("n", [1, 2, 7, 1000, 1 << 14, 1 << 16])
def test_rgg_generator(ctx, n):
    """Device RGG (kspn_gen_rgg) = the oracle's orc_rgg_points/orc_rgg_edges
    restatement: same edge count, same CSR after dedupe, same transpose."""
    import kaspan_b200.graphs as KG

    g, r2 = KG.rgg_params(n)
    assert (g, r2) == O.rgg_params(n)
    G = O.rgg(n, 3)
    DG = KG.rgg(ctx, n, 3)
    assert DG.m == G.m
    fwh, fwc, bwh, bwc = DG.to_host()
    assert np.array_equal(fwh, G.fwh) and np.array_equal(fwc[: G.m], G.fwc[: G.m])
    assert np.array_equal(bwh, G.bwh) and np.array_equal(bwc[: G.m], G.bwc[: G.m])


def test_rgg_capacity_error(ctx):
    import torch

    import kaspan_b200.graphs as KG

    n = 1 << 12
    g, r2 = KG.rgg_params(n)
    m = ctx.gen_rgg(n, 3, g, r2)
    assert m > 0
    src = torch.empty(m - 1, dtype=torch.int32, device="cuda")
    dst = torch.empty(m - 1, dtype=torch.int32, device="cuda")
    with pytest.raises(K.KspnError):
        ctx.gen_rgg(n, 3, g, r2, src, dst, m - 1)


def _wcc(G, keep):
    """Weakly connected pieces of the sub-graph induced by `keep` (bool[n]):
    (piece label per vertex, internal edge count per piece)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    src = np.repeat(np.arange(G.n), np.diff(G.fwh.astype(np.int64)))
    dst = G.fwc[: G.m].astype(np.int64)
    ok = keep[src] & keep[dst] & (src != dst)
    A = csr_matrix((np.ones(int(ok.sum())), (src[ok], dst[ok])), shape=(G.n, G.n))
    _, lab = connected_components(A, directed=True, connection="weak")
    edges = np.bincount(lab[src[ok]], minlength=lab.max() + 1)
    return lab, edges


@pytest.mark.parametrize("name,G", GRAPHS, ids=[g[0] for g in GRAPHS])
def test_residual(ctx, name, G):
    """kspn_residual = Tarjan on the sub-graph induced by the undecided
    vertices (variant/scc_trim_ex_residual.hpp:110-127), each SCC named by
    its smallest member -- for every weakly connected piece of at most 512
    vertices and 2048 internal edges; larger pieces stay undecided."""
    rng = np.random.default_rng(len(name))
    for frac in (1.0, 0.6):
        keep = rng.random(G.n) < frac if frac < 1.0 else np.ones(G.n, bool)
        sid = np.where(keep, np.uint32(0xFFFFFFFF), np.arange(G.n, dtype=np.uint32)).astype(np.uint32)
        d_bits, d_sid = bits_to_dev(O.bits_from_bytes(keep.astype(np.uint8), G.n)), u32_to_dev(sid)
        fwh, fwc, _, _ = device(G)
        decided, left = ctx.residual(G.n, G.m, fwh, fwc, d_bits, d_sid)
        after = O.bytes_from_bits(dev_to_bits(d_bits), G.n).astype(bool)
        ids = dev_to_u32(d_sid)[: G.n]
        # expected: Tarjan of the induced sub-graph
        src = np.repeat(np.arange(G.n, dtype=np.uint32), np.diff(G.fwh.astype(np.int64)))
        dst = G.fwc[: G.m]
        ok = keep[src] & keep[dst]
        truth = O.tarjan(O.from_edges(G.n, src[ok], dst[ok]))
        lab, edges = _wcc(G, keep)
        size = np.bincount(lab, minlength=lab.max() + 1)
        small = (size <= 512) & (edges <= 2048)
        fits = keep & small[lab]
        assert left == len(np.unique(lab[keep & ~small[lab]]))
        assert decided == int(fits.sum())
        assert np.array_equal(after, keep & ~fits)
        assert np.array_equal(ids[fits], truth[fits])
        assert np.array_equal(ids[~keep], sid[~keep])
        assert np.all(ids[keep & ~fits] == 0xFFFFFFFF)
