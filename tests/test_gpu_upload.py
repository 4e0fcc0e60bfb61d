"""Host CSR upload with the CSC built while the upload runs
(kspn_upload_transpose, and kspn_scc with bw = NULL which uses it): the
device CSR must equal the host one and the device CSC the oracle's
transpose (the reference's backward_complement_graph,
kaspan/scc/backward_complement.hpp:22-68: rows ascending), bit for bit, for
chunk sizes that cut rows anywhere, including one hub row spread over many
chunks; invalid input is rejected without touching memory outside the
arrays."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O
from kspn_testlib import edge_case_graphs

pytestmark = pytest.mark.gpu


def upload(ctx, G, chunk, pinned):
    import torch

    n, m = G.n, G.m
    fwh_h = torch.from_numpy(G.fwh.view(np.int64).copy())
    fwc_h = torch.from_numpy(G.fwc[: max(m, 1)].view(np.int32).copy())
    if pinned:
        fwh_h, fwc_h = fwh_h.pin_memory(), fwc_h.pin_memory()
    fwh = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
    fwc = torch.full((max(m, 1),), -1, dtype=torch.int32, device="cuda")
    bwh = torch.full((n + 1,), -1, dtype=torch.int64, device="cuda")
    bwc = torch.full((max(m, 1),), -1, dtype=torch.int32, device="cuda")
    ctx.upload_transpose(n, m, fwh_h, fwc_h, fwh, fwc, bwh, bwc, chunk)
    return (fwh.cpu().numpy().view(np.uint64), fwc.cpu().numpy().view(np.uint32)[:m],
            bwh.cpu().numpy().view(np.uint64), bwc.cpu().numpy().view(np.uint32)[:m])


def check(ctx, G, chunk, pinned=True):
    fwh, fwc, bwh, bwc = upload(ctx, G, chunk, pinned)
    m = G.m
    assert np.array_equal(fwh, G.fwh) and np.array_equal(fwc, G.fwc[:m])
    assert np.array_equal(bwh, G.bwh), "CSC heads differ from the oracle's transpose"
    assert np.array_equal(bwc, G.bwc[:m]), "CSC rows differ from the oracle's transpose"


@pytest.mark.parametrize("name,G", edge_case_graphs(), ids=[g[0] for g in edge_case_graphs()])
def test_edge_cases(ctx, name, G):
    for chunk in (0, 1, 3, 64):
        check(ctx, G, chunk)


@pytest.mark.parametrize("chunk", [0, 7, 1000, 4096, 65536])
def test_rmat_chunks(ctx, chunk):
    G = O.rmat(12, 8, 21)
    check(ctx, G, chunk, pinned=chunk != 1000)  # one pageable-memory case


def test_hub_row_over_many_chunks(ctx):
    # vertex 0 points at every other vertex and every vertex points at 0,
    # plus a random sprinkle: one row of n-1 entries crosses ~40 chunks
    n = 50000
    rng = np.random.default_rng(4)
    others = np.arange(1, n, dtype=np.uint32)
    src = np.concatenate([np.zeros(n - 1, np.uint32), others, rng.integers(0, n, 20000, dtype=np.uint32)])
    dst = np.concatenate([others, np.zeros(n - 1, np.uint32), rng.integers(0, n, 20000, dtype=np.uint32)])
    G = O.from_edges(n, src, dst)
    check(ctx, G, 1237)
    check(ctx, G, 0)


def test_scc_host_path_chunked_matches_tarjan(ctx):
    # kspn_scc with bw = NULL goes through the chunked upload; a graph larger
    # than one default chunk (8 Mi edges) checks the multi-chunk route end to end
    G = O.rmat(19, 20, 8)
    assert G.m > (8 << 20)
    want = O.tarjan(G)
    got = ctx.scc(G.n, G.fwh, G.fwc)
    assert np.array_equal(got, want)
    fwh, fwc, bwh, bwc = upload(ctx, G, 0, True)
    assert np.array_equal(bwh, G.bwh) and np.array_equal(bwc, G.bwc[: G.m])


def test_invalid_input_rejected(ctx):
    G = O.gnm(4096, 30000, 3)
    bad = G.fwc.copy()
    bad[5] = 1 << 20  # id >= n: the upload stays in bounds, validation reports it
    with pytest.raises(K.KspnError) as e:
        ctx.scc(G.n, G.fwh, bad)
    assert e.value.status == 2
    heads = G.fwh.copy()
    heads[-1] += 1  # head[n] != m
    with pytest.raises(K.KspnError) as e:
        _upload_bad_heads(ctx, G, heads)
    assert e.value.status == 2
    # the context stays usable
    assert np.array_equal(ctx.scc(G.n, G.fwh, G.fwc), O.tarjan(G))


def _upload_bad_heads(ctx, G, heads):
    import torch

    fwh = torch.empty(G.n + 1, dtype=torch.int64, device="cuda")
    fwc = torch.empty(G.m, dtype=torch.int32, device="cuda")
    bwh = torch.empty(G.n + 1, dtype=torch.int64, device="cuda")
    bwc = torch.empty(G.m, dtype=torch.int32, device="cuda")
    ctx.upload_transpose(G.n, G.m, heads, G.fwc, fwh, fwc, bwh, bwc, 1000)
