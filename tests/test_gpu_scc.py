"""GPU parity of the whole path (kspn_scc / kspn_scc_device) against the CPU
oracle's Tarjan and the reference's own kaspan::scc, after canonical
relabelling.  Bit-exact: integer ids."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O
from kspn_testlib import KAT_IDS, device, edge_case_graphs, fuzzy_cases, kat_graph

pytestmark = pytest.mark.gpu

PIPELINES = [K.PIPELINE_FAST, K.PIPELINE_REFERENCE, K.PIPELINE_HPC_LIKE, K.PIPELINE_HPC_TRIM_EX, K.PIPELINE_ISPAN_LIKE,
             K.PIPELINE_TRIM_EX, K.PIPELINE_TRIM_EX_LIGHT_RESIDUAL, K.PIPELINE_TRIM_EX_RESIDUAL]


def run_device(ctx, G, pipeline, with_bw=True):
    import torch

    fwh, fwc, bwh, bwc = device(G)
    out = torch.empty(max(G.n, 1), dtype=torch.int32, device="cuda")
    st = K.Stats()
    ctx.scc_device(G.n, G.m, fwh, fwc, bwh if with_bw else None, bwc if with_bw else None, out, K.default_options(pipeline=pipeline), st)
    return out.cpu().numpy().view(np.uint32)[: G.n].copy(), st


@pytest.mark.parametrize("pipeline", PIPELINES)
def test_known_answer(ctx, pipeline):
    ids, _ = run_device(ctx, kat_graph(), pipeline)
    assert np.array_equal(ids, KAT_IDS)


@pytest.mark.parametrize("pipeline", PIPELINES)
def test_fuzzy_sweep(ctx, pipeline):
    """Planted partitions: the n < 300 sweep of test/test_tarjan_fuzzy.cpp
    (every 7th n here) and the n of test_mpi/test_scc_fuzzy.cpp."""
    ns = sorted(set(range(1, 300, 7)) | {1, 6, 8, 16, 33, 64})
    for key, G, planted in fuzzy_cases(ns, seeds=(0, 1), degrees=(0.5, 1.0, 4.0)):
        ids, _ = run_device(ctx, G, pipeline)
        assert np.array_equal(ids, planted), key


@pytest.mark.parametrize("pipeline", PIPELINES)
def test_edge_cases(ctx, pipeline):
    for name, G in edge_case_graphs():
        ids, _ = run_device(ctx, G, pipeline)
        assert np.array_equal(ids, O.tarjan(G)), name


@pytest.mark.parametrize("pipeline", PIPELINES)
@pytest.mark.parametrize("shape", ["gnm16", "rmat14", "rmat16", "rgg14", "rgg16"])
def test_synthetic_vs_tarjan(ctx, pipeline, shape):
    G = {
        "gnm16": lambda: O.gnm(1 << 16, 1 << 19, 1),
        "rmat14": lambda: O.rmat(14, 16, 2),
        "rmat16": lambda: O.rmat(16, 16, 2),
        "rgg14": lambda: O.rgg(1 << 14, 3),
        "rgg16": lambda: O.rgg(1 << 16, 3),
    }[shape]()
    ids, st = run_device(ctx, G, pipeline)
    assert np.array_equal(ids, O.tarjan(G))
    assert sum(st.decided[i] for i in range(8)) == G.n


def test_reference_scc_equal(ctx):
    """Bit-identical to the reference's own kaspan::scc after normalise."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    for G in (O.gnm(1 << 14, 1 << 17, 5), O.rmat(13, 8, 9), O.rgg(1 << 13, 4)):
        ref, _ = O.ref_scc(G)
        for p in PIPELINES:
            ids, _ = run_device(ctx, G, p)
            assert np.array_equal(ids, ref)


def test_host_api_and_device_transpose(ctx):
    G = O.rmat(12, 8, 11)
    want = O.tarjan(G)
    got = ctx.scc(G.n, G.fwh, G.fwc, G.bwh, G.bwc)
    assert np.array_equal(got, want)
    got2 = ctx.scc(G.n, G.fwh, G.fwc)  # bw built on the device
    assert np.array_equal(got2, want)
    ids, _ = run_device(ctx, G, K.PIPELINE_FAST, with_bw=False)
    assert np.array_equal(ids, want)


def test_invalid_graph_rejected(ctx):
    G = O.gnm(64, 256, 3)
    bad = G.fwc.copy()
    bad[5] = 1000  # id >= n: caught by validation before any traversal
    with pytest.raises(K.KspnError) as e:
        ctx.scc(G.n, G.fwh, bad, G.bwh, G.bwc)
    assert e.value.status == 2
    heads = G.fwh.copy()
    heads[10], heads[11] = heads[11], heads[10] + 1  # offsets decrease
    with pytest.raises(K.KspnError) as e:
        ctx.scc(G.n, heads, G.fwc, G.bwh, G.bwc)
    assert e.value.status == 2
    # the context stays usable
    assert np.array_equal(ctx.scc(G.n, G.fwh, G.fwc, G.bwh, G.bwc), O.tarjan(G))


def test_iteration_cap_reports_timeout(ctx):
    """A level cap of 1 ends the search with KSPN_ERR_TIMEOUT, context intact."""
    G = O.from_edges(1000, np.arange(1000, dtype=np.uint32), (np.arange(1000, dtype=np.uint32) + 1) % 1000)
    opt = K.default_options(max_levels=1)
    with pytest.raises(K.KspnError) as e:
        ctx.scc(G.n, G.fwh, G.fwc, G.bwh, G.bwc, options=opt)
    assert e.value.status == 4
    assert np.array_equal(ctx.scc(G.n, G.fwh, G.fwc, G.bwh, G.bwc), O.tarjan(G))


@pytest.mark.parametrize("graph,drop", [("rmat", 1), ("rmat", 2), ("rmat", 4), ("cycle", 18), ("cycle", 19)])
def test_barrier_wait_limit_reports_timeout(ctx, graph, drop):
    """The resident launch's grid barrier gives up after its wait limit: the
    grid's last block leaves barrier `drop` without arriving (the test hook
    kspn_options.drop_barrier, a block that never arrives), the other blocks'
    bounded waits run out, the launch ends through the barrier's error word,
    and the call reports KSPN_ERR_TIMEOUT.  The next call on the same context
    is exact.  On the long cycle the dropped barriers lie where the search
    moves to its worklist tail (after 16 levels)."""
    if graph == "rmat":
        G = O.rmat(14, 8, 3)
    else:
        n = 60000
        c = np.arange(n, dtype=np.uint32)
        G = O.from_edges(n, c, (c + 1) % n)
    want = O.tarjan(G)
    for limit in (1 << 10, 1 << 14):
        with pytest.raises(K.KspnError) as e:
            ctx.scc(G.n, G.fwh, G.fwc, G.bwh, G.bwc, options=K.default_options(drop_barrier=drop, wait_limit=limit))
        assert e.value.status == 4
        assert "barrier" in str(e.value)
        assert np.array_equal(ctx.scc(G.n, G.fwh, G.fwc, G.bwh, G.bwc), want)


@pytest.mark.parametrize("variant", sorted(K.PIPELINES))
def test_variant_matches_reference(ctx, variant):
    """Each reference entry point (kaspan::scc and variant/*.hpp, compiled
    from its sources) and the kspn pipeline of the same name give the same
    partition after the min-id relabel."""
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    graphs = [kat_graph(), O.gnm(1 << 12, 1 << 14, 3), O.rmat(12, 8, 5), O.rgg(1 << 12, 6)]
    graphs += [G for _, G, _ in fuzzy_cases((40, 200), seeds=(3,), degrees=(1.0, 4.0))]
    for G in graphs:
        ref, _ = O.ref_scc(G, variant)
        ids, _ = run_device(ctx, G, K.PIPELINES[variant])
        assert np.array_equal(ids, ref), (variant, G.n, G.m)
