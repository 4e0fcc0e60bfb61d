"""CPU: the C restatement (oracle/kspn_oracle.c) pinned against the
reference's own code (oracle/_ref, compiled from its sources) and against
the committed golden fixtures (tests/golden, made by make_golden.py from the
reference).  No GPU."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle as O
from kspn_testlib import KAT_IDS, edge_case_graphs, full_bits, fuzzy_cases, kat_graph

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def ref():
    R = O.ref_lib()
    if R is None:
        pytest.skip("oracle/_ref not built")
    return R


def test_known_answer_tiny():
    G = kat_graph()
    assert np.array_equal(O.tarjan(G), KAT_IDS)
    ids, _, _ = O.scc(G)
    assert np.array_equal(ids, KAT_IDS)


def test_known_answer_reference_all_variants():
    ref()
    G = kat_graph()
    for v in O.VARIANTS:
        ids, _ = O.ref_scc(G, v)
        assert np.array_equal(ids, KAT_IDS), v
    assert np.array_equal(O.ref_tarjan(G)[0], KAT_IDS)


def test_fuzzy_planted_tarjan_sweep():
    """test/test_tarjan_fuzzy.cpp:17-40 strategy: n < 300, d in {0.5, 1, 4}."""
    for key, G, planted in fuzzy_cases(range(0, 300, 3), seeds=(0, 1), degrees=(0.5, 1.0, 4.0)):
        if G.n == 0:
            continue
        assert np.array_equal(O.tarjan(G), planted), key


def test_fuzzy_planted_pipelines_vs_reference():
    """test_mpi/test_scc_fuzzy.cpp:31-80 n values, all seven reference
    pipelines and the restated default pipeline agree with the plant."""
    ref()
    for key, G, planted in fuzzy_cases((1, 6, 8, 16, 33, 64), seeds=range(6), degrees=(0.5, 1.0, 4.0, -1.0)):
        s, _, _ = O.scc(G)
        assert np.array_equal(s, planted), key
        for v in O.VARIANTS:
            r, _ = O.ref_scc(G, v)
            assert np.array_equal(r, planted), (key, v)


def test_edge_cases_vs_reference():
    ref()
    for name, G in edge_case_graphs():
        t = O.tarjan(G)
        assert np.array_equal(O.ref_tarjan(G)[0], t), name
        assert np.array_equal(O.scc(G)[0], t), name
        assert np.array_equal(O.ref_scc(G)[0], t), name


@pytest.mark.parametrize("shape", ["gnm", "rmat", "rgg"])
def test_synthetic_vs_reference(shape):
    ref()
    G = {"gnm": lambda: O.gnm(1 << 14, 1 << 17, 1), "rmat": lambda: O.rmat(14, 16, 2), "rgg": lambda: O.rgg(1 << 14, 3)}[shape]()
    t = O.tarjan(G)
    assert np.array_equal(O.ref_tarjan(G)[0], t)
    assert np.array_equal(O.ref_scc(G)[0], t)
    assert np.array_equal(O.scc(G)[0], t)


def _phase_graphs():
    out = [kat_graph()] + [G for _, G in edge_case_graphs()]
    out += [G for _, G, _ in fuzzy_cases((33, 64, 150), seeds=(0, 1), degrees=(1.0, 4.0))]
    out += [O.gnm(1 << 12, 1 << 15, 1), O.rmat(12, 16, 2), O.rgg(1 << 12, 3)]
    return out


def test_phases_vs_reference():
    """Each restated phase leaves the reference phase's exact state."""
    R = ref()
    L = O.lib()
    for G in _phase_graphs():
        n = G.n
        bits = full_bits(n)
        sid_r = np.full(max(n, 1), O.UNDECIDED, np.uint32)
        pivot_r = R.kref_trim_1_first(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid_r)
        und, sid = O.new_state(n)
        pivot = L.orc_trim_1_first(n, G.fwh, G.bwh, und, sid, None)
        assert pivot == pivot_r
        assert np.array_equal(und[:n], O.bytes_from_bits(bits, n))
        if pivot < n:
            R.kref_fw_bw(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid_r, pivot)
            L.orc_fw_bw(n, G.fwh, G.fwc, G.bwh, G.bwc, und, sid, pivot)
            assert np.array_equal(und[:n], O.bytes_from_bits(bits, n))
            assert np.array_equal(sid[:n], sid_r[:n])
        R.kref_trim_1_normal(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid_r)
        L.orc_trim_1_normal(n, G.fwh, G.fwc, G.bwh, G.bwc, und, sid)
        assert np.array_equal(und[:n], O.bytes_from_bits(bits, n))
        for rot in range(1, 9):
            if not und[:n].any():
                break
            R.kref_label_search_pull(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid_r, rot)
            L.orc_label_search_pull(n, G.fwh, G.fwc, G.bwh, G.bwc, und, sid, rot, None)
            assert np.array_equal(und[:n], O.bytes_from_bits(bits, n)), rot
            assert np.array_equal(sid[:n], sid_r[:n]), rot


def test_trim_exhaustive_first_vs_reference():
    R = ref()
    L = O.lib()
    for G in _phase_graphs():
        n = G.n
        bits = full_bits(n)
        sid_r = np.full(max(n, 1), O.UNDECIDED, np.uint32)
        od_r = np.zeros(max(n, 1), np.uint32)
        id_r = np.zeros(max(n, 1), np.uint32)
        R.kref_trim_1_exhaustive_first(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid_r, od_r, id_r)
        und, sid = O.new_state(n)
        od = np.zeros(max(n, 1), np.uint32)
        idg = np.zeros(max(n, 1), np.uint32)
        L.orc_trim_1_exhaustive_first(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, und, sid, od, idg)
        live = O.bytes_from_bits(bits, n).astype(bool)
        assert np.array_equal(und[:n].astype(bool), live)
        assert np.array_equal(od[:n][live], od_r[:n][live])
        assert np.array_equal(idg[:n][live], id_r[:n][live])
        # the restated fixpoint decides a superset, never a vertex of a non-trivial SCC
        und2, sid2 = O.new_state(n)
        L.orc_trim_1_fixpoint(n, G.fwh, G.fwc, G.bwh, G.bwc, und2, sid2)
        assert not (und2[:n] & ~und[:n].astype(bool)).any()
        t = O.tarjan(G)
        sizes = np.bincount(t, minlength=max(n, 1))
        assert (sizes[t[und2[:n] == 0]] == 1).all()


def test_generators_deterministic_and_shaped():
    a = O.rmat_edges(10, 8, 3)
    b = O.rmat_edges(10, 8, 3)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    c = O.rmat_edges(10, 8, 4)
    assert not np.array_equal(a[0], c[0])
    # the permutation is a bijection of [0, 2^scale)
    key = O.lib().orc_seed_key(3 ^ 0x5045524D55544531)
    for scale in (1, 5, 10, 11):
        img = {O.lib().orc_rmat_perm(x, scale, key) for x in range(1 << scale)}
        assert img == set(range(1 << scale))
    # G(n, m): uniform endpoints
    s, d = O.gnm_edges(1 << 10, 1 << 16, 9)
    assert s.max() < 1 << 10 and abs(np.bincount(s).mean() - 64) < 1
    # RGG: about 4n directed edges at mean undirected degree 8
    G = O.rgg(1 << 14, 3)
    assert 3.6 < G.m / G.n < 4.1


def test_golden_fixtures():
    """The oracle reproduces the reference outputs committed in tests/golden."""
    path = os.path.join(GOLDEN, "reference_outputs.json")
    with open(path) as f:
        cases = json.load(f)
    assert len(cases) >= 10
    for case in cases:
        G = _golden_graph(case["graph"])
        assert G.m == case["m"], case["graph"]
        ids = O.tarjan(G)
        assert _digest(ids) == case["tarjan_digest"], case["graph"]
        assert _digest(O.scc(G)[0]) == case["scc_digest"], case["graph"]
        und, sid = O.new_state(G.n)
        assert O.lib().orc_trim_1_first(G.n, G.fwh, G.bwh, und, sid, None) == case["trim_1_first_pivot"]
        if "ids" in case:
            assert ids.tolist() == case["ids"]
        _, pd, calls = O.scc(G)
        assert pd.tolist() == case["phase_decided"], case["graph"]
        assert calls == case["label_calls"], case["graph"]


def _digest(a: np.ndarray) -> str:
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()[:32]


def _golden_graph(spec: dict):
    kind = spec["kind"]
    if kind == "kat":
        return kat_graph()
    if kind == "fuzzy":
        return O.fuzzy(spec["seed"], spec["n"], spec["d"])[0]
    if kind == "gnm":
        return O.gnm(spec["n"], spec["draws"], spec["seed"])
    if kind == "rmat":
        return O.rmat(spec["scale"], spec["ef"], spec["seed"], spec.get("a", 0.57), spec.get("b", 0.19), spec.get("c", 0.19))
    if kind == "rgg":
        return O.rgg(spec["n"], spec["seed"])
    if kind == "edge":
        return dict(edge_case_graphs())[spec["name"]]
    raise ValueError(kind)
