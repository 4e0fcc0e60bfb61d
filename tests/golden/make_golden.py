"""Regenerates tests/golden/reference_outputs.json from the REFERENCE's own
code (oracle/_ref/libkspn_ref.so, compiled from the reference sources by
oracle/Makefile) -- run where those sources are present:

    make -C oracle && python tests/golden/make_golden.py

For every case it records, from the reference: the edge count of the
generated graph, a digest of its Tarjan min-id labels (kaspan/scc/tarjan.hpp
via test_tarjan_vs_kaspan.cpp's naming), a digest of kaspan::scc's output
after normalise_scc_id, trim_1_first's pivot, the per-phase decided counts
and label-search calls of kaspan::scc (via the reference's phase functions),
and for small graphs the full label array.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

import oracle as O  # noqa: E402
from kspn_testlib import edge_case_graphs, full_bits, kat_graph  # noqa: E402
from test_oracle import _golden_graph  # noqa: E402

CASES = (
    [{"kind": "kat"}]
    + [{"kind": "edge", "name": name} for name, _ in edge_case_graphs()]
    + [{"kind": "fuzzy", "seed": 100 + i, "n": n, "d": d} for i, (n, d) in enumerate([(1, 1.0), (6, 0.5), (8, 4.0), (16, 1.0), (33, 4.0), (64, 0.5), (64, 4.0), (150, 1.0), (299, 4.0), (299, 0.5)])]
    + [
        {"kind": "gnm", "n": 1 << 16, "draws": 1 << 19, "seed": 1},
        {"kind": "gnm", "n": 1 << 12, "draws": 1 << 12, "seed": 2},
        {"kind": "rmat", "scale": 14, "ef": 16, "seed": 2},
        {"kind": "rmat", "scale": 16, "ef": 16, "seed": 2},
        {"kind": "rmat", "scale": 12, "ef": 16, "seed": 1000, "a": 0.45, "b": 0.25, "c": 0.25},
        {"kind": "rgg", "n": 1 << 14, "seed": 3},
        {"kind": "rgg", "n": 1 << 16, "seed": 3},
    ]
)


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.uint32).tobytes()).hexdigest()[:32]


def reference_phases(G):
    """kaspan::scc's phase sequence run through the reference's own phase
    functions: decided counts per phase and the number of label calls."""
    R = O.ref_lib()
    n = G.n
    bits = full_bits(n)
    sid = np.full(max(n, 1), O.UNDECIDED, np.uint32)

    def undecided():
        return int(O.bytes_from_bits(bits, n).sum())

    pd = [0, 0, 0, 0]
    pivot = R.kref_trim_1_first(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid)
    pd[0] = n - undecided()
    if undecided():
        before = undecided()
        R.kref_fw_bw(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid, pivot)
        pd[1] = before - undecided()
    if undecided():
        before = undecided()
        R.kref_trim_1_normal(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid)
        pd[2] = before - undecided()
    calls = 0
    while undecided():
        before = undecided()
        calls += 1
        R.kref_label_search_pull(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, bits, sid, calls)
        pd[3] += before - undecided()
    return pivot, pd, calls, sid[:n]


def main():
    if O.ref_lib() is None:
        sys.exit("oracle/_ref/libkspn_ref.so missing: run `make -C oracle` where the reference sources exist")
    out = []
    for spec in CASES:
        G = _golden_graph(spec)
        tar, _ = O.ref_tarjan(G)
        sc, _ = O.ref_scc(G)
        pivot, pd, calls, raw = reference_phases(G)
        assert np.array_equal(O.normalise(raw), sc)
        case = {
            "graph": spec,
            "m": G.m,
            "tarjan_digest": digest(tar),
            "scc_digest": digest(sc),
            "trim_1_first_pivot": int(pivot),
            "phase_decided": pd,
            "label_calls": calls,
            "components": int(len(np.unique(tar))),
        }
        if G.n <= 300:
            case["ids"] = tar.tolist()
        out.append(case)
        print(spec, G.n, G.m, pd, calls)
    with open(os.path.join(HERE, "reference_outputs.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
