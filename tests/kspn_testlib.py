"""Shared helpers for the kspn tests: graph fixtures from the CPU oracle,
device copies, and the reference bitset <-> numpy conversions."""
from __future__ import annotations

import numpy as np

import oracle as O

# The 7-vertex, 11-edge known-answer graph of
# extern/ispan_test/test_ispan_tiny.cpp:21-90 (SCCs {0,2}, {1,3,4}, {5,6}).
KAT_EDGES = [(0, 2), (1, 0), (1, 2), (1, 3), (2, 0), (3, 2), (3, 4), (4, 1), (4, 3), (5, 6), (6, 5)]
KAT_IDS = np.array([0, 1, 0, 1, 1, 5, 5], np.uint32)


def kat_graph() -> O.Graph:
    src = np.array([u for u, _ in KAT_EDGES], np.uint32)
    dst = np.array([v for _, v in KAT_EDGES], np.uint32)
    return O.from_edges(7, src, dst)


def edge_case_graphs():
    """(name, Graph) pairs covering the shapes the reference's tests and
    the domain call for: empty, isolated, self-loops, duplicates, cycles,
    chains, stars, cliques."""
    out = []
    out.append(("n1_empty", O.from_edges(1, [], [])))
    out.append(("n5_isolated", O.from_edges(5, [], [])))
    out.append(("selfloops", O.from_csr(4, np.array([0, 1, 3, 4, 4], np.uint64), np.array([0, 1, 2, 2], np.uint32))))
    # duplicates and self-loops kept in the CSR (the boundary allows both)
    out.append(("dups", O.from_csr(3, np.array([0, 3, 5, 6], np.uint64), np.array([1, 1, 2, 0, 0, 1], np.uint32))))
    n = 1000
    cyc = np.arange(n, dtype=np.uint32)
    out.append(("big_cycle", O.from_edges(n, cyc, (cyc + 1) % n)))
    out.append(("chain", O.from_edges(n, cyc[:-1], cyc[1:])))
    # chain of 2-cycles: i <-> i+1 for even i, i+1 -> i+2
    a = np.arange(0, n - 1, 2, dtype=np.uint32)
    src = np.concatenate([a, a + 1, (a + 1)[:-1]])
    dst = np.concatenate([a + 1, a, (a + 2)[:-1]])
    out.append(("pair_chain", O.from_edges(n, src, dst)))
    star_out = np.zeros(n - 1, np.uint32)
    out.append(("star", O.from_edges(n, np.concatenate([star_out, cyc[1:]]), np.concatenate([cyc[1:], star_out]))))
    k = 40
    u, v = np.meshgrid(np.arange(k, dtype=np.uint32), np.arange(k, dtype=np.uint32))
    out.append(("clique", O.from_edges(k, u.ravel(), v.ravel())))
    # two cliques joined one way, plus a tail
    src = np.concatenate([u.ravel(), u.ravel() + k, np.array([0, 2 * k - 1, 2 * k], np.uint32)])
    dst = np.concatenate([v.ravel(), v.ravel() + k, np.array([k, 2 * k, 2 * k + 1], np.uint32)])
    out.append(("two_cliques_tail", O.from_edges(2 * k + 2, src, dst)))
    return out


def device(G: O.Graph):
    import torch

    def t(a, dt, cnt):
        a = np.ascontiguousarray(a[: max(cnt, 1)])
        return torch.from_numpy(a.view(dt).copy()).cuda()

    m = G.m
    return (t(G.fwh, np.int64, G.n + 1), t(G.fwc, np.int32, m), t(G.bwh, np.int64, G.n + 1), t(G.bwc, np.int32, m))


def full_bits(n: int) -> np.ndarray:
    """Reference bitset with bits [0, n) set (make_bits_filled)."""
    words = np.zeros((n + 63) // 64 or 1, np.uint64)
    full, rem = divmod(n, 64)
    words[:full] = np.uint64(0xFFFFFFFFFFFFFFFF)
    if rem:
        words[full] = np.uint64((1 << rem) - 1)
    return words


def bits_to_dev(words: np.ndarray):
    import torch

    return torch.from_numpy(words.view(np.int64).copy()).cuda()


def dev_to_bits(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint64).copy()


def u32_to_dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32).copy()).cuda()


def dev_to_u32(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32).copy()


def bits_equal(a: np.ndarray, b: np.ndarray, n: int) -> bool:
    return np.array_equal(O.bytes_from_bits(a, n), O.bytes_from_bits(b, n))


def fuzzy_cases(ns, seeds, degrees):
    for n in ns:
        for s in seeds:
            for d in degrees:
                G, planted = O.fuzzy(1_000_003 * s + 7919 * n + int(d * 100), n, d)
                yield (n, s, d), G, planted
