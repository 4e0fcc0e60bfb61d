"""Heavy rows (over 2048 entries) in the resident launch, built so that
every heavy route runs: a hub whose in-row starts with 3000 vertices the
forward search never reaches and ends with one it does (a bottom-up sweep
cuts the row short, a fix-up step finds the late neighbour), and hubs
whose heavy out-rows all end at dead ends (left to the trim tail, which
counts them in slices).  Output bit-identical to the oracle Tarjan."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import kaspan_b200.graphs as KG
import oracle as O

pytestmark = pytest.mark.gpu


def _heavy_graph():
    rng = np.random.default_rng(1)
    src, dst = [], []
    C2 = 3000                      # a cycle the pivot never reaches: ids 0..2999
    src += list(range(C2)); dst += [(i + 1) % C2 for i in range(C2)]
    H = 5000                       # the hub
    src += list(range(C2)); dst += [H] * C2            # C2 -> H, first in H's in-row
    g0, g1 = 6000, 40000           # the giant: a dense random SCC on ids [6000, 40000)
    n_g = g1 - g0
    src += list(range(g0, g1)); dst += [g0 + (i + 1) % n_g for i in range(n_g)]   # a Hamiltonian cycle
    e = 60 * n_g                   # dense: its vertices' in * out beats H's and the decoys'; one of them is the pivot
    src += list(rng.integers(g0, g1, e)); dst += list(rng.integers(g0, g1, e))
    src += [g1 - 1]; dst += [H]    # the one reached in-neighbour, last in H's in-row
    src += [H]; dst += [g0]        # H -> giant: H belongs to the giant SCC
    # 3 hubs fed by one giant vertex each, with 2100 out-edges to dead ends:
    # undecided after FW-BW, their heavy out-rows counted in slices by the trim tail
    n = 60000
    dead = 44000
    for d in range(3):
        hub = 41000 + d
        src += [g0 + 7 * d]; dst += [hub]
        src += [hub] * 2100; dst += list(range(dead + d * 2100, dead + (d + 1) * 2100))
    return n, np.array(src, np.uint32), np.array(dst, np.uint32)


def test_heavy_routes_match_tarjan(ctx):
    import torch

    n, s, d = _heavy_graph()
    G = KG.from_edges(ctx, n, torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda())
    fwh, fwc, bwh, bwc = G.to_host()
    want = O.tarjan(O.Graph(n, fwh, fwc, bwh, bwc))
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    # bottom-up from the first level on (enter when frontier edges > m_u), so
    # H's in-row is swept bottom-up before the giant's last vertex is expanded
    for opt in (K.default_options(validate=0), K.default_options(validate=0, bu_enter_div=1000, bu_leave_div=1)):
        st = K.Stats()
        ctx.scc_device(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, opt, st)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
        d_ = st.as_dict()
        assert d_["heavy"]["cut_rows"] > 0 and d_["heavy"]["trim_seeds"] >= 3
        assert want[d_["pivot"]] == want[6000]  # the pivot lies in the giant
    assert d_["heavy"]["fixups"] > 0
    # H is in the giant SCC
    assert want[5000] == want[6000]


def _chain_graph():
    """A giant random SCC, chains of 3000 vertices into it and out of it
    (the trim tail peels them one vertex per level), and a chain vertex with
    2500 out-edges to dead ends (a heavy row inside the peeling)."""
    rng = np.random.default_rng(2)
    src, dst = [], []
    g0, g1 = 0, 20000
    n_g = g1 - g0
    src += list(range(g0, g1)); dst += [g0 + (i + 1) % n_g for i in range(n_g)]
    e = 20 * n_g
    src += list(rng.integers(g0, g1, e)); dst += list(rng.integers(g0, g1, e))
    nxt = g1
    for c in range(4):
        L = 3000
        ch = list(range(nxt, nxt + L)); nxt += L
        if c % 2 == 0:       # into the giant: ch[0] -> ch[1] -> ... -> giant
            src += ch[:-1]; dst += ch[1:]; src += [ch[-1]]; dst += [g0 + c]
        else:                # out of the giant: giant -> ch[0] -> ... -> ch[-1]
            src += [g0 + c]; dst += [ch[0]]; src += ch[:-1]; dst += ch[1:]
        if c == 0:           # a heavy vertex in the middle of the first chain
            hv = ch[L // 2]
            src += [hv] * 2500; dst += list(range(nxt, nxt + 2500)); nxt += 2500
    return nxt, np.array(src, np.uint32), np.array(dst, np.uint32)


def test_trim_worklist_tail(ctx):
    import torch

    n, s, d = _chain_graph()
    G = KG.from_edges(ctx, n, torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda())
    fwh, fwc, bwh, bwc = G.to_host()
    want = O.tarjan(O.Graph(n, fwh, fwc, bwh, bwc))
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    st = K.Stats()
    for _ in range(2):  # a second call reuses the (all-zero) worklist
        ctx.scc_device(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, K.default_options(validate=0), st)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
        assert st.as_dict()["trim_worklist"] == 1


def _long_cycle_graph(n_cyc=60000, heavy=False):
    """A cycle of n_cyc vertices (so both searches outlast the level loop and
    finish on the worklist), the pivot on it by degree, plus side chains
    that FW reaches but BW does not and vice versa (FW(p) and BW(p) each
    hold vertices outside the SCC), and with `heavy` a hub on the cycle
    whose out- and in-rows are sliced (slice items of both directions)."""
    rng = np.random.default_rng(7)
    src, dst = [], []
    cyc = np.arange(n_cyc)
    src += list(cyc); dst += list((cyc + 1) % n_cyc)
    n = n_cyc
    # the pivot: vertex 0 gets extra in and out edges from/to cycle vertices
    k = 40
    src += [0] * k; dst += list(rng.integers(1, n_cyc, k))
    src += list(rng.integers(1, n_cyc, k)); dst += [0] * k
    # side chains: out of the cycle (FW only) and into it (BW only)
    for start in rng.integers(0, n_cyc, 30):
        L = 500
        ids = np.arange(n, n + L); n += L
        src += [int(start)] + list(ids[:-1]); dst += list(ids)
    for start in rng.integers(0, n_cyc, 30):
        L = 500
        ids = np.arange(n, n + L); n += L
        src += list(ids); dst += list(ids[1:]) + [int(start)]
    if heavy:
        # vertex n_cyc // 2 (on the cycle) points at 5000 fresh dead ends and
        # is pointed at by 5000 fresh sources: both its rows are heavy
        h = n_cyc // 2
        outs = np.arange(n, n + 5000); n += 5000
        ins = np.arange(n, n + 5000); n += 5000
        src += [h] * 5000 + list(ins); dst += list(outs) + [h] * 5000
    return n, np.array(src, np.uint32), np.array(dst, np.uint32)


@pytest.mark.parametrize("heavy", [False, True])
def test_joint_worklist_search(ctx, heavy):
    import torch

    n, s, d = _long_cycle_graph(heavy=heavy)
    G = KG.from_edges(ctx, n, torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda())
    fwh, fwc, bwh, bwc = G.to_host()
    want = O.tarjan(O.Graph(n, fwh, fwc, bwh, bwc))
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    for _ in range(2):  # a second call reuses the (all-zero) worklist
        st = K.Stats()
        ctx.scc_device(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, K.default_options(validate=0), st)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
        dct = st.as_dict()
        assert dct["fwbw_joint"] == 1, "FW and BW run side by side"
        assert dct["search_worklist"] == 1, "and finish on the worklist together"


def _path_core_chain_graph():
    """Pivot p (largest in*out: 3000 in-edges from sources, 3000 out-edges to
    sinks, both decided by trim_1_first) -> a 12-vertex path -> a dense core
    of 20000 vertices (levels 13-15 top-down; level 16 turns bottom-up, and
    the level that builds its frontier from the sweeps' finds comes after
    level 16 with a small frontier, so it switches straight to the
    worklist) -> a 3000-vertex chain back to p.  One SCC of p + path +
    core + chain."""
    rng = np.random.default_rng(11)
    C, P, L, X = 20000, 12, 3000, 3000
    p = C
    path = np.arange(C + 1, C + 1 + P)
    chain = np.arange(C + 1 + P, C + 1 + P + L)
    sinks = np.arange(chain[-1] + 1, chain[-1] + 1 + X)
    srcs = np.arange(sinks[-1] + 1, sinks[-1] + 1 + X)
    n = int(srcs[-1]) + 1
    src, dst = [], []
    core = np.arange(C)
    src += list(core); dst += list((core + 1) % C)                      # the core is one cycle ...
    e = 20 * C
    src += list(rng.integers(0, C, e)); dst += list(rng.integers(0, C, e))  # ... and dense
    src += [p] + list(path[:-1]) + [int(path[-1])]; dst += list(path) + [0]  # p -> path -> core
    src += [1] + list(chain[:-1]) + [int(chain[-1])]; dst += list(chain) + [p]  # core -> chain -> p
    src += [p] * X + list(srcs); dst += list(sinks) + [p] * X
    return n, np.array(src, np.uint32), np.array(dst, np.uint32)


def test_bottom_up_then_worklist(ctx):
    import torch

    n, s, d = _path_core_chain_graph()
    G = KG.from_edges(ctx, n, torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda())
    fwh, fwc, bwh, bwc = G.to_host()
    want = O.tarjan(O.Graph(n, fwh, fwc, bwh, bwc))
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    for _ in range(2):
        st = K.Stats()
        ctx.scc_device(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, K.default_options(validate=0), st)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
        dct = st.as_dict()
        assert dct["levels_bottom_up"] > 0, "the search should run bottom-up levels in the core"
        assert dct["search_worklist"] == 1, "and finish on the worklist after them"


# The worklist tail leaves a find's take to its consumer until a warp's
# reservation passes half the worklist (4 M items and more), which no small
# graph reaches; kspn_options.aw_exact_after moves that switch so the exact
# branch (finds taken by the warp that found them) and the switch itself run
# here.  1: exact after the first reservation; 2000: mid-phase.
@pytest.mark.parametrize("after", [1, 2000])
@pytest.mark.parametrize("shape", ["joint", "joint_heavy", "bottom_up_then_worklist", "chain", "heavy"])
def test_worklist_exact_takes(ctx, shape, after):
    import torch

    n, s, d = {"joint": lambda: _long_cycle_graph(), "joint_heavy": lambda: _long_cycle_graph(heavy=True),
               "bottom_up_then_worklist": _path_core_chain_graph, "chain": _chain_graph, "heavy": _heavy_graph}[shape]()
    G = KG.from_edges(ctx, n, torch.from_numpy(s.view(np.int32)).cuda(), torch.from_numpy(d.view(np.int32)).cuda())
    fwh, fwc, bwh, bwc = G.to_host()
    want = O.tarjan(O.Graph(n, fwh, fwc, bwh, bwc))
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    for _ in range(2):  # the worklist must be left all zeros for the next call
        st = K.Stats()
        ctx.scc_device(n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, K.default_options(validate=0, aw_exact_after=after), st)
        assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
    if shape.startswith("joint"):
        assert st.as_dict()["search_worklist"] == 1
