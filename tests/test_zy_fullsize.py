"""Full-size parity on every benchmark configuration, in the default GPU run:
G(2^16, 2^19) (C1), R-MAT s24 (C2), RGG 2^24 (C3) and R-MAT s26 (C4) are
generated on the device at their full size, decomposed by the FAST
pipeline, and compared bit for bit with the reference's own Tarjan
(oracle/_ref, kaspan/scc/tarjan.hpp:124-136) on the same CSR; C1 and C2 are
also compared with the reference's own kaspan::scc (kaspan/scc/scc.hpp:21-87)
after normalise_scc_id.  The 4096-graph batch mix (C5) is decomposed by
kspn_scc_batched in one call and compared, graph by graph, with the
reference Tarjan of the whole mix as one graph with global ids (its SCCs are
the graphs' SCCs), through both batched routes.  Minutes of host time in all; collected before
test_zz_no_alloc.py."""
from __future__ import annotations

import time

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

SHAPES = {
    "c1_gnm16": lambda ctx, KG: KG.gnm(ctx, 1 << 16, 1 << 19, 1),
    "c2_rmat24": lambda ctx, KG: KG.rmat(ctx, 24, 16, 2),
    "c3_rgg24": lambda ctx, KG: KG.rgg(ctx, 1 << 24, 3),
    "c4_rmat26": lambda ctx, KG: KG.rmat(ctx, 26, 16, 4),
}
WITH_REFERENCE_SCC = {"c1_gnm16", "c2_rmat24"}


def _need_ref():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")


@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_full_size_vs_reference(ctx, shape):
    import torch

    import kaspan_b200.graphs as KG

    _need_ref()
    DG = SHAPES[shape](ctx, KG)
    out = torch.empty(DG.n, dtype=torch.int32, device="cuda")
    st = K.Stats()
    ctx.scc_device(DG.n, DG.m, DG.fwh, DG.fwc, DG.bwh, DG.bwc, out, K.default_options(), st)
    ids = out.cpu().numpy().view(np.uint32).copy()
    fwh, fwc, bwh, bwc = DG.to_host()
    del DG, out
    torch.cuda.empty_cache()
    n = len(fwh) - 1
    t0 = time.time()
    ref, secs = O.ref_tarjan(O.Graph(n, np.ascontiguousarray(fwh), np.ascontiguousarray(fwc), None, None))
    print(f"{shape}: n={n} m={int(fwh[-1])} reference tarjan {secs:.1f} s ({time.time() - t0:.1f} s wall), "
          f"kspn {st.ms_total:.2f} ms, components {int((ref == np.arange(n, dtype=np.uint32)).sum())}")
    assert np.array_equal(ids, ref)
    if shape in WITH_REFERENCE_SCC:
        ref_scc, secs = O.ref_scc(O.Graph(n, np.ascontiguousarray(fwh), np.ascontiguousarray(fwc), np.ascontiguousarray(bwh), np.ascontiguousarray(bwc)))
        print(f"{shape}: reference kaspan::scc {secs:.1f} s")
        assert np.array_equal(ids, ref_scc)


def test_full_batch_mix_vs_reference_tarjan(ctx):
    """C5: 4096 G(n, m) graphs, n = round(2^U[8, 18]), m = round(n U[0.8, 6])
    draws, seed 5 -- the whole mix in one kspn_scc_batched call."""
    import torch

    import kaspan_b200.graphs as KG

    _need_ref()
    B = KG.batch(ctx, 4096, 5)
    out = torch.empty(B.n, dtype=torch.int32, device="cuda")
    st = ctx.scc_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out, None)
    got = out.cpu().numpy().view(np.uint32).copy()
    # the mix as one graph with global ids (rows hold local ids): every row's
    # entries shifted by its graph's first vertex
    sizes = torch.from_numpy(np.asarray(B.sizes, dtype=np.int64)).cuda()
    first = torch.cumsum(sizes, 0) - sizes
    row_first = torch.repeat_interleave(first, sizes)
    deg = B.fwh[1:] - B.fwh[:-1]
    glob = (B.fwc[: B.m].to(torch.int64) + torch.repeat_interleave(row_first, deg)).to(torch.int32)
    fwh = B.fwh.cpu().numpy().view(np.uint64).copy()
    fwc = glob.cpu().numpy().view(np.uint32).copy()
    base = row_first.cpu().numpy().astype(np.uint64)
    del glob, deg, row_first, out
    torch.cuda.empty_cache()
    ref, secs = O.ref_tarjan(O.Graph(B.n, fwh, fwc, None, None))
    want = (ref.astype(np.uint64) - base).astype(np.uint32)
    print(f"C5: graphs={B.count} n={B.n} m={B.m} reference tarjan {secs:.1f} s, kspn {st.ms:.2f} ms, "
          f"small={st.graphs_small} large={st.graphs_large}")
    assert st.graphs_small + st.graphs_large == B.count
    assert np.array_equal(got, want)
    # route 1 (the mix as one graph through a super-source) on the same mix
    o = K.BatchOptions()
    K.lib().kspn_batch_options_default(__import__("ctypes").byref(o))
    o.route = 1
    out = torch.empty(B.n, dtype=torch.int32, device="cuda")
    st = ctx.scc_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out, o)
    print(f"C5 union route: kspn {st.ms:.2f} ms, taken={st.graphs_large == B.count}")
    assert np.array_equal(out.cpu().numpy().view(np.uint32), want)
