"""The manifest graph format on the device (kspn_manifest_load): pinned
chunks, raw copies and the decode kernel give the same arrays the
reference's own loader gives (oracle/_ref), for every entry width and both
byte orders; the loaded graph decomposes like Tarjan; out-of-range entries
and short files are errors."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import kaspan_b200.graphs as KG
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("head_bytes,csr_bytes,big", [(8, 4, False), (4, 4, True), (3, 2, False), (8, 8, True), (5, 3, True)])
def test_device_load_matches(ctx, tmp_path, head_bytes, csr_bytes, big):
    import torch

    g = O.rmat(12, 8, 3)
    path = K.manifest_write(str(tmp_path), "r", g.n, g.fwh, g.fwc, g.bwh, g.bwc, head_bytes, csr_bytes, big)
    G = KG.from_manifest(ctx, path)
    fwh, fwc, bwh, bwc = G.to_host()
    assert np.array_equal(fwh, g.fwh) and np.array_equal(bwh, g.bwh)
    assert np.array_equal(fwc[: g.m], g.fwc[: g.m]) and np.array_equal(bwc[: g.m], g.bwc[: g.m])
    if O.ref_lib() is not None:
        n, rfwh, rfwc, rbwh, rbwc = O.ref_manifest_load(path)
        assert np.array_equal(fwh, rfwh) and np.array_equal(fwc[: g.m], rfwc)
    out = torch.empty(G.n, dtype=torch.int32, device="cuda")
    ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out)
    assert np.array_equal(out.cpu().numpy().view(np.uint32), O.tarjan(g))


def test_large_chunked_load(ctx, tmp_path):
    """More entries than one 32 Mi-entry chunk: the double-buffered chunks."""
    g = O.gnm(1 << 20, 34 << 20, 9)
    path = K.manifest_write(str(tmp_path), "big", g.n, g.fwh, g.fwc, g.bwh, g.bwc, 8, 4, False)
    G = KG.from_manifest(ctx, path)
    fwh, fwc, bwh, bwc = G.to_host()
    assert np.array_equal(fwc[: g.m], g.fwc[: g.m]) and np.array_equal(bwh, g.bwh)


def test_out_of_range_and_short_files(ctx, tmp_path):
    g = O.gnm(200, 800, 2)
    bad = g.fwc.copy()
    bad[5] = g.n + 7  # an id >= n
    path = K.manifest_write(str(tmp_path), "bad", g.n, g.fwh, bad, g.bwh, g.bwc, 8, 4, False)
    with pytest.raises(K.KspnError) as e:
        KG.from_manifest(ctx, path)
    assert e.value.status == 2  # KSPN_ERR_INVALID_GRAPH
    path = K.manifest_write(str(tmp_path), "short", g.n, g.fwh, g.fwc, g.bwh, g.bwc, 8, 4, False)
    mf = K.manifest_read(path)
    with open(mf.bw_csr_path.decode(), "r+b") as f:
        f.truncate(10)
    with pytest.raises(K.KspnError):
        KG.from_manifest(ctx, path)
