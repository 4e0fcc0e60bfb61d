"""Full-size parity (run with KSPN_FULLSIZE=1; minutes of CPU time for the
reference's Tarjan): R-MAT s24 / s26, RGG 2^24 and G(2^16, 2^19) generated on
the device at their full size, decomposed by the FAST pipeline, and compared bit for bit with
the reference's own Tarjan (oracle/_ref, tarjan.hpp:20-136) on the same CSR.
Collected before test_zz_no_alloc.py."""
from __future__ import annotations

import os
import time

import numpy as np
import pytest

import kaspan_b200 as K
import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow,
              pytest.mark.skipif(os.environ.get("KSPN_FULLSIZE") != "1", reason="set KSPN_FULLSIZE=1 for full-size parity")]

SHAPES = {
    "rmat26": lambda ctx, KG: KG.rmat(ctx, 26, 16, 4),
    "rmat24": lambda ctx, KG: KG.rmat(ctx, 24, 16, 2),
    "rgg24": lambda ctx, KG: KG.rgg(ctx, 1 << 24, 3),
    "gnm16": lambda ctx, KG: KG.gnm(ctx, 1 << 16, 1 << 19, 1),
}


@pytest.mark.parametrize("shape", sorted(SHAPES))
def test_full_size_vs_reference_tarjan(ctx, shape):
    import torch

    import kaspan_b200.graphs as KG

    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    DG = SHAPES[shape](ctx, KG)
    out = torch.empty(DG.n, dtype=torch.int32, device="cuda")
    st = K.Stats()
    ctx.scc_device(DG.n, DG.m, DG.fwh, DG.fwc, DG.bwh, DG.bwc, out, K.default_options(), st)
    ids = out.cpu().numpy().view(np.uint32)
    fwh, fwc, _, _ = DG.to_host()
    del DG, out
    torch.cuda.empty_cache()
    n = len(fwh) - 1
    t0 = time.time()
    ref, secs = O.ref_tarjan(O.Graph(n, np.ascontiguousarray(fwh), np.ascontiguousarray(fwc), None, None))
    print(f"{shape}: n={n} m={int(fwh[-1])} reference tarjan {secs:.1f} s ({time.time() - t0:.1f} s wall), "
          f"kspn {st.ms_total:.2f} ms, components {int((ref == np.arange(n, dtype=np.uint32)).sum())}")
    assert np.array_equal(ids, ref)
