"""A shard of the batch mix (kaspan_b200.graphs.batch(graphs=...)) holds
exactly the graphs the whole mix holds, and decomposes to the same ids."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import kaspan_b200.graphs as KG

pytestmark = pytest.mark.gpu


def test_shard_matches_whole(ctx):
    import torch

    full = KG.batch(ctx, 64, 21, 6, 12)
    parts = KG.batch_partition(full.sizes.astype(np.float64), 3)
    want = torch.empty(full.n, dtype=torch.int32, device="cuda")
    ctx.scc_batched(full.count, full.n, full.vtx_off, full.fwh, full.fwc, full.bwh, full.bwc, want)
    want = want.cpu().numpy().view(np.uint32)
    vo = np.concatenate([[0], np.cumsum(full.sizes, dtype=np.uint64)])
    for part in parts:
        sh = KG.batch(ctx, 64, 21, 6, 12, graphs=part)
        for j, g in enumerate(part[:5]):
            a, b = full.graph(int(g)), sh.graph(j)
            assert a[0] == b[0] and all(np.array_equal(x, y) for x, y in zip(a[1:], b[1:]))
        out = torch.empty(sh.n, dtype=torch.int32, device="cuda")
        ctx.scc_batched(sh.count, sh.n, sh.vtx_off, sh.fwh, sh.fwc, sh.bwh, sh.bwc, out)
        got = out.cpu().numpy().view(np.uint32)
        svo = np.concatenate([[0], np.cumsum(sh.sizes, dtype=np.uint64)])
        for j, g in enumerate(part):
            assert np.array_equal(got[int(svo[j]): int(svo[j + 1])], want[int(vo[g]): int(vo[g + 1])])
