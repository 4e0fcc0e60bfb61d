"""The autotuner (no reference counterpart): the settings it returns give
the same ids as the defaults (the tuner itself checks every candidate
against the first run on the device), and they are never slower than the
defaults as it measured them."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import kaspan_b200.graphs as KG
import oracle as O

pytestmark = pytest.mark.gpu


def test_autotune_fast_pipeline(ctx):
    import torch

    G = KG.rmat(ctx, 16, 16, 7)
    out = torch.empty(G.n, dtype=torch.int32, device="cuda")
    best, rep = ctx.autotune(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, reps=2)
    assert rep.candidates >= 10
    assert rep.best_ms <= rep.default_ms
    ids = out.cpu().numpy().view(np.uint32).copy()
    fwh, fwc, bwh, bwc = G.to_host()
    assert np.array_equal(ids, O.tarjan(O.Graph(G.n, fwh, fwc, bwh, bwc)))
    # the chosen settings, run again through the normal entry point
    out2 = torch.empty_like(out)
    ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out2, best)
    assert np.array_equal(out2.cpu().numpy().view(np.uint32), ids)


def test_autotune_batched(ctx):
    import torch

    B = KG.batch(ctx, 200, 13, 6, 14, 0.8, 6.0)
    out = torch.empty(B.n, dtype=torch.int32, device="cuda")
    best, rep = ctx.autotune_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out, reps=2)
    assert rep.candidates >= 8
    assert rep.best_ms <= rep.default_ms
    ids = out.cpu().numpy().view(np.uint32).copy()
    out2 = torch.empty_like(out)
    ctx.scc_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out2)
    assert np.array_equal(out2.cpu().numpy().view(np.uint32), ids)
