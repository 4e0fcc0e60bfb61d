"""The learned pivot (no reference counterpart): the library's own CUDA
feature, forward, gradient and Adam kernels against the numpy restatement
in oracle/mlp.py (float tolerances stated per check), training on the GPU,
and what the trained model gains over the plain max(in * out) pivot at the
same (exact) output."""
from __future__ import annotations

import numpy as np
import pytest

import kaspan_b200 as K
import mlp as M
import oracle as O

pytestmark = pytest.mark.gpu


def _graph(ctx, scale=12, seed=5, decoys=3, fan=300):
    from kaspan_b200.pivot_train import decoy_rmat

    return decoy_rmat(ctx, scale, seed, 0.57, decoys=decoys, fan=fan)


def test_features_match_oracle(ctx):
    import torch

    G, hubs = _graph(ctx)
    fwh, fwc, bwh, bwc = G.to_host()
    verts = np.unique(np.concatenate([np.arange(0, G.n, 7), hubs])).astype(np.uint32)
    dv = torch.from_numpy(verts.view(np.int32).copy()).cuda()
    f = torch.empty((len(verts), K.MLP_FEATURES), dtype=torch.float32, device="cuda")
    ctx.mlp_features(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, dv, f)
    ref = M.features(fwh, fwc, bwh, bwc, verts)
    # FP32 sums of at most 64 integer degrees and log2f: 1e-5 absolute
    np.testing.assert_allclose(f.cpu().numpy(), ref, rtol=0, atol=1e-5)
    # the decoys' dead ends show in feature 4 (share of sampled out-neighbours
    # that survive trim round 1) and feature 6 (removed in trim round 2)
    fd = f.cpu().numpy()[np.isin(verts, hubs)]
    assert np.all(fd[:, 4] == 0.0) and np.all(fd[:, 6] == 0.5)


def test_forward_gradient_adam_match_oracle(ctx):
    import torch

    rng = np.random.default_rng(3)
    for n in (1, 37, 5000):
        params = (rng.standard_normal(K.MLP_PARAMS) * 0.3).astype(np.float32)
        x = rng.uniform(0, 1.2, (n, 8)).astype(np.float32)
        y = (rng.random(n) < 0.4).astype(np.float32)
        dp, dx, dy = (torch.from_numpy(a).cuda() for a in (params, x, y))
        z = torch.empty(n, dtype=torch.float32, device="cuda")
        ctx.mlp_forward(dx, dp, z)
        zr, _ = M.forward(params, x.astype(np.float64))
        # FP32 accumulation over 8 + 32 + 32 terms of BF16 weights: 1e-4 relative
        np.testing.assert_allclose(z.cpu().numpy(), zr, rtol=1e-4, atol=1e-5)
        g = torch.empty(K.MLP_PARAMS, dtype=torch.float32, device="cuda")
        loss = torch.empty(1, dtype=torch.float32, device="cuda")
        ctx.mlp_gradient(dx, dy, dp, g, loss)
        lr_, gr = M.loss_and_grad(params, x.astype(np.float64), y.astype(np.float64))
        assert abs(loss.item() - lr_) <= 1e-5 * max(1.0, abs(lr_))
        # gradients: FP32 sums in a different order (shared-memory and global
        # atomics): 1e-3 relative to the largest component, per component
        scale = np.abs(gr).max()
        np.testing.assert_allclose(g.cpu().numpy(), gr, rtol=0, atol=1e-3 * scale + 1e-7)
        # one Adam step (step 1: m = .1 g, v = .001 g^2)
        m = torch.zeros_like(g)
        v = torch.zeros_like(g)
        p2 = dp.clone()
        ctx.mlp_adam(p2, g, m, v, 0.01, 1)
        gg = g.cpu().numpy().astype(np.float64)
        mh, vh = 0.1 * gg / 0.1, 0.001 * gg * gg / 0.001
        want = params - 0.01 * mh / (np.sqrt(vh) + 1e-8)
        np.testing.assert_allclose(p2.cpu().numpy(), want, rtol=1e-5, atol=1e-6)


def test_training_lowers_loss(ctx):
    import torch

    from kaspan_b200.pivot_train import label_entropy, samples, train

    xs, ys = [], []
    for seed in (11, 12, 13, 14):
        G, hubs = _graph(ctx, scale=13, seed=seed, decoys=4 if seed % 2 else 0, fan=400)
        x, y = samples(ctx, G, hubs, k=256)
        xs.append(x)
        ys.append(y)
    X, Y = torch.cat(xs), torch.cat(ys)
    _, losses = train(ctx, X, Y, steps=300, lr=1e-2)
    # soft labels: the loss cannot go below their mean binary entropy; the
    # excess over that floor at least halves
    floor = label_entropy(Y)
    assert losses[-1][1] >= floor - 1e-4
    assert losses[-1][1] - floor < 0.5 * (losses[0][1] - floor), (losses, floor)


def test_learned_pivot_gains_over_plain(ctx):
    """Trained on decoy-hub R-MAT graphs, evaluated on held-out seeds: the
    learned pivot starts FW-BW inside the largest SCC, where the plain
    max(in * out) pivot starts at a decoy (a singleton SCC), so the learned
    run decides the giant component in FW-BW instead of in the later rounds
    -- with the identical partition."""
    import torch

    from kaspan_b200.pivot_train import samples, train

    xs, ys = [], []
    for seed in range(20, 28):
        G, hubs = _graph(ctx, scale=14, seed=seed, decoys=6 if seed % 2 else 0, fan=None)
        x, y = samples(ctx, G, hubs, k=512)
        xs.append(x)
        ys.append(y)
    params, _ = train(ctx, torch.cat(xs), torch.cat(ys), steps=400, lr=1e-2)
    ctx.set_pivot_model(params)
    try:
        for seed in (101, 103):
            G, hubs = _graph(ctx, scale=14, seed=seed, decoys=6, fan=None)
            res = {}
            for learned in (0, 1):
                out = torch.empty(G.n, dtype=torch.int32, device="cuda")
                st = K.Stats()
                ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, K.default_options(learned_pivot=learned), st)
                res[learned] = (out.cpu().numpy().view(np.uint32).copy(), st.as_dict())
            fwh, fwc, bwh, bwc = G.to_host()
            truth = O.tarjan(O.Graph(G.n, fwh, fwc, bwh, bwc))
            assert np.array_equal(res[0][0], truth) and np.array_equal(res[1][0], truth)
            plain, learned = res[0][1], res[1][1]
            assert plain["pivot"] in set(int(h) for h in hubs)  # the decoy wins max(in * out)
            big = int(np.bincount(truth).max())
            assert learned["decided"]["fwbw"] == big > plain["decided"]["fwbw"]
    finally:
        ctx.set_pivot_model(None)


def test_in_kernel_check_costs_no_launch(ctx):
    """Where the model accepts the plain max(in * out) pivot (no decoys), the
    learned rule adds no launch: the resident launch scores its own pivot
    during its first level and goes on."""
    import torch

    from kaspan_b200.pivot_train import samples, train

    xs, ys = [], []
    for seed in range(30, 36):
        G, hubs = _graph(ctx, scale=13, seed=seed, decoys=4 if seed % 2 else 0, fan=None)
        x, y = samples(ctx, G, hubs, k=512)
        xs.append(x)
        ys.append(y)
    params, _ = train(ctx, torch.cat(xs), torch.cat(ys), steps=400, lr=1e-2)
    ctx.set_pivot_model(params)
    try:
        for seed in (201, 202):
            G, _ = _graph(ctx, scale=14, seed=seed, decoys=0)
            res = {}
            for learned in (0, 1):
                out = torch.empty(G.n, dtype=torch.int32, device="cuda")
                st = K.Stats()
                ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, K.default_options(learned_pivot=learned), st)
                res[learned] = (out.cpu().numpy().view(np.uint32).copy(), st.as_dict())
            assert np.array_equal(res[0][0], res[1][0])
            plain, learned = res[0][1], res[1][1]
            assert learned["pivot"] == plain["pivot"]
            assert learned["kernel_launches"] == plain["kernel_launches"]
            assert learned["decided"] == plain["decided"]
    finally:
        ctx.set_pivot_model(None)


@pytest.mark.parametrize("pipeline", [K.PIPELINE_REFERENCE, K.PIPELINE_HPC_LIKE, K.PIPELINE_HPC_TRIM_EX, K.PIPELINE_TRIM_EX])
def test_learned_seed_order_exact(ctx, pipeline):
    """The label searches with the learned seed order (the shipped model
    ranks the seeds, kspn_options.learned_seeds) give the identical
    partition on every pipeline that runs them: planted-partition graphs
    and the synthetic shapes, against Tarjan."""
    import torch

    from kspn_testlib import device, fuzzy_cases

    model = K.default_pivot_model()
    if model is None:
        pytest.skip("no shipped pivot model")
    ctx.set_pivot_model(model)
    try:
        graphs = [G for _, G, _ in fuzzy_cases((37, 150, 299), seeds=(4,), degrees=(1.0, 4.0))]
        graphs += [O.rmat(13, 8, 3), O.rgg(1 << 13, 5), O.gnm(5000, 20000, 6)]
        calls = []
        for G in graphs:
            fwh, fwc, bwh, bwc = device(G)
            want = O.tarjan(G)
            for seeds in (0, 1):
                out = torch.empty(max(G.n, 1), dtype=torch.int32, device="cuda")
                st = K.Stats()
                ctx.scc_device(G.n, G.m, fwh, fwc, bwh, bwc, out, K.default_options(pipeline=pipeline, learned_seeds=seeds), st)
                assert np.array_equal(out.cpu().numpy().view(np.uint32)[: G.n], want), (G.n, seeds)
                calls.append(st.label_calls)
        assert sum(calls) > 0, "the pipeline should run label searches on these graphs"
    finally:
        ctx.set_pivot_model(None)
