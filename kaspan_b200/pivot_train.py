"""Training data and training loop of the learned pivot (no reference
counterpart), on the GPU through the library's own kernels.

    python -m kaspan_b200.pivot_train [--out kaspan_b200/pivot_model.npy]

Training set: the 64 R-MAT scale-20 graphs with a ~ U[.45, .65] and
b = c = (1 - a - .05) / 2, seeds 1000..1063; every second one carries
decoy hubs (a vertex with `fan` in-edges from random vertices and `fan`
out-edges to fresh dead ends, `fan` sized so that its in * out beats every
real vertex, while its SCC is itself).  Labels come from plain runs of the FAST
pipeline and are soft: log2(1 + |SCC(v)|) / log2(1 + |largest SCC|), 1 in
the largest SCC, near 0 for a singleton -- a pivot is worth the share of
the graph its FW-BW round decides, so a vertex of a large SCC that is not
the largest is not taught as a miss.  The logit's sign is the decision: a
vertex is accepted where the model predicts a label of at least 1/2 (an
SCC of about the square root of the largest one or more).  Samples: the
1024 vertices with the largest in * out, plus the decoys.  Loss: mean
binary cross-entropy against the soft labels (its floor is the labels'
mean binary entropy); optimiser: Adam (kspn_mlp_gradient / kspn_mlp_adam).
"""
from __future__ import annotations

import argparse
import os

import numpy as np

from . import MLP_FEATURES, MLP_PARAMS, PIPELINE_FAST, Context, default_options
from . import graphs as KG

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "pivot_model.npy")


def decoy_rmat(ctx: Context, scale: int, seed: int, a: float, decoys: int = 0, fan: int | None = None, edge_factor: int = 16):
    """R-MAT (a, b = c = (1 - a - .05) / 2) plus `decoys` decoy hubs with
    their dead ends; returns (DeviceGraph, decoy ids).  fan=None sizes the
    decoys so that fan^2 exceeds 1.44 x the largest in * out of the R-MAT
    edge list (counted with duplicates): each decoy then wins max(in * out)."""
    import torch

    b = (1.0 - a - 0.05) / 2.0
    n0 = 1 << scale
    draws = edge_factor << scale
    ta, tab, tabc = KG.rmat_thresholds(a, b, b)
    base_s = torch.empty(draws, dtype=torch.int32, device="cuda")
    base_d = torch.empty(draws, dtype=torch.int32, device="cuda")
    ctx.gen_rmat(scale, draws, seed, ta, tab, tabc, True, base_s, base_d)
    if fan is None:
        outd = torch.bincount(base_s.long(), minlength=n0).double()
        ind = torch.bincount(base_d.long(), minlength=n0).double()
        fan = int(1.2 * float((outd * ind).max().item()) ** 0.5) + 1
    extra = 2 * decoys * fan
    src = torch.empty(draws + extra, dtype=torch.int32, device="cuda")
    dst = torch.empty(draws + extra, dtype=torch.int32, device="cuda")
    src[:draws] = base_s
    dst[:draws] = base_d
    del base_s, base_d
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    hubs = np.arange(n0, n0 + decoys, dtype=np.int64)
    for d in range(decoys):
        o = draws + 2 * d * fan
        hub = n0 + d
        src[o: o + fan] = torch.randint(0, n0, (fan,), generator=gen, device="cuda", dtype=torch.int32)
        dst[o: o + fan] = hub
        src[o + fan: o + 2 * fan] = hub
        dst[o + fan: o + 2 * fan] = torch.arange(n0 + decoys + d * fan, n0 + decoys + (d + 1) * fan, device="cuda", dtype=torch.int32)
    n = n0 + decoys + decoys * fan
    torch.cuda.synchronize()  # the edge list was written on torch's stream
    return KG.from_edges(ctx, n, src, dst), hubs


def scc_size_labels(ctx: Context, G) -> "torch.Tensor":
    """log2(1 + |SCC(v)|) / log2(1 + |largest SCC|) per vertex (plain FAST
    run): 1.0 in the largest SCC."""
    import torch

    out = torch.empty(G.n, dtype=torch.int32, device="cuda")
    ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, default_options(pipeline=PIPELINE_FAST))
    ids = out.long()
    size = torch.bincount(ids, minlength=G.n).double()
    return (torch.log2(1.0 + size[ids]) / torch.log2(1.0 + size.max())).float()


def label_entropy(Y) -> float:
    """Mean binary entropy of soft labels (nats): the BCE loss's floor."""
    import torch

    y = Y.double().clamp(1e-12, 1 - 1e-12)
    return float((-(y * torch.log(y) + (1 - y) * torch.log(1 - y))).mean().item())


def candidates(G, k: int = 1024, extra=None):
    """The k vertices with the largest in * out (plus `extra`)."""
    import torch

    outd = (G.fwh[1:] - G.fwh[:-1]).double()
    ind = (G.bwh[1:] - G.bwh[:-1]).double()
    top = torch.topk(outd * ind, min(k, G.n)).indices
    if extra is not None and len(extra):
        top = torch.unique(torch.cat([top, torch.as_tensor(extra, device="cuda", dtype=top.dtype)]))
    return top.to(torch.int32)


def features(ctx: Context, G, verts):
    import torch

    f = torch.empty((verts.numel(), MLP_FEATURES), dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()  # verts may come from torch's stream
    ctx.mlp_features(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, verts, f)
    return f


def samples(ctx: Context, G, hubs, k: int = 1024):
    import torch

    y = scc_size_labels(ctx, G)
    c = candidates(G, k, hubs)
    return features(ctx, G, c), y[c.long()].contiguous()


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform(+-1/sqrt(fan_in)) weights, zero biases."""
    rng = np.random.default_rng(seed)
    p = np.zeros(MLP_PARAMS, np.float32)
    o = 0
    for rows, cols in ((32, 8), (32, 0), (32, 32), (32, 0), (32, 0), (1, 0)):
        size = rows * max(cols, 1)
        if cols:
            p[o: o + size] = rng.uniform(-1, 1, size) / np.sqrt(cols)
        o += size
    p[256 + 32 + 1024 + 32: 256 + 32 + 1024 + 32 + 32] = rng.uniform(-1, 1, 32) / np.sqrt(32)  # w3
    return p


def train(ctx: Context, X, Y, steps: int = 400, lr: float = 1e-2, seed: int = 0, params=None):
    """Adam on the mean BCE; returns (params float32[MLP_PARAMS], losses)."""
    import torch

    p = torch.from_numpy(init_params(seed) if params is None else np.asarray(params, np.float32)).cuda()
    g = torch.zeros_like(p)
    m = torch.zeros_like(p)
    v = torch.zeros_like(p)
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()  # inputs written on torch's stream
    losses = []
    for step in range(1, steps + 1):
        ctx.mlp_gradient(X, Y, p, g, loss)
        ctx.mlp_adam(p, g, m, v, lr, step)
        if step == 1 or step % 50 == 0 or step == steps:
            losses.append((step, float(loss.item())))
    return p.cpu().numpy(), losses


def training_set(ctx: Context, count: int = 64, scale: int = 20, first_seed: int = 1000):
    """(features, labels) of the C4 training graphs, decoys on every second."""
    import torch

    rng = np.random.default_rng(first_seed)
    xs, ys = [], []
    for i in range(count):
        a = float(rng.uniform(0.45, 0.65))
        G, hubs = decoy_rmat(ctx, scale, first_seed + i, a, decoys=8 if i % 2 else 0)
        x, y = samples(ctx, G, hubs)
        xs.append(x)
        ys.append(y)
        del G
    return torch.cat(xs), torch.cat(ys)


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--graphs", type=int, default=64)
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--steps", type=int, default=600)
    args = ap.parse_args()
    with Context(0, stream=torch.cuda.current_stream()) as ctx:
        X, Y = training_set(ctx, args.graphs, args.scale)
        params, losses = train(ctx, X, Y, steps=args.steps)
    np.save(args.out, params)
    print(f"{len(Y)} samples ({int((Y == 1).sum().item())} in a largest SCC); loss {losses[0][1]:.4f} -> {losses[-1][1]:.4f} "
          f"(floor {label_entropy(Y):.4f}); wrote {args.out}")


if __name__ == "__main__":
    main()
