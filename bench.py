"""SCC throughput benchmark (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kspn|reference]
                    [--workload rmat24|rmat26|rgg24|gnm16] [--pipeline fast|reference]

A step is one complete decomposition of the workload graph (strongly
connected components, canonical min-id labels).  Default workload: the
learned-pivot configuration, directed R-MAT scale 26 (2^26 vertices, 1.06 B
edges after dedup), edge factor 16, a,b,c,d = .57,.19,.19,.05, seeded id
permutation, self-loops and duplicates removed, u32 ids, u64 offsets --
generated on the device by the library's own seeded generator.

value   = edges of the graph / device time per step (CUDA events on the
          library's stream; graph and transpose resident in HBM, > L2).
e2e     = the same metric through the host C-ABI call kspn_scc with pinned
          HOST buffers: forward CSR copied in, transpose built on the device,
          labels copied out, every step.
roofline: the dominant kernel's algorithmic bytes / its event-timed
          duration, against MEASURED_PEAKS.json's HBM copy bandwidth.
learned_vs_plain: the workload decomposed from the plain max(in * out)
          pivot and from the shipped pivot model's, same output asserted;
          and the same on the workload with decoy hubs.
cpu_baseline: the reference's own kaspan::scc (oracle/_ref, compiled from its
          sources; 1 core, MPI absent), one call on a bounded sample: the
          workload itself where one call takes seconds, R-MAT scale 24
          (a quarter of the scale-26 workload) for R-MAT scale 26.
other_rmat = the other R-MAT configuration (scale 24 beside the scale-26
          workload, and the reverse): device time, roofline, learned vs
          plain pivot, end to end.

--impl reference: the reference's kaspan::scc on the host cores on the
identical graph (the oracle's C generator draws the same edges as the
device generator), one call per step; where one call takes tens of seconds
(R-MAT scale 26: 1.06 B edges and a 16 GiB hash set at one rank) the arm
times as many calls as fit in --reference-seconds (at least one) and
states the count.

Multi-GPU (torchrun): every rank decomposes its own seeded instance (seed +
rank); value = edges over all ranks / max-over-ranks time ("weak" scaling,
no data-path collective).  A `sharded` section adds ONE graph
(--sharded-workload, R-MAT scale 22 by default) decomposed over all ranks
with a frontier exchange per level (kaspan_b200/shard.py).  --impl
reference runs on rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SCC edges/sec on 1 B200 (learned vs plain pivots, exact) + % HBM roofline"
UNIT = "edges/s"

WORKLOADS = {
    # name: (kind, params, description)
    "rmat24": ("rmat", dict(scale=24, ef=16, seed=2), "R-MAT scale 24, edge factor 16, a,b,c,d=.57,.19,.19,.05, permuted ids"),
    "rmat26": ("rmat", dict(scale=26, ef=16, seed=4), "R-MAT scale 26, edge factor 16, a,b,c,d=.57,.19,.19,.05, permuted ids"),
    "gnm16": ("gnm", dict(n=1 << 16, draws=1 << 19, seed=1), "directed G(n,m) n=2^16, 2^19 draws"),
    "rmat22": ("rmat", dict(scale=22, ef=16, seed=2), "R-MAT scale 22, edge factor 16, a,b,c,d=.57,.19,.19,.05, permuted ids"),
    "rmat20": ("rmat", dict(scale=20, ef=16, seed=2), "R-MAT scale 20, edge factor 16, a,b,c,d=.57,.19,.19,.05, permuted ids"),
    "rgg24": ("rgg", dict(n=1 << 24, seed=3), "2D random geometric graph n=2^24, mean undirected degree 8, each pair u->v / v->u / both / neither with p=.25"),
    "rgg22": ("rgg", dict(n=1 << 22, seed=3), "2D random geometric graph n=2^22, mean undirected degree 8, each pair u->v / v->u / both / neither with p=.25"),
    "rgg20": ("rgg", dict(n=1 << 20, seed=3), "2D random geometric graph n=2^20, mean undirected degree 8, each pair u->v / v->u / both / neither with p=.25"),
}
# kspn pipelines by name: the FAST pipeline, kaspan::scc's phase order
# ("reference") and the reference's six variants (variant/*.hpp)
PIPELINES = {"fast": 0, "reference": 1, "hpc_like": 2, "hpc_trim_ex": 3, "ispan_like": 4, "trim_ex": 5, "trim_ex_light_residual": 6, "trim_ex_residual": 7}

# The other R-MAT configuration reported beside an R-MAT workload, and the
# bounded sample the kspn arm's cpu_baseline decomposes on the host.
OTHER_RMAT = {"rmat26": "rmat24", "rmat24": "rmat26"}
CPU_SAMPLE = {"rmat26": "rmat24"}


def measured_peak_gbs():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = [r.split(", ") for r in (self.out or "").strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_graph(ctx, name, rank_seed=0):
    import kaspan_b200.graphs as KG

    kind, p, _ = WORKLOADS[name]
    if kind == "rmat":
        return KG.rmat(ctx, p["scale"], p["ef"], p["seed"] + rank_seed)
    if kind == "rgg":
        return KG.rgg(ctx, p["n"], p["seed"] + rank_seed)
    return KG.gnm(ctx, p["n"], p["draws"], p["seed"] + rank_seed)


def host_graph(name):
    """The workload graph on the host, drawn by the oracle's C generators
    (the same edges as the device generators, tested bit-identical)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    kind, p, _ = WORKLOADS[name]
    if kind == "rmat":
        return O.rmat(p["scale"], p["ef"], p["seed"])
    if kind == "rgg":
        return O.rgg(p["n"], p["seed"])
    return O.gnm(p["n"], p["draws"], p["seed"])


def reference_calls(G, steps, warmup=0, budget_s=None):
    """The reference's kaspan::scc (oracle/_ref) on host graph G: edges/s of
    each timed call, or None when oracle/_ref is absent.  With budget_s the
    warm-up calls are skipped and the timed calls stop once their total
    passes budget_s (at least one call)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if O.ref_lib() is None:
        return None
    if budget_s is None:
        for _ in range(warmup):
            O.ref_scc(G)
    rates, spent = [], 0.0
    for _ in range(steps):
        secs = O.ref_scc(G)[1]
        rates.append(G.m / secs)
        spent += secs
        if budget_s is not None and spent >= budget_s:
            break
    return rates


def run_reference(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    if O.ref_lib() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkspn_ref.so was not built (reference sources absent at build time)"}))
        return 0
    t0 = time.perf_counter()
    G = host_graph(args.workload)
    gen_s = time.perf_counter() - t0
    budget = args.reference_seconds if G.m > (1 << 29) else None
    rates = reference_calls(G, args.steps, args.warmup, budget)
    v = statistics.mean(rates)
    sample = (f"the workload graph itself ({WORKLOADS[args.workload][2]}: n={G.n}, m={G.m}), one kaspan::scc call per step "
              "(reference code compiled from its sources, 1 rank, 1 core)")
    if budget is not None:
        sample += (f"; {len(rates)} timed call(s) of the {args.steps} asked, no warm-up calls: one call takes "
                   f"{1e3 * G.m / v / 1e3:.0f} s, so the arm stops after {budget:.0f} s of calls")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": len(rates),
        "warmup": 0 if budget is not None else args.warmup, "steps_asked": args.steps,
        "ms_per_step": 1e3 * G.m / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded generators standing in for KaGen R-MAT / G(n,m) / RGG)",
        "config": {"workload": WORKLOADS[args.workload][2], "n": G.n, "m": G.m, "same_graph": True, "sample": sample,
                   "host_generation_s": round(gen_s, 1), "mpi": "absent on this host: single rank"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_batched(ctx, stream, args, K, world=1, rank=0):
    """The batch mix (4096 G(n, m) graphs, n log-uniform in [2^8, 2^18],
    mean out-degree U[0.8, 6], seed 5) through kspn_scc_batched: device time
    per call, whole-pipeline roofline, and the reference kaspan::scc on the
    host cores over a bounded sample of the same graphs.  On N GPUs each
    rank decomposes its shard (greedy edge-balanced bin packing of the
    graphs, no communication); the time is the max over ranks."""
    import numpy as np
    import torch
    import torch.distributed as dist

    import kaspan_b200.graphs as KG

    shard = None
    if world > 1:
        n_all, d_all = K.batch_shape(args.batch_graphs, 5, 8, args.batch_max_log2)
        shard = KG.batch_partition(n_all.astype(np.float64) + d_all.astype(np.float64), world)[rank]
    B = KG.batch(ctx, args.batch_graphs, 5, 8, args.batch_max_log2, graphs=shard)
    out = torch.empty(B.n, dtype=torch.int32, device="cuda")
    steps = max(3, min(args.steps, 10))

    def sync():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(o):
        for _ in range(2):
            ctx.scc_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out, o)
        sync()
        l0 = ctx.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = None
        for _ in range(steps):
            st = ctx.scc_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out, o)
        e1.record(stream)
        sync()
        t = e0.elapsed_time(e1) / steps
        if world > 1:
            x = torch.tensor([t], device="cuda")
            dist.all_reduce(x, op=dist.ReduceOp.MAX)
            t = float(x.item())
        return t, (ctx.launches - l0) / steps, st

    m_all = float(B.m)
    n_all_v = float(B.n)
    if world > 1:
        x = torch.tensor([m_all, n_all_v], device="cuda", dtype=torch.float64)
        dist.all_reduce(x)
        m_all, n_all_v = float(x[0].item()), float(x[1].item())
    ms, launches, st = timed(None)
    # every rank tunes its own shard (the same steps on every rank)
    best, rep = ctx.autotune_batched(B.count, B.n, B.vtx_off, B.fwh, B.fwc, B.bwh, B.bwc, out, reps=2)
    ms_t, _, st_t = timed(best)
    # route 1: the mix as one graph (a super-source linked to every graph's
    # pivot, the single-graph pipeline), same ids checked
    ref_ids = out.clone()
    uo = K.BatchOptions()
    K.lib().kspn_batch_options_default(__import__("ctypes").byref(uo))
    uo.route = 1
    ms_u, launches_u, st_u = timed(uo)
    union_same = bool(torch.equal(out, ref_ids))
    assert union_same, "the union route must give the per-graph route's ids"
    peak, peak_kind = measured_peak_gbs()
    b_min = 2 * (8 * (n_all_v + 1) + 4 * m_all) + 4 * n_all_v
    res = {
        "workload": f"{args.batch_graphs} directed G(n,m) graphs, n = round(2^U[8,{args.batch_max_log2}]), m = round(n * U[0.8, 6]) draws, seed 5, self-loops and duplicates removed, local u32 ids, one concatenated CSR + CSC",
        "graphs": args.batch_graphs, "n": int(n_all_v), "m": int(m_all), "steps": steps, "n_gpus": world,
        "scaling": "strong" if world > 1 else None, "sharding": "greedy edge-balanced bin packing of whole graphs, no communication" if world > 1 else None,
        "value": m_all / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
        "launches_per_step": launches, "captured": "one CUDA graph per call (plan + solve kernels), replayed",
        "stats": st.as_dict(),
        "pipeline_min_bytes": b_min, "pipeline_frac": (b_min / (ms * 1e-3)) / 1e9 / peak, "peak": peak, "peak_source": peak_kind,
        "union_route": {"value": m_all / (ms_u * 1e-3), "ms_per_step": ms_u, "launches_per_step": launches_u, "identical_output": union_same,
                        "taken": st_u.graphs_small == 0 and st_u.graphs_large == B.count,
                        "how": "kspn_batch_options.route = 1: the mix as ONE graph with global ids plus a super-source whose rows list every graph's pivot; the single-graph pipeline (trim, one FW-BW deciding a component in every graph at once, trim fixpoint, residual); host-driven, not one captured graph"},
        "tuned": {"value": m_all / (ms_t * 1e-3), "ms_per_step": ms_t, "candidates": rep.candidates, "tuner_default_ms": rep.default_ms, "tuner_best_ms": rep.best_ms,
                  "best": {"cluster_size": best.cluster_size, "cluster_min": best.cluster_min, "rem_tarjan": best.rem_tarjan, "max_rounds": best.max_rounds}},
    }
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        # the reference's kaspan::scc on the host cores, one call per graph,
        # over the first 256 graphs of the mix (a bounded sample)
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        if O.ref_lib() is not None:
            secs, edges = 0.0, 0
            for g in range(min(256, B.count)):
                n, fwh, fwc, bwh, bwc = B.graph(g)
                _, t = O.ref_scc(O.Graph(n, fwh, np.ascontiguousarray(fwc) if fwc.size else np.zeros(1, np.uint32), bwh,
                                         np.ascontiguousarray(bwc) if bwc.size else np.zeros(1, np.uint32)))
                secs += t
                edges += int(fwh[-1])
            res["cpu_baseline"] = {"value": edges / secs, "unit": UNIT, "cores": 1, "kind": "reference",
                                   "sample": f"the first 256 graphs of the mix ({edges} edges), one kaspan::scc call each (reference code, 1 rank, 1 core)"}
    del B, out
    torch.cuda.empty_cache()
    return res


def timed_steps(ctx, stream, G, opt, steps, out):
    """`steps` decompositions of device graph G back to back between two
    CUDA events on the library's stream: (ms per step, Stats of each step)."""
    import torch

    import kaspan_b200 as K

    stats = [K.Stats() for _ in range(steps)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(steps):
        ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, opt, stats[i])
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, stats


def resident_roofline(step_stats, peak):
    """The resident launch k_fwbw over the timed steps: algorithmic bytes per
    launch (its device counters) / its CUDA-event duration."""
    res = [d["resident"] for d in step_stats if d["resident"]["ms"] > 0]
    if not res:
        return None
    kms = sum(r["ms"] for r in res) / len(res)
    kbytes = sum(r["bytes"] for r in res) / len(res)
    achieved = (kbytes / (kms * 1e-3)) / 1e9
    return {"kernel": "k_fwbw", "achieved": achieved, "frac": achieved / peak, "bytes_per_step": kbytes, "ms_per_step": kms}


def host_e2e(ctx, stream, G, opt, steps, warmup):
    """kspn_scc with pinned host buffers (forward CSR in, transpose built on
    the device, labels out) every step: (ms per step, labels of the last)."""
    import numpy as np
    import torch

    fwh_h = G.fwh.cpu().pin_memory()
    fwc_h = G.fwc.cpu().pin_memory()
    out_h = torch.empty(G.n, dtype=torch.int32).pin_memory()
    for _ in range(warmup):
        ctx.scc_host_ptr(G.n, G.m, fwh_h, fwc_h, None, None, out_h, opt)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(steps):
        ctx.scc_host_ptr(G.n, G.m, fwh_h, fwc_h, None, None, out_h, opt)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max(e0.elapsed_time(e1), (time.perf_counter() - t0) * 1e3) / steps
    return ms, out_h.numpy().view(np.uint32).copy()


def learned_vs_plain(ctx, stream, graph, pipeline, steps):
    """The same graph decomposed from the plain pivot (largest in * out) and
    from the learned one; identical output asserted."""
    import numpy as np
    import torch

    import kaspan_b200 as K

    o = torch.empty(graph.n, dtype=torch.int32, device="cuda")
    res = {"n": graph.n, "m": graph.m}
    ids = {}
    for name, opt in (("plain", K.default_options(pipeline=pipeline, validate=0)),
                      ("learned", K.default_options(pipeline=pipeline, validate=0, learned_pivot=1))):
        timed_steps(ctx, stream, graph, opt, 1, o)
        ms, st = timed_steps(ctx, stream, graph, opt, steps, o)
        d = st[-1].as_dict()
        ids[name] = o.cpu().numpy().view(np.uint32).copy()
        res[name] = {"ms_per_step": ms, "edges_scanned": d["edges_scanned"], "pivot": d["pivot"], "fwbw_decided": d["decided"]["fwbw"]}
    assert np.array_equal(ids["plain"], ids["learned"]), "learned and plain pivots must give the same partition"
    res["speedup"] = res["plain"]["ms_per_step"] / res["learned"]["ms_per_step"]
    res["identical_output"] = True
    return res


def seed_order(ctx, stream, graph, steps):
    """The label searches' seed order, rotated ids (the reference's) vs the
    pivot model's ranking, in kaspan::scc's phase order (trim_1_first,
    FW-BW, trim_1_normal, label searches until done); identical output
    asserted."""
    import numpy as np
    import torch

    import kaspan_b200 as K

    o = torch.empty(graph.n, dtype=torch.int32, device="cuda")
    res = {"pipeline": "scc (the reference's phase order)"}
    ids = {}
    for name, seeds in (("rotated", 0), ("learned", 1)):
        opt = K.default_options(pipeline=K.PIPELINE_REFERENCE, validate=0, learned_seeds=seeds)
        timed_steps(ctx, stream, graph, opt, 1, o)
        ms, st = timed_steps(ctx, stream, graph, opt, steps, o)
        d = st[-1].as_dict()
        ids[name] = o.cpu().numpy().view(np.uint32).copy()
        res[name] = {"ms_per_step": ms, "label_calls": d["label_calls"], "label_decided": d["decided"]["label"]}
    assert np.array_equal(ids["rotated"], ids["learned"]), "the seed order must not change the partition"
    res["speedup"] = res["rotated"]["ms_per_step"] / res["learned"]["ms_per_step"]
    res["identical_output"] = True
    return res


def run_other_rmat(ctx, stream, args, peak, K, name, cpu_sample):
    """The other R-MAT configuration (`name`: scale 24 beside the scale-26
    workload, or the reverse): device time per decomposition, k_fwbw's
    roofline, learned vs plain pivot and end to end through kspn_scc.  With
    cpu_sample, also one reference kaspan::scc call on this graph's host
    copy (the kspn arm's bounded cpu_baseline sample)."""
    import numpy as np
    import torch

    G = make_graph(ctx, name)
    out = torch.empty(G.n, dtype=torch.int32, device="cuda")
    opt = K.default_options(validate=0)
    steps = max(3, min(args.steps, 10))
    timed_steps(ctx, stream, G, opt, 3, out)
    ms, st = timed_steps(ctx, stream, G, opt, steps, out)
    dicts = [s.as_dict() for s in st]
    res = {"workload": WORKLOADS[name][2], "n": G.n, "m": G.m, "steps": steps, "value": G.m / (ms * 1e-3), "unit": UNIT,
           "ms_per_step": ms, "roofline": resident_roofline(dicts, peak),
           "pipeline_frac": (2 * (8 * (G.n + 1) + 4 * G.m) + 4 * G.n) / (ms * 1e-3) / 1e9 / peak}
    model = K.default_pivot_model()
    if model is not None:
        ctx.set_pivot_model(model)
        res["learned_vs_plain"] = learned_vs_plain(ctx, stream, G, K.PIPELINE_FAST, steps)
        ctx.set_pivot_model(None)
    e2e_ms, _ = host_e2e(ctx, stream, G, K.default_options(validate=0), 3, 1)
    res["e2e"] = {"value": G.m / (e2e_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_ms, "h2d_bytes_per_step": 8 * (G.n + 1) + 4 * G.m,
                  "d2h_bytes_per_step": 4 * G.n}
    cpu = None
    if cpu_sample:
        fwh, fwc, bwh, bwc = G.to_host()
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O

        HG = O.Graph(G.n, np.ascontiguousarray(fwh), np.ascontiguousarray(fwc), np.ascontiguousarray(bwh), np.ascontiguousarray(bwc))
        rates = reference_calls(HG, 1)
        if rates is not None:
            cpu = {"value": rates[0], "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": f"{WORKLOADS[name][2]} (n={G.n}, m={G.m}), the same generator at a quarter of the workload's scale: "
                             "one kaspan::scc call (reference code, 1 rank, 1 core); --impl reference times the workload itself"}
            # the reference's own sequential Tarjan on the same sample (its oracle)
            _, secs = O.ref_tarjan(HG)
            cpu["tarjan"] = {"value": G.m / secs, "unit": UNIT, "cores": 1, "kind": "reference", "what": "kaspan::tarjan (kaspan/scc/tarjan.hpp), one call"}
    del G, out
    torch.cuda.empty_cache()
    return res, cpu


def run_sharded(ctx, args, K, world, rank):
    """ONE graph over all ranks (kaspan_b200/shard.py: a contiguous vertex
    range per GPU, frontier exchange over NCCL every level): the graph of
    --sharded-workload (seed 0 on every rank), sharded; time per
    decomposition = max over ranks (the ranks meet at a collective every
    level).  Its ids are checked against the single-GPU decomposition of the
    same graph."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from kaspan_b200 import shard as SH

    G = make_graph(ctx, args.sharded_workload, rank_seed=0)
    want = torch.empty(G.n, dtype=torch.int32, device="cuda")
    ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, want, K.default_options(validate=0))
    fwh_h = G.fwh.cpu().numpy().view(np.uint64)
    bounds = SH.partition_bounds(G.n, fwh_h, world)
    lo, hi = bounds[rank], bounds[rank + 1]
    bwh_h = G.bwh.cpu().numpy().view(np.uint64)
    fb, fe, bb, be = int(fwh_h[lo]), int(fwh_h[hi]), int(bwh_h[lo]), int(bwh_h[hi])
    S = SH.Shard(G.n, rank, world, bounds, (G.fwh[lo: hi + 1] - fb).contiguous(), G.fwc[fb: max(fe, fb + 1)].contiguous(),
                 (G.bwh[lo: hi + 1] - bb).contiguous(), G.bwc[bb: max(be, bb + 1)].contiguous())
    want_local = want[lo:hi].cpu().numpy().view(np.uint32).copy()
    m = G.m
    del G, want
    torch.cuda.empty_cache()
    ex = SH.Exchange()
    times, st = [], None
    for i in range(3):
        dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = SH.ShardStats()
        ids = SH.scc_sharded(SH.CudaShardOps(ctx, S), ex, S, stats=st)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        t = torch.tensor([dt], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        times.append(float(t.item()))
    ok = bool(np.array_equal(ids.cpu().numpy().view(np.uint32), want_local))
    okt = torch.tensor([1 if ok else 0], device="cuda")
    dist.all_reduce(okt, op=dist.ReduceOp.MIN)
    ms = 1e3 * min(times[1:])
    return {"workload": WORKLOADS[args.sharded_workload][2], "n": S.n, "m": m, "ranks": world, "bounds": bounds,
            "value": m / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "scaling": "strong (one graph, all ranks)",
            "timing": "host wall clock around the whole sharded call, max over ranks (every level meets at a collective), best of 2 after 1 warm-up",
            "exchange": "NCCL all_to_all_single of frontier ids per level + all-reduces", "identical_to_single_gpu": bool(okt.item()),
            "rounds": st.rounds, "levels": st.levels, "ids_sent_rank0": st.exchanged,
            "decided": {"trim_first": st.decided_trim, "fwbw": st.decided_fwbw, "residual": st.decided_residual}}


def run_kspn(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    import kaspan_b200 as K

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    # one stream for the context's kernels, torch's work and the timing
    # events (the legacy default stream's handle is 0, which the context
    # would read as "make your own")
    stream = torch.cuda.Stream(device=local)
    torch.cuda.set_stream(stream)
    ctx = K.Context(local, stream=stream)
    G = make_graph(ctx, args.workload, rank_seed=rank)
    torch.cuda.synchronize()
    out = torch.empty(G.n, dtype=torch.int32, device="cuda")
    pipeline = PIPELINES[args.pipeline]
    opt = K.default_options(pipeline=pipeline, validate=0)
    prof_opt = K.default_options(pipeline=pipeline, validate=0, profile=1)
    trace_opt = K.default_options(pipeline=pipeline, validate=0, trace=1)
    peak, peak_kind = measured_peak_gbs()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-resident steps
    st = K.Stats()
    for _ in range(args.warmup):
        ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, opt, st)
    # one Stats per timed step, converted to dicts after the timed region
    stats_objs = [K.Stats() for _ in range(args.steps)]
    barrier()
    l0 = ctx.launches
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for i in range(args.steps):
            ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, opt, stats_objs[i])
        ev1.record(stream)
        barrier()
    step_stats = [s.as_dict() for s in stats_objs]
    launches = ctx.launches - l0
    ms = ev0.elapsed_time(ev1) / args.steps
    ids = out.cpu().numpy().view(np.uint32).copy()
    # phase stamps of the persistent searches (one extra step, not timed)
    ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, trace_opt, st)
    marks = st.as_dict()["search_marks"]
    search_phases = {}
    for (ph, t1), (_, t0) in zip(marks[1:], marks[:-1]):
        if t1 > t0:
            search_phases[ph] = search_phases.get(ph, 0.0) + (t1 - t0) * 1e-6

    # per-kernel-class device time: the same decomposition with the library's
    # event brackets on (levels driven from the host so every expansion
    # kernel launch is bracketed on the library's stream)
    agg = {k: [0.0, 0, 0] for k in K.KERNEL_CLASSES}
    prof_steps = args.profile_steps if args.profile_steps is not None else max(1, min(args.steps, 3))
    trace = []
    for _ in range(prof_steps):
        ctx.scc_device(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, prof_opt, st)
        trace = st.as_dict()["trace"]
        for k, v in st.as_dict()["kernels"].items():
            agg[k][0] += v["ms"]
            agg[k][1] += v["bytes"]
            agg[k][2] += v["calls"]
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        mt = torch.tensor([float(G.m)], device="cuda", dtype=torch.float64)
        dist.all_reduce(mt)
        m_total = float(mt.item())
    else:
        m_total = float(G.m)
    value = m_total / (ms * 1e-3)

    # ---- learned vs plain pivot (same output): the workload, and the
    # workload with decoy hubs (vertices whose in * out beats every real one
    # while their out-edges all end at dead ends)
    lvp = None
    model = K.default_pivot_model()
    if model is not None and args.workload.startswith("rmat") and world == 1:
        from kaspan_b200.pivot_train import decoy_rmat

        ctx.set_pivot_model(model)
        lvp = {"model": "kaspan_b200/pivot_model.npy (8-32-32-1, trained on the GPU: python -m kaspan_b200.pivot_train)"}
        lvp["workload"] = learned_vs_plain(ctx, stream, G, pipeline, max(3, min(args.steps, 10)))
        lvp["seed_order"] = seed_order(ctx, stream, G, 3)
        p_ = WORKLOADS[args.workload][1]
        Gd, _hubs = decoy_rmat(ctx, p_["scale"], p_["seed"] + 100, 0.57, decoys=8)
        lvp["workload_with_decoys"] = learned_vs_plain(ctx, stream, Gd, pipeline, max(3, min(args.steps, 10)))
        del Gd
        ctx.set_pivot_model(None)
        torch.cuda.empty_cache()

    # ---- autotuner on the workload (FAST pipeline switch points, trim-2,
    # learned pivot): what it picks and what it gains over the defaults
    autotune = None
    if world == 1 and not args.no_batched:
        best, rep = ctx.autotune(G.n, G.m, G.fwh, G.fwc, G.bwh, G.bwc, out, K.default_options(pipeline=pipeline, validate=0), reps=3)
        autotune = {"candidates": rep.candidates, "default_ms": rep.default_ms, "best_ms": rep.best_ms,
                    "best": {"bu_enter_div": best.bu_enter_div, "bu_leave_div": best.bu_leave_div, "trim2": best.trim2, "learned_pivot": best.learned_pivot}}

    # ---- batched path: the 4096-graph uneven G(n, m) mix in one captured
    # launch sequence, with the defaults and with the autotuned settings
    batched = None
    if not args.no_batched:
        batched = run_batched(ctx, stream, args, K, world, rank)

    # correctness spot check of the last step (canonical ids are min members)
    assert (ids <= np.arange(G.n, dtype=np.uint32)).all(), "ids must name a member no larger than the vertex"

    # ---- end to end through the host C ABI (pinned buffers, bw built on device)
    barrier()
    e2e_ms, e2e_ids = host_e2e(ctx, stream, G, K.default_options(pipeline=opt.pipeline, validate=0), max(1, min(args.steps, 5)), max(1, min(args.warmup, 2)))
    if world > 1:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    assert np.array_equal(e2e_ids, ids), "host path and device path disagree"
    h2d = 8 * (G.n + 1) + 4 * G.m
    d2h = 4 * G.n

    # ---- roofline of the dominant kernel: the resident launch (k_fwbw:
    # FW-BW, trim fixpoint and every id in one persistent kernel), timed by
    # the library's CUDA events around that launch on its stream, with the
    # algorithmic bytes its device counters give (model in include/kspn.h)
    roof = resident_roofline(step_stats, peak)
    if roof is None:  # the call did not take the resident path (profiled or oversized)
        dom = max(agg, key=lambda k: agg[k][0])
        kms, kbytes, _ = (x / max(prof_steps, 1) for x in agg[dom])
        a_ = (kbytes / (kms * 1e-3)) / 1e9 if kms > 0 else 0.0
        roof = {"kernel": dom, "achieved": a_, "frac": a_ / peak, "bytes_per_step": kbytes, "ms_per_step": kms}
    traffic, traffic_note = None, None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        try:
            tj = json.load(open(tp))
            traffic = tj.get(f"{args.workload}:{roof['kernel']}")
            traffic_note = tj.get(f"{args.workload}:{roof['kernel']}:note")
        except Exception:
            traffic = None
    last = step_stats[-1]
    b_min = 2 * (8 * (G.n + 1) + 4 * G.m) + 4 * G.n

    other, other_cpu = None, None
    oname = OTHER_RMAT.get(args.workload)
    if rank == 0 and world == 1 and oname and not args.no_other_rmat:
        other, other_cpu = run_other_rmat(ctx, stream, args, peak, K, oname, not args.no_cpu_baseline and CPU_SAMPLE.get(args.workload) == oname)
    sharded = None
    if world > 1:
        # an extra section: a failure here must not cost the main line
        try:
            sharded = run_sharded(ctx, args, K, world, rank)
        except Exception as exc:  # noqa: BLE001
            sharded = {"error": f"{type(exc).__name__}: {exc}"[:300]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded device generator standing in for KaGen; graph > L2 so no flush between steps)",
            "config": {"workload": WORKLOADS[args.workload][2], "n": G.n, "m": G.m, "pipeline": args.pipeline,
                       "parallelism": f"{world} independent instance(s), one per GPU", "l2": "inputs larger than L2 (126 MB)"},
            "e2e": {"value": m_total / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": roof["kernel"], "achieved": roof["achieved"], "peak": peak, "unit": "GB/s", "frac": roof["frac"],
                         "traffic": traffic, "traffic_source": traffic_note, "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_kind})",
                         "bytes_per_step": roof["bytes_per_step"], "ms_per_step": roof["ms_per_step"], "calls_per_step": 1.0,
                         "timing": f"CUDA events around the {roof['kernel']} launch on the library stream, every timed step",
                         "model": last["resident"],
                         "pipeline_min_bytes": b_min, "pipeline_frac": (b_min / (ms * 1e-3)) / 1e9 / peak,
                         "pipeline_frac_note": "B_min = CSR + CSC read once + ids written (the survey's end-to-end bound); the pipeline reads far less "
                                               "(it scans a few percent of the edges), so a fraction above 1 is not bandwidth above the peak"},
            "clocks": clk.summary(),
            "learned_vs_plain": lvp,
            "other_rmat": other,
            "sharded": sharded,
            "autotune": autotune,
            "batched": batched,
            "phases": {"decided": last["decided"], "ms": {k: round(v, 4) for k, v in last["ms"].items()}, "levels_fw": last["levels_fw"],
                       "levels_bw": last["levels_bw"], "bottom_up": last["levels_bottom_up"], "label_calls": last["label_calls"],
                       "edges_scanned": last["edges_scanned"], "trace": trace,
                       "search_phase_ms": {{4: "expand", 5: "sweep", 7: "materialize", 8: "init", 9: "end", 10: "finalize", 11: "trim_seed", 12: "trim_level", 13: "worklist", 14: "fix_up", 15: "trim_heavy", 16: "trim_worklist"}.get(k, k): round(v, 4) for k, v in search_phases.items()},
                       "kernels": {k: {"ms": round(a[0] / max(prof_steps, 1), 4), "GB/s": round(a[1] / (a[0] * 1e-3) / 1e9, 1) if a[0] else 0}
                                   for k, a in agg.items()}},
        }
        if other_cpu is not None:
            line["cpu_baseline"] = other_cpu
        elif not args.no_cpu_baseline and world == 1 and args.workload not in CPU_SAMPLE:
            # the reference's kaspan::scc on this very graph (its host copy), one call
            fwh, fwc, bwh, bwc = G.to_host()
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O

            rates = reference_calls(O.Graph(G.n, np.ascontiguousarray(fwh), np.ascontiguousarray(fwc), np.ascontiguousarray(bwh), np.ascontiguousarray(bwc)), 1)
            if rates is not None:
                line["cpu_baseline"] = {"value": rates[0], "unit": UNIT, "cores": 1, "kind": "reference",
                                        "sample": f"the workload graph itself (n={G.n}, m={G.m}), one kaspan::scc call (reference code, 1 rank, 1 core)"}
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kspn", choices=["kspn", "reference"])
    ap.add_argument("--workload", default="rmat26", choices=sorted(WORKLOADS))
    ap.add_argument("--pipeline", default="fast", choices=sorted(PIPELINES), help="fast (default), or the phase order of a reference entry point")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-path and autotuner sections")
    ap.add_argument("--no-other-rmat", action="store_true", help="skip the other R-MAT configuration's section")
    ap.add_argument("--sharded-workload", default="rmat22", choices=sorted(WORKLOADS),
                    help="graph of the N > 1 sharded section (one graph over all ranks; default R-MAT scale 22)")
    ap.add_argument("--reference-seconds", type=float, default=100.0,
                    help="--impl reference on graphs above 2^29 edges: stop timing calls after this many seconds (at least one call)")
    ap.add_argument("--batch-graphs", type=int, default=4096, help="graphs of the batch mix (default 4096)")
    ap.add_argument("--batch-max-log2", type=int, default=18, help="largest graph of the batch mix: 2^this vertices (default 18)")
    ap.add_argument("--profile-steps", type=int, default=None, help="steps run with per-kernel event timing (default min(steps, 3))")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "kspn":
        args.warmup = 3
    return run_reference(args) if args.impl == "reference" else run_kspn(args)


if __name__ == "__main__":
    sys.exit(main())
