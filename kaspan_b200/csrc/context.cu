// C ABI of libkspn: contexts, workspace, the whole-path entry points and the
// phase-level entry points (include/kspn.h).  No exception crosses the ABI:
// every entry point catches, records the detail on the context and returns
// a KSPN_ERR_* status.
//
// Pipelines (both end in the canonical min-id relabel):
//  REFERENCE  the phase order of kaspan::scc (kaspan/scc/scc.hpp:21-87):
//             trim_1_first -> FW-BW(pivot) -> trim_1_normal -> label
//             searches with rotation 1, 2, 3, ... until every vertex is
//             decided.
//  FAST       trim_1_first -> FW-BW from its pivot -> rounds of {trim-1
//             fixpoint, trim-2, label search} until every vertex is decided.
//             Same partition (every phase only decides whole SCCs).
#include "kspn_internal.cuh"

#include <functional>
#include <vector>

#include "prim.cuh"

#include <algorithm>
#include <cstring>
#include <new>

namespace kspn {

namespace {

constexpr size_t ALIGN = 256;

size_t
align_up(size_t x)
{
  return (x + ALIGN - 1) & ~(ALIGN - 1);
}

struct carver
{
  char*  base;
  size_t off = 0;
  template<typename T>
  T* take(size_t count)
  {
    off    = align_up(off);
    T* p   = base ? reinterpret_cast<T*>(base + off) : nullptr;
    off += count * sizeof(T);
    return p;
  }
};

// Lays out (or, with base == nullptr, measures) the workspace.
size_t
layout(workspace& ws, char* base, uint32_t n, uint64_t m)
{
  carver         c{ base };
  size_t const   words = (static_cast<size_t>(n) + 63) / 64 * 2 + 2; // u32 words, u64-rounded
  size_t const   nn    = static_cast<size_t>(n) + 2;
  ws.ctr               = c.take<uint32_t>(64);
  ws.ctr64             = reinterpret_cast<uint64_t*>(ws.ctr ? ws.ctr + 32 : nullptr); // same block: one D2H copy
  ws.q0                = c.take<uint32_t>(nn);
  ws.q1                = c.take<uint32_t>(nn);
  ws.vis_a             = c.take<uint32_t>(words);
  ws.vis_b             = c.take<uint32_t>(words);
  ws.mark              = c.take<uint32_t>(words);
  ws.fresh             = c.take<uint32_t>(words);
  ws.fresh_bw          = c.take<uint32_t>(words);
  ws.cand_bw           = c.take<uint32_t>(words);
  ws.und               = c.take<uint32_t>(words);
  ws.label             = c.take<uint32_t>(nn);
  ws.indeg             = c.take<uint32_t>(nn);
  ws.outdeg            = c.take<uint32_t>(nn);
  ws.prefix            = c.take<uint64_t>(nn);
  ws.prefix2           = c.take<uint64_t>(nn);
  ws.blocks            = c.take<uint64_t>(std::max<size_t>(scan_partial_entries(nn), 4096));
  ws.pivot             = c.take<uint64_t>(8192);
  ws.tile_start        = c.take<uint32_t>(m / 2048 + 4);
  ws.tile_start2       = c.take<uint32_t>(m / 2048 + 4);
  ws.q2                = c.take<uint32_t>(nn);
  ws.q3                = c.take<uint32_t>(nn);
  ws.prefix3           = c.take<uint64_t>(nn);
  ws.prefix4           = c.take<uint64_t>(nn);
  ws.tile_start3       = c.take<uint32_t>(m / 2048 + 4);
  ws.tile_start4       = c.take<uint32_t>(m / 2048 + 4);
  ws.tile_zero         = c.take<uint32_t>(m / 2048 + 4);
  ws.seed_q            = c.take<uint32_t>(4);
  ws.seed_prefix       = c.take<uint64_t>(4);
  ws.gbar              = c.take<char>(4096);
  ws.heavy_cap         = heavy_capacity(n, m);
  ws.aw_entries        = 4 * nn + 2 * AW_STALE + 4 * (m / HEAVY_SLICE) + 128; // see run_async: half for duplicates, the passes around the switch, one winning item per vertex and direction, the heavy-row slices
  ws.aw                = c.take<unsigned long long>(ws.aw_entries);
  ws.rstate            = c.take<char>(4096);
  ws.heavy             = c.take<uint32_t>(4 * ws.heavy_cap);
  ws.cutmap            = c.take<uint32_t>(2 * words);
  return align_up(c.off);
}

} // namespace

void
ensure_workspace(kspn_context* ctx, uint32_t n, uint64_t m)
{
  auto& ws = ctx->ws;
  if (ws.base && n <= ws.n_cap && m <= ws.m_cap) return;
  uint32_t const ncap = std::max(n, ws.n_cap);
  uint64_t const mcap = std::max(m, ws.m_cap);
  if (ws.base) {
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    release_graphs(ctx); // they name the old workspace
    cudaFree(ws.base);
    ws.base = nullptr;
  }
  size_t const bytes = layout(ws, nullptr, ncap, mcap);
  void*        p     = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    cudaGetLastError();
    ws.n_cap = ws.m_cap = 0;
    throw error{ KSPN_ERR_OOM, "workspace of " + std::to_string(bytes) + " bytes" };
  }
  ws.base  = p;
  ws.bytes = bytes;
  ws.n_cap = ncap;
  ws.m_cap = mcap;
  layout(ws, static_cast<char*>(p), ncap, mcap);
  KSPN_CUDA(cudaMemsetAsync(ws.ctr, 0, 64 * sizeof(uint32_t), ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.tile_zero, 0, (mcap / 2048 + 4) * sizeof(uint32_t), ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.gbar, 0, 4096, ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.aw, 0, ws.aw_entries * sizeof(unsigned long long), ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.cutmap, 0, 2 * ((static_cast<size_t>(ncap) + 63) / 64 * 2 + 2) * sizeof(uint32_t), ctx->stream));
}

void*
context_buffer(kspn_context* ctx, int slot, size_t bytes)
{
  auto& b = ctx->bufs[slot];
  if (b.p && b.bytes >= bytes) return b.p;
  if (b.p) {
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    release_graphs(ctx); // a cached graph may name the old buffer
    cudaFree(b.p);
    b = {};
  }
  if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
    cudaGetLastError();
    b = {};
    throw error{ KSPN_ERR_OOM, "device buffer of " + std::to_string(bytes) + " bytes" };
  }
  b.bytes = bytes;
  return b.p;
}

void
read_counters(kspn_context* ctx)
{
  KSPN_CUDA(cudaMemcpyAsync(ctx->h_ctr, ctx->ws.ctr, 64 * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
}

void
zero_counters(kspn_context* ctx)
{
  KSPN_CUDA(cudaMemsetAsync(ctx->ws.ctr, 0, CTR_COUNT * sizeof(uint32_t), ctx->stream));
}

int
fail(kspn_context* ctx, error const& e)
{
  if (ctx) ctx->last_error = e.what;
  return e.code;
}

namespace {

// Owned device copy of a host graph (and a device-built transpose).
struct graph_store
{
  void*  base  = nullptr;
  size_t bytes = 0;
  ~graph_store()
  {
    if (base) cudaFree(base);
  }
};

void
check_options(kspn_options const& o)
{
  if (o.pipeline < 0 || o.pipeline >= KSPN_PIPELINE_COUNT) throw error{ KSPN_ERR_INVALID_ARGUMENT, "unknown pipeline" };
}

kspn_options
options_or_default(kspn_options const* opt)
{
  kspn_options o;
  kspn_options_default(&o);
  if (opt) {
    if (opt->struct_size != sizeof(kspn_options)) throw error{ KSPN_ERR_INVALID_ARGUMENT, "kspn_options.struct_size mismatch (use kspn_options_default)" };
    o = *opt;
  }
  check_options(o);
  return o;
}

struct phase_clock
{
  kspn_context* ctx;
  kspn_stats*   st;
  int           next = 1;
  void          start() { KSPN_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream)); }
  // attributes the device time since the previous mark to `phase`
  void mark(int phase)
  {
    if (!st) return;
    KSPN_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
    KSPN_CUDA(cudaEventSynchronize(ctx->ev[1]));
    float ms = 0;
    KSPN_CUDA(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]));
    st->ms[phase] += ms;
    std::swap(ctx->ev[0], ctx->ev[1]);
  }
};

// The whole path on a resident graph; writes the canonical ids into scc_id.
void
run_pipeline(kspn_context* ctx, dgraph const& g, uint32_t* scc_id, kspn_options const& opt, kspn_stats* st)
{
  auto& ws = ctx->ws;
  ensure_workspace(ctx, g.n, g.m);
  if (st) {
    std::memset(st, 0, sizeof(*st));
    st->n     = g.n;
    st->m     = g.m;
    st->pivot = g.n;
  }
  uint64_t const launches0 = ctx->launches;
  KSPN_CUDA(cudaMemsetAsync(ws.ctr, 0, 64 * sizeof(uint32_t), ctx->stream));
  std::memset(ctx->h_ctr, 0, 64 * sizeof(uint32_t));
  ctx->td_edges = 0;
  ctx->prof     = (opt.profile && st) ? st : nullptr;
  struct prof_reset
  {
    kspn_context* c;
    ~prof_reset() { c->prof = nullptr; }
  } prof_guard{ ctx };
  cudaEvent_t t_begin = ctx->ev[KSPN_PHASES], t_end = ctx->ev[KSPN_PHASES + 1];
  KSPN_CUDA(cudaEventRecord(t_begin, ctx->stream));
  phase_clock clk{ ctx, st };
  clk.start();
  if (opt.validate) validate(ctx, g);
  if (g.n == 0) return;

  uint32_t* und         = ws.und;
  uint64_t  decided     = 0;
  bool      label_ran   = false;
  bool      und_checked = false; // und already counted empty on the device
  auto      add     = [&](int phase, uint32_t d) {
    decided += d;
    if (st) st->decided[phase] += d;
    clk.mark(phase);
  };
  uint32_t const round_cap = opt.max_rounds ? opt.max_rounds : g.n + 2;

  if (opt.pipeline == KSPN_PIPELINE_REFERENCE) {
    uint32_t const pivot = trim_1_first(ctx, g, und, scc_id, nullptr, nullptr, false);
    add(KSPN_PHASE_TRIM_FIRST, ctx->h_ctr[CTR_AUX]);
    if (decided < g.n) {
      if (st) st->pivot = pivot;
      add(KSPN_PHASE_FWBW, fw_bw(ctx, g, und, scc_id, pivot, opt, st, true));
    }
    if (decided < g.n) add(KSPN_PHASE_TRIM_NORMAL, trim_1_normal(ctx, g, und, scc_id));
    int rotation = 0;
    while (decided < g.n) {
      if (st && st->label_calls >= round_cap) throw error{ KSPN_ERR_TIMEOUT, "label-search call cap exceeded" };
      label_ran = true;
      add(KSPN_PHASE_LABEL, label_search(ctx, g, und, scc_id, ++rotation, opt, st));
    }
  } else if (opt.pipeline != KSPN_PIPELINE_FAST) {
    // the reference's variants (variant/*.hpp), phase order at one rank
    int        p        = opt.pipeline;
    int        rotation = 0;
    uint32_t   calls    = 0;
    auto const label_rounds = [&](bool trim_between) {
      while (decided < g.n) {
        if (++calls > round_cap) throw error{ KSPN_ERR_TIMEOUT, "label-search call cap exceeded" };
        label_ran = true;
        add(KSPN_PHASE_LABEL, label_search(ctx, g, und, scc_id, ++rotation, opt, st));
        if (trim_between && decided < g.n) add(KSPN_PHASE_TRIM, trim_fixpoint(ctx, g, und, scc_id, false, 0));
      }
    };
    auto const fwbw_from = [&](uint32_t pivot) {
      if (st) st->pivot = pivot;
      add(KSPN_PHASE_FWBW, fw_bw(ctx, g, und, scc_id, pivot, opt, st, true));
    };
    bool const exhaustive = p == KSPN_PIPELINE_HPC_TRIM_EX || p == KSPN_PIPELINE_TRIM_EX || p == KSPN_PIPELINE_TRIM_EX_LIGHT_RESIDUAL || p == KSPN_PIPELINE_TRIM_EX_RESIDUAL;
    uint32_t   pivot      = g.n;
    if (exhaustive) add(KSPN_PHASE_TRIM_FIRST, trim_exhaustive_first(ctx, g, und, scc_id, ws.outdeg, ws.indeg));
    else {
      pivot = trim_1_first(ctx, g, und, scc_id, nullptr, nullptr, false);
      add(KSPN_PHASE_TRIM_FIRST, ctx->h_ctr[CTR_AUX]);
    }
    switch (p) {
    case KSPN_PIPELINE_HPC_LIKE: // scc_hpc_like.hpp:33-66
      if (decided < g.n) fwbw_from(pivot);
      label_rounds(false);
      break;
    case KSPN_PIPELINE_HPC_TRIM_EX: // scc_hpc_trim_ex.hpp:33-73
      if (decided < g.n) fwbw_from(select_pivot_live(ctx, g, und));
      label_rounds(false);
      break;
    case KSPN_PIPELINE_ISPAN_LIKE: // scc_ispan_like.hpp:33-84
      if (decided < g.n) fwbw_from(pivot);
      if (decided < g.n) add(KSPN_PHASE_TRIM_NORMAL, trim_1_normal(ctx, g, und, scc_id));
      if (decided < g.n) add(KSPN_PHASE_TRIM_NORMAL, trim_1_normal(ctx, g, und, scc_id));
      if (decided < g.n) add(KSPN_PHASE_RESIDUAL, residual(ctx, g, und, scc_id, nullptr));
      label_rounds(false);
      break;
    case KSPN_PIPELINE_TRIM_EX: // scc_trim_ex.hpp:33-99
      if (decided < g.n) fwbw_from(select_pivot_live(ctx, g, und));
      if (decided < g.n) add(KSPN_PHASE_TRIM, trim_fixpoint(ctx, g, und, scc_id, false, 0));
      label_rounds(true);
      break;
    case KSPN_PIPELINE_TRIM_EX_LIGHT_RESIDUAL: // scc_trim_ex_light_residual.hpp:33-118 (threshold 0 at one rank)
      if (decided < g.n) add(KSPN_PHASE_TRIM, trim_fixpoint(ctx, g, und, scc_id, false, 0));
      if (decided < g.n) add(KSPN_PHASE_RESIDUAL, residual(ctx, g, und, scc_id, nullptr));
      label_rounds(false);
      break;
    default: // KSPN_PIPELINE_TRIM_EX_RESIDUAL, scc_trim_ex_residual.hpp:33-127 (threshold 0 at one rank)
      if (decided < g.n) add(KSPN_PHASE_RESIDUAL, residual(ctx, g, und, scc_id, nullptr));
      label_rounds(false);
      break;
    }
  } else {
    // trim_1_first's pivot (argmax in*out) lies in the giant component of
    // the graphs this targets; FW-BW runs before any further trimming, and
    // the trim fixpoint then only walks the (small) remainder
    uint32_t rounds  = 0;
    bool     trimmed = false; // this round's trim fixpoint already ran
    // A large remainder after the first FW-BW means its pivot missed the
    // giant component (e.g. a hub whose out-edges all end at dead ends):
    // FW-BW again from the largest live in * out (degrees are current after
    // a trim fixpoint), while each round still decides a share of it.
    auto const fwbw_again = [&]() {
      if (ctx->union_route) return; // a batch mix: one pivot decides one component of one graph
      uint64_t const big = std::max<uint64_t>(g.n / 16, 1u << 16);
      for (uint32_t again = 0; again < 3 && g.n - decided >= big; ++again) {
        uint64_t const left = g.n - decided;
        uint32_t const pv   = select_pivot_live(ctx, g, und);
        if (pv >= g.n) break;
        uint64_t const d0 = decided;
        if (!ctx->prof && resident_fits(g)) {
          // one resident launch: FW-BW and the trim fixpoint (its worklist
          // tail takes long peeling chains without a barrier per level)
          auto const r = fw_bw_trim(ctx, g, und, scc_id, pv, opt, st);
          add(KSPN_PHASE_FWBW, r.first);
          add(KSPN_PHASE_TRIM, r.second);
        } else {
          add(KSPN_PHASE_FWBW, fw_bw(ctx, g, und, scc_id, pv, opt, st, true));
          if (decided < g.n) add(KSPN_PHASE_TRIM, trim_fixpoint(ctx, g, und, scc_id, false, 0));
        }
        if ((decided - d0) * 64 < left) break;
      }
    };
    if (!ctx->prof && resident_fits(g)) {
      // trim_1_first, then FW-BW and the trim fixpoint in ONE persistent
      // launch that takes the pivot from device memory: one host sync
      trim_1_first_async(ctx, g, und);
      KSPN_CUDA(cudaEventRecord(ctx->ev[2], ctx->stream));
      // with the learned rule the launch first scores the plain pivot (no
      // extra launch when the model accepts it)
      fw_bw_trim_async(ctx, g, und, scc_id, opt, st, ctx->ev[4]);
      KSPN_CUDA(cudaMemcpyAsync(ctx->h_ctr, ws.ctr, 64 * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
      KSPN_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
      KSPN_CUDA(cudaEventSynchronize(ctx->ev[3]));
      resident_result r = fw_bw_trim_result(ctx, g, opt, st);
      if (r.resumed) {
        // the phase clock's end after the resume launch
        KSPN_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
        KSPN_CUDA(cudaEventSynchronize(ctx->ev[3]));
      }
      if (r.pivot_rejected) {
        // the model rejected the plain pivot: score every candidate, then
        // the resident launch from the model's choice (no second check)
        learned_pivot(ctx, g, ctx->pivot_model, false);
        kspn_options o2  = opt;
        o2.learned_pivot = 0;
        fw_bw_trim_async(ctx, g, und, scc_id, o2, st, ctx->ev[4]);
        KSPN_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
        KSPN_CUDA(cudaEventSynchronize(ctx->ev[3]));
        r = fw_bw_trim_result(ctx, g, opt, st);
        if (r.resumed) {
          KSPN_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
          KSPN_CUDA(cudaEventSynchronize(ctx->ev[3]));
        }
      }
      uint32_t const        tf = ctx->h_ctr[CTR_DECIDED];
      decided += static_cast<uint64_t>(tf) + r.fwbw_decided + r.trim_decided;
      if (st) {
        float a = 0, b = 0;
        KSPN_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[2]));
        KSPN_CUDA(cudaEventElapsedTime(&b, ctx->ev[2], ctx->ev[3]));
        float k = 0;
        KSPN_CUDA(cudaEventElapsedTime(&k, ctx->ev[2], ctx->ev[4]));
        st->resident_ms = k;
        st->ms[KSPN_PHASE_TRIM_FIRST] += a;
        st->ms[KSPN_PHASE_FWBW] += b * r.fwbw_share;
        st->ms[KSPN_PHASE_TRIM] += b * (1.0 - r.fwbw_share);
        st->decided[KSPN_PHASE_TRIM_FIRST] += tf;
        st->decided[KSPN_PHASE_FWBW] += r.fwbw_decided;
        st->decided[KSPN_PHASE_TRIM] += r.trim_decided;
        st->pivot = r.pivot;
      }
      std::swap(ctx->ev[0], ctx->ev[3]); // later phases are timed from here
      if (decided > g.n || r.und_left != g.n - decided) throw error{ KSPN_ERR_INTERNAL, "resident pipeline: undecided count does not match" };
      rounds      = 1;
      trimmed     = true;
      und_checked = decided == g.n; // the launch counted und: empty
      if (decided < g.n) fwbw_again();
      // what is left splits into small pieces on most graphs: Tarjan per
      // piece in shared memory; larger pieces go on to the rounds below
      if (decided < g.n) add(KSPN_PHASE_RESIDUAL, residual(ctx, g, und, scc_id, nullptr));
    } else {
      uint32_t pivot = trim_1_first(ctx, g, und, scc_id, nullptr, nullptr, false);
      add(KSPN_PHASE_TRIM_FIRST, ctx->h_ctr[CTR_AUX]);
      if (decided < g.n && opt.learned_pivot && ctx->pivot_model) {
        // the model's choice among trim_1_first's per-block candidates
        learned_pivot(ctx, g, ctx->pivot_model);
        KSPN_CUDA(cudaMemcpyAsync(&pivot, reinterpret_cast<uint32_t*>(ws.pivot + 4096) + PV_FINAL, sizeof(pivot), cudaMemcpyDeviceToHost, ctx->stream));
        KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
      }
      if (decided < g.n) {
        if (st) st->pivot = pivot;
        add(KSPN_PHASE_FWBW, fw_bw(ctx, g, und, scc_id, pivot, opt, st, true));
      }
      if (decided < g.n && g.n - decided >= std::max<uint64_t>(g.n / 16, 1u << 16)) {
        add(KSPN_PHASE_TRIM, trim_fixpoint(ctx, g, und, scc_id, false, 0));
        fwbw_again();
      }
    }
    int rotation = 0;
    while (decided < g.n) {
      if (!trimmed) {
        if (++rounds > round_cap) throw error{ KSPN_ERR_TIMEOUT, "pipeline round cap exceeded" };
        add(KSPN_PHASE_TRIM, trim_fixpoint(ctx, g, und, scc_id, false, 0));
      }
      trimmed = false;
      if (decided < g.n && opt.trim2) {
        uint32_t const d2 = trim_2(ctx, g, und, scc_id);
        add(KSPN_PHASE_TRIM2, d2);
        if (d2 && decided < g.n) add(KSPN_PHASE_TRIM, trim_fixpoint(ctx, g, und, scc_id, false, 0));
      }
      if (decided < g.n) {
        label_ran = true;
        add(KSPN_PHASE_LABEL, label_search(ctx, g, und, scc_id, ++rotation, opt, st));
      }
    }
    if (st) st->rounds = rounds;
  }
  if (decided != g.n || (!und_checked && count_undecided(ctx, g.n, und) != 0)) throw error{ KSPN_ERR_INTERNAL, "decided-vertex count does not match n" };
  if (st) st->edges_scanned = ctx->h_ctr64[0] + ctx->td_edges;
  // trim (id = itself), trim-2 (id = the smaller of the pair) and FW-BW
  // (id = smallest member) already name components canonically; label
  // searches name them after their root, so only then is a relabel needed
  if (und_checked) {
    // everything was decided by the resident launch, whose completion
    // event (now ev[0]) the host already waited for: no further sync
    t_end = ctx->ev[0];
  } else {
    if (label_ran) canonicalise(ctx, g.n, scc_id, ws.label, true);
    add(KSPN_PHASE_CANON, 0);
    KSPN_CUDA(cudaEventRecord(t_end, ctx->stream));
    KSPN_CUDA(cudaEventSynchronize(t_end));
  }
  if (st) {
    float ms = 0;
    KSPN_CUDA(cudaEventElapsedTime(&ms, t_begin, t_end));
    st->ms_total        = ms;
    st->kernel_launches = ctx->launches - launches0;
  }
}

// The batch mix as one graph (kspn_batch_options.route = 1, batch_union.cu):
// false when the super-source would not be the pipeline's pivot (the
// caller then takes the per-graph route).
bool
scc_batched_union(kspn_context* ctx, uint32_t count, uint64_t n, uint64_t const* vtx_off, uint64_t const* fh, uint32_t const* fc, uint64_t const* bh, uint32_t const* bc,
                  uint32_t* scc_id, kspn_batch_stats* st)
{
  if (count == 0 || n == 0) return true;
  if (n + 1 >= static_cast<uint64_t>(UNDECIDED)) return false; // the super-source needs an id below UNDECIDED
  uint64_t m = 0;
  KSPN_CUDA(cudaMemcpyAsync(&m, fh + n, sizeof(m), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  size_t const heads = align_up((n + 2) * sizeof(uint64_t)), rows = align_up(std::max<uint64_t>(m + count, 1) * sizeof(uint32_t));
  size_t const ids = align_up((n + 1) * sizeof(uint32_t)), piv = align_up(static_cast<size_t>(count) * sizeof(uint32_t));
  char* const  base = static_cast<char*>(context_buffer(ctx, BUF_UNION, 2 * heads + 2 * rows + ids + piv + 256));
  auto* const  ufh  = reinterpret_cast<uint64_t*>(base);
  auto* const  ubh  = reinterpret_cast<uint64_t*>(base + heads);
  auto* const  ufc  = reinterpret_cast<uint32_t*>(base + 2 * heads);
  auto* const  ubc  = reinterpret_cast<uint32_t*>(base + 2 * heads + rows);
  auto* const  uid  = reinterpret_cast<uint32_t*>(base + 2 * heads + 2 * rows);
  auto* const  pv   = reinterpret_cast<uint32_t*>(base + 2 * heads + 2 * rows + ids);
  auto* const  pn   = reinterpret_cast<uint32_t*>(base + 2 * heads + 2 * rows + ids + piv);
  auto* const  mx   = reinterpret_cast<unsigned long long*>(base + 2 * heads + 2 * rows + ids + piv + 128);
  unsigned long long maxprod = 0;
  uint32_t const     P       = union_build(ctx, count, n, m, vtx_off, fh, fc, bh, bc, ufh, ufc, ubh, ubc, pv, pn, mx, &maxprod);
  if (static_cast<unsigned long long>(P) * P <= maxprod) return false;
  dgraph const ug{ static_cast<uint32_t>(n + 1), m + P, ufh, ufc, ubh, ubc };
  kspn_options o{};
  kspn_options_default(&o);
  o.validate = 0;
  struct route_flag
  {
    kspn_context* c;
    ~route_flag() { c->union_route = false; }
  } flag{ ctx };
  ctx->union_route = true;
  kspn_stats ps;
  run_pipeline(ctx, ug, uid, o, st ? &ps : nullptr);
  union_rename(ctx, count, n, vtx_off, uid, scc_id);
  if (st) {
    // the single-graph pipeline's phases in the batch stats' slots:
    // trim_first, trim (+ trim-2), FW-BW, residual + label + relabel
    st->graphs_large = count;
    st->fwbw_rounds  = 1;
    st->phase_ms[0]  = ps.ms[KSPN_PHASE_TRIM_FIRST];
    st->phase_ms[1]  = ps.ms[KSPN_PHASE_TRIM] + ps.ms[KSPN_PHASE_TRIM2] + ps.ms[KSPN_PHASE_TRIM_NORMAL];
    st->phase_ms[3]  = ps.ms[KSPN_PHASE_FWBW];
    st->phase_ms[4]  = ps.ms[KSPN_PHASE_RESIDUAL] + ps.ms[KSPN_PHASE_LABEL] + ps.ms[KSPN_PHASE_CANON];
    st->label_calls  = ps.label_calls;
  }
  return true;
}

// Resolves the transpose: given, or built on the device into `store`.
dgraph
with_transpose(kspn_context* ctx, uint32_t n, uint64_t m, uint64_t const* fh, uint32_t const* fc, uint64_t const* bh, uint32_t const* bc, graph_store& store)
{
  dgraph g{ n, m, fh, fc, bh, bc };
  if ((bh == nullptr) != (bc == nullptr)) throw error{ KSPN_ERR_INVALID_ARGUMENT, "bw_head and bw_csr must both be given or both be NULL" };
  if (!bh) {
    size_t const bytes = align_up((static_cast<size_t>(n) + 1) * 8) + align_up(std::max<uint64_t>(m, 1) * 4);
    char*        base  = static_cast<char*>(context_buffer(ctx, BUF_TRANSPOSE, bytes));
    (void)store;
    auto* nbh = reinterpret_cast<uint64_t*>(base);
    auto* nbc = reinterpret_cast<uint32_t*>(base + align_up((static_cast<size_t>(n) + 1) * 8));
    transpose(ctx, n, m, fh, fc, nbh, nbc, nullptr);
    g.bh = nbh;
    g.bc = nbc;
  }
  return g;
}

int
guard(kspn_context* ctx, auto&& body)
{
  try {
    body();
    return KSPN_OK;
  } catch (error const& e) {
    return fail(ctx, e);
  } catch (std::bad_alloc const&) {
    return fail(ctx, error{ KSPN_ERR_OOM, "host allocation" });
  } catch (...) {
    return fail(ctx, error{ KSPN_ERR_INTERNAL, "unexpected exception" });
  }
}

void
require(bool ok, char const* what)
{
  if (!ok) throw error{ KSPN_ERR_INVALID_ARGUMENT, what };
}

void
bind_device(kspn_context* ctx)
{
  KSPN_CUDA(cudaSetDevice(ctx->device));
}

// The phase entry points take the reference's u64 bitset; clear the bits
// past n in its last word so device words past n stay zero.
void
clear_bitset_tail(kspn_context* ctx, uint64_t* bits, uint32_t n)
{
  if (n % 64) KSPN_CUDA(cudaMemsetAsync(bits + n / 64, 0, 8, ctx->stream)); // rewritten by the kernel for bits < n
}

} // namespace

} // namespace kspn

using namespace kspn;

namespace kspn {
namespace {

// ids differing from the first run's (autotuner check)
__global__ void
k_tune_diff(uint64_t n, uint32_t const* __restrict__ a, uint32_t const* __restrict__ b, uint32_t* diff)
{
  uint32_t d = 0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) d += a[i] != b[i];
  if (d) atomicAdd(diff, d);
}

// Coordinate descent over `axes` (each a list of candidate setters on a
// copy of the current best); run(T) times one candidate and returns its ms.
template<typename T, typename Run>
T
tune(T base, std::vector<std::vector<std::function<void(T&)>>> const& axes, Run&& run, kspn_tune_report* rep)
{
  T     cur    = base;
  float t_cur  = run(cur);
  float t_base = t_cur;
  uint32_t cand = 1;
  for (auto const& axis : axes)
    for (auto const& set : axis) {
      T c = cur;
      set(c);
      if (std::memcmp(&c, &cur, sizeof(T)) == 0) continue;
      float const t = run(c);
      ++cand;
      if (t < 0.98f * t_cur) {
        // confirm against the incumbent, timed again back to back (one
        // fast run of a candidate is often noise)
        float const t_inc = run(cur);
        float const t_c   = run(c);
        if (t_c < 0.98f * t_inc) cur = c, t_cur = t_c;
        else t_cur = std::min(t_cur, t_inc);
      }
    }
  if (rep) {
    std::memset(rep, 0, sizeof(*rep));
    rep->candidates = cand;
    rep->default_ms = t_base;
    rep->best_ms    = t_cur;
  }
  return cur;
}

// The first run's ids, kept in a context buffer; later runs compared with it.
struct tune_check
{
  kspn_context* ctx;
  uint64_t      n;
  uint32_t*     ref  = nullptr;
  bool          have = false;
  void          take(uint32_t const* ids)
  {
    if (!n) return;
    if (!have) {
      ref = static_cast<uint32_t*>(context_buffer(ctx, BUF_GEN, n * sizeof(uint32_t)));
      KSPN_CUDA(cudaMemcpyAsync(ref, ids, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, ctx->stream));
      have = true;
      return;
    }
    uint32_t* const diff = ctx->ws.ctr + CTR_ERR;
    KSPN_CUDA(cudaMemsetAsync(diff, 0, sizeof(uint32_t), ctx->stream));
    k_tune_diff<<<148 * 8, 256, 0, ctx->stream>>>(n, ref, ids, diff);
    KSPN_CHECK_LAUNCH();
    uint32_t h = 0;
    KSPN_CUDA(cudaMemcpyAsync(&h, diff, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h) throw error{ KSPN_ERR_INTERNAL, "autotune: a candidate gave different ids" };
  }
};

} // namespace

} // namespace kspn

using kspn::tune;
using kspn::tune_check;
using kspn::k_tune_diff;

extern "C" {

int
kspn_options_default(kspn_options* opt)
{
  if (!opt) return KSPN_ERR_INVALID_ARGUMENT;
  std::memset(opt, 0, sizeof(*opt));
  opt->struct_size  = sizeof(kspn_options);
  opt->pipeline     = KSPN_PIPELINE_FAST;
  opt->trim2        = 1;
  opt->validate     = 1;
  opt->bu_enter_div = 24;
  opt->bu_leave_div = 96;
  return KSPN_OK;
}

size_t
kspn_options_size(void)
{
  return sizeof(kspn_options);
}

size_t
kspn_stats_size(void)
{
  return sizeof(kspn_stats);
}

const char*
kspn_strerror(int status)
{
  switch (status) {
    case KSPN_OK: return "ok";
    case KSPN_ERR_INVALID_ARGUMENT: return "invalid argument";
    case KSPN_ERR_INVALID_GRAPH: return "invalid graph";
    case KSPN_ERR_OOM: return "out of memory";
    case KSPN_ERR_TIMEOUT: return "iteration cap or wait limit reached";
    case KSPN_ERR_CUDA: return "CUDA error";
    case KSPN_ERR_NO_DEVICE: return "no CUDA device";
    case KSPN_ERR_INTERNAL: return "internal consistency check failed";
    default: return "unknown status";
  }
}

const char*
kspn_last_error(const kspn_context* ctx)
{
  return ctx ? ctx->last_error.c_str() : "";
}

int
kspn_context_create_on_stream(int device, void* stream, kspn_context** out)
{
  if (!out) return KSPN_ERR_INVALID_ARGUMENT;
  *out      = nullptr;
  if (device == KSPN_DEVICE_CURRENT && cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return KSPN_ERR_NO_DEVICE;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) {
    cudaGetLastError();
    return KSPN_ERR_NO_DEVICE;
  }
  auto* ctx   = new (std::nothrow) kspn_context;
  if (!ctx) return KSPN_ERR_OOM;
  ctx->device = device;
  int const rc = guard(ctx, [&] {
    bind_device(ctx);
    if (stream) {
      ctx->stream = static_cast<cudaStream_t>(stream);
    } else {
      KSPN_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
      ctx->own_stream = true;
    }
    void* h = nullptr;
    KSPN_CUDA(cudaMallocHost(&h, 64 * sizeof(uint32_t)));
    ctx->h_ctr   = static_cast<uint32_t*>(h);
    ctx->h_ctr64 = reinterpret_cast<uint64_t*>(ctx->h_ctr + 32);
    KSPN_CUDA(cudaMallocHost(&ctx->h_state, 4096));
    for (auto& e : ctx->ev) KSPN_CUDA(cudaEventCreate(&e));
    for (auto& e : ctx->pe) KSPN_CUDA(cudaEventCreate(&e));
  });
  if (rc != KSPN_OK) {
    kspn_context_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return KSPN_OK;
}

int
kspn_context_create(int device, kspn_context** out)
{
  return kspn_context_create_on_stream(device, nullptr, out);
}

int
kspn_context_destroy(kspn_context* ctx)
{
  if (!ctx) return KSPN_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  release_graphs(ctx);
  batch_release(ctx);
  if (ctx->pivot_model) cudaFree(ctx->pivot_model);
  if (ctx->ws.base) cudaFree(ctx->ws.base);
  if (ctx->h_ctr) cudaFreeHost(ctx->h_ctr);
  if (ctx->h_state) cudaFreeHost(ctx->h_state);
  for (auto& b : ctx->bufs)
    if (b.p) cudaFree(b.p);
  for (auto& e : ctx->ev)
    if (e) cudaEventDestroy(e);
  for (auto& e : ctx->pe)
    if (e) cudaEventDestroy(e);
  if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream), cudaStreamDestroy(ctx->copy_stream);
  if (ctx->copy_ev) cudaEventDestroy(ctx->copy_ev);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return KSPN_OK;
}

int
kspn_context_synchronize(kspn_context* ctx)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] { KSPN_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

uint64_t
kspn_context_launches(const kspn_context* ctx)
{
  return ctx ? ctx->launches : 0;
}

int
kspn_scc_device(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint32_t* d_scc_id, const kspn_options* opt, kspn_stats* stats)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && (m == 0 || d_fw_csr) && (n == 0 || d_scc_id), "null device pointer");
    require(n < UNDECIDED, "n must be below 2^32 - 1");
    kspn_options const o = options_or_default(opt);
    bind_device(ctx);
    graph_store  store;
    dgraph const g = with_transpose(ctx, n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, store);
    run_pipeline(ctx, g, d_scc_id, o, stats);
  });
}

int
kspn_scc(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* fw_head, const uint32_t* fw_csr, const uint64_t* bw_head, const uint32_t* bw_csr, uint32_t* scc_id, const kspn_options* opt, kspn_stats* stats)
{
  kspn_context* own = nullptr;
  if (!ctx) {
    int const rc = kspn_context_create(0, &own);
    if (rc != KSPN_OK) return rc;
    ctx = own;
  }
  int const rc = guard(ctx, [&] {
    require(fw_head && (m == 0 || fw_csr) && (n == 0 || scc_id), "null host pointer");
    require((bw_head == nullptr) == (bw_csr == nullptr), "bw_head and bw_csr must both be given or both be NULL");
    require(n < UNDECIDED, "n must be below 2^32 - 1");
    kspn_options const o = options_or_default(opt);
    bind_device(ctx);
    cudaStream_t const s         = ctx->stream;
    size_t const       head_b    = align_up((static_cast<size_t>(n) + 1) * 8);
    size_t const       csr_b     = align_up(std::max<uint64_t>(m, 1) * 4);
    size_t const       out_b     = align_up(std::max<size_t>(n, 1) * 4);
    bool const         has_bw    = bw_head != nullptr;
    size_t const       bytes     = 2 * head_b + 2 * csr_b + out_b;
    char*              p         = static_cast<char*>(context_buffer(ctx, BUF_HOST_GRAPH, bytes));
    auto* dfh = reinterpret_cast<uint64_t*>(p);
    auto* dbh = reinterpret_cast<uint64_t*>(p + head_b);
    auto* dfc = reinterpret_cast<uint32_t*>(p + 2 * head_b);
    auto* dbc = reinterpret_cast<uint32_t*>(p + 2 * head_b + csr_b);
    auto* dout = reinterpret_cast<uint32_t*>(p + 2 * head_b + 2 * csr_b);
    if (has_bw) {
      KSPN_CUDA(cudaMemcpyAsync(dfh, fw_head, (static_cast<size_t>(n) + 1) * 8, cudaMemcpyHostToDevice, s));
      if (m) KSPN_CUDA(cudaMemcpyAsync(dfc, fw_csr, m * 4, cudaMemcpyHostToDevice, s));
      KSPN_CUDA(cudaMemcpyAsync(dbh, bw_head, (static_cast<size_t>(n) + 1) * 8, cudaMemcpyHostToDevice, s));
      if (m) KSPN_CUDA(cudaMemcpyAsync(dbc, bw_csr, m * 4, cudaMemcpyHostToDevice, s));
    } else {
      // the CSC is built while the CSR is still arriving
      upload_transpose(ctx, n, m, fw_head, fw_csr, dfh, dfc, dbh, dbc, 0);
    }
    dgraph const g{ n, m, dfh, dfc, dbh, dbc };
    run_pipeline(ctx, g, dout, o, stats);
    if (n) KSPN_CUDA(cudaMemcpyAsync(scc_id, dout, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost, s));
    KSPN_CUDA(cudaStreamSynchronize(s));
  });
  if (own) {
    if (rc != KSPN_OK) std::fprintf(stderr, "kspn_scc: %s\n", own->last_error.c_str());
    kspn_context_destroy(own);
  }
  return rc;
}

int
kspn_trim_1_first(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint64_t* d_bw_head, uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* pivot)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_bw_head && d_undecided && d_scc_id && pivot, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    clear_bitset_tail(ctx, d_undecided, n);
    dgraph const g{ n, m, d_fw_head, nullptr, d_bw_head, nullptr };
    *pivot = n ? trim_1_first(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id, nullptr, nullptr, false) : 0;
  });
}

int
kspn_forward_backward_search(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t pivot, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_undecided && d_scc_id, "null pointer");
    require(pivot < n, "pivot must be < n");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    kspn_options o;
    kspn_options_default(&o);
    dgraph const   g{ n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr };
    uint32_t const d = fw_bw(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id, pivot, o, nullptr, false);
    if (decided) *decided = d;
  });
}

int
kspn_trim_1_normal(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_undecided && d_scc_id, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    dgraph const   g{ n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr };
    uint32_t const d = n ? trim_1_normal(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id) : 0;
    if (decided) *decided = d;
  });
}

int
kspn_label_search(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint64_t* d_undecided, uint32_t* d_scc_id, int rotation, uint32_t* d_label, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_undecided && d_scc_id, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    kspn_options o;
    kspn_options_default(&o);
    dgraph const   g{ n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr };
    uint32_t const d = n ? label_search(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id, rotation, o, nullptr) : 0;
    if (d_label && n) KSPN_CUDA(cudaMemcpyAsync(d_label, ctx->ws.label, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToDevice, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    if (decided) *decided = d;
  });
}

int
kspn_trim_1_exhaustive_first(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* d_outdegree, uint32_t* d_indegree, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_undecided && d_scc_id && d_outdegree && d_indegree, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    clear_bitset_tail(ctx, d_undecided, n);
    dgraph const   g{ n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr };
    uint32_t const d = n ? trim_exhaustive_first(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id, d_outdegree, d_indegree) : 0;
    if (decided) *decided = d;
  });
}

int
kspn_trim_1_fixpoint(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_undecided && d_scc_id, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    dgraph const   g{ n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr };
    uint32_t const d = n ? trim_fixpoint(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id, false, 0) : 0;
    if (decided) *decided = d;
  });
}

int
kspn_trim_2(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_undecided && d_scc_id, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    dgraph const   g{ n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr };
    uint32_t const d = n ? trim_2(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id) : 0;
    if (decided) *decided = d;
  });
}

int
kspn_set_pivot_model(kspn_context* ctx, const float* params)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    bind_device(ctx);
    if (!params) {
      if (ctx->pivot_model) {
        KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->pivot_model);
      }
      ctx->pivot_model = nullptr;
      return;
    }
    if (!ctx->pivot_model) {
      void* p = nullptr;
      if (cudaMalloc(&p, KSPN_MLP_PARAMS * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        throw error{ KSPN_ERR_OOM, "pivot model" };
      }
      ctx->pivot_model = static_cast<float*>(p);
    }
    KSPN_CUDA(cudaMemcpyAsync(ctx->pivot_model, params, KSPN_MLP_PARAMS * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_mlp_features(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint32_t count,
                  const uint32_t* d_vertices, float* d_features)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(count == 0 || (d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_vertices && d_features), "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    dgraph const g{ n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr };
    mlp_features(ctx, g, count, d_vertices, d_features);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_mlp_forward(kspn_context* ctx, uint32_t count, const float* d_features, const float* d_params, float* d_logits)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_params && (count == 0 || (d_features && d_logits)), "null pointer");
    bind_device(ctx);
    mlp_forward(ctx, count, d_features, d_params, d_logits);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_mlp_gradient(kspn_context* ctx, uint32_t count, const float* d_features, const float* d_labels, const float* d_params, float* d_grad, float* d_loss)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_params && d_grad && d_loss && (count == 0 || (d_features && d_labels)), "null pointer");
    bind_device(ctx);
    mlp_grad(ctx, count, d_features, d_labels, d_params, d_grad, d_loss);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_mlp_adam(kspn_context* ctx, float* d_params, const float* d_grad, float* d_m, float* d_v, float lr, int step)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_params && d_grad && d_m && d_v, "null pointer");
    require(step >= 1, "step counts from 1");
    bind_device(ctx);
    mlp_adam(ctx, d_params, d_grad, d_m, d_v, lr, step);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_residual(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided, uint32_t* pieces_left)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && (m == 0 || d_fw_csr) && d_undecided && d_scc_id, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, m);
    dgraph const   g{ n, m, d_fw_head, d_fw_csr, nullptr, nullptr };
    uint32_t       left = 0;
    uint32_t const d    = n ? residual(ctx, g, reinterpret_cast<uint32_t*>(d_undecided), d_scc_id, &left) : 0;
    if (decided) *decided = d;
    if (pieces_left) *pieces_left = left;
  });
}

void
kspn_batch_options_default(kspn_batch_options* opt)
{
  if (opt) std::memset(opt, 0, sizeof(*opt));
}

int
kspn_scc_batched(kspn_context* ctx, uint32_t count, uint64_t n_total, const uint64_t* d_vtx_off, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head,
                 const uint32_t* d_bw_csr, uint32_t* d_scc_id, const kspn_batch_options* opt, kspn_batch_stats* stats)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(count == 0 || (d_vtx_off && d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_scc_id), "null pointer");
    require(n_total < 0xFFFFFFFFull, "n_total must be below 2^32 - 1");
    bind_device(ctx);
    kspn_batch_options o{};
    if (opt) o = *opt;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    KSPN_CUDA(cudaEventRecord(ctx->ev[KSPN_PHASES], ctx->stream));
    if (o.route != 1 || !scc_batched_union(ctx, count, n_total, d_vtx_off, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, d_scc_id, stats))
      scc_batched(ctx, count, n_total, d_vtx_off, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, d_scc_id, o, stats);
    KSPN_CUDA(cudaEventRecord(ctx->ev[KSPN_PHASES + 1], ctx->stream));
    KSPN_CUDA(cudaEventSynchronize(ctx->ev[KSPN_PHASES + 1]));
    if (stats) KSPN_CUDA(cudaEventElapsedTime(&stats->ms, ctx->ev[KSPN_PHASES], ctx->ev[KSPN_PHASES + 1]));
  });
}

int
kspn_autotune(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head, const uint32_t* d_bw_csr, uint32_t* d_scc_id,
              const kspn_options* base, uint32_t reps, kspn_options* best, kspn_tune_report* report)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && (m == 0 || d_fw_csr) && (n == 0 || d_scc_id) && best, "null pointer");
    require(n < UNDECIDED, "n must be below 2^32 - 1");
    kspn_options o = options_or_default(base);
    o.validate     = 0; // validated once below
    bind_device(ctx);
    graph_store  store;
    dgraph const g = with_transpose(ctx, n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, store);
    ensure_workspace(ctx, g.n, g.m); // counters of the validation and the check
    if (base == nullptr || base->validate) validate(ctx, g);
    uint32_t const R = reps ? reps : 3;
    tune_check chk{ ctx, n };
    auto run = [&](kspn_options const& c) {
      run_pipeline(ctx, g, d_scc_id, c, nullptr); // warm-up
      chk.take(d_scc_id);
      float best_ms = 1e30f;
      for (uint32_t r = 0; r < R; ++r) {
        KSPN_CUDA(cudaEventRecord(ctx->ev[KSPN_PHASES], ctx->stream));
        run_pipeline(ctx, g, d_scc_id, c, nullptr);
        KSPN_CUDA(cudaEventRecord(ctx->ev[KSPN_PHASES + 1], ctx->stream));
        KSPN_CUDA(cudaEventSynchronize(ctx->ev[KSPN_PHASES + 1]));
        float ms = 0;
        KSPN_CUDA(cudaEventElapsedTime(&ms, ctx->ev[KSPN_PHASES], ctx->ev[KSPN_PHASES + 1]));
        best_ms = std::min(best_ms, ms);
      }
      return best_ms;
    };
    using S = std::function<void(kspn_options&)>;
    std::vector<std::vector<S>> axes;
    {
      std::vector<S> a;
      for (uint32_t v : { 6u, 12u, 24u, 48u, 96u }) a.push_back([v](kspn_options& x) { x.bu_enter_div = v; });
      axes.push_back(a);
    }
    {
      std::vector<S> a;
      for (uint32_t v : { 24u, 48u, 96u, 192u, 384u }) a.push_back([v](kspn_options& x) { x.bu_leave_div = v; });
      axes.push_back(a);
    }
    axes.push_back({ [](kspn_options& x) { x.trim2 = 0; }, [](kspn_options& x) { x.trim2 = 1; } });
    if (ctx->pivot_model) axes.push_back({ [](kspn_options& x) { x.learned_pivot = 0; }, [](kspn_options& x) { x.learned_pivot = 1; } });
    kspn_options r = tune(o, axes, run, report);
    r.validate     = base ? base->validate : 1;
    *best          = r;
    run_pipeline(ctx, g, d_scc_id, r, nullptr); // leave the chosen settings' ids
  });
}

int
kspn_autotune_batched(kspn_context* ctx, uint32_t count, uint64_t n_total, const uint64_t* d_vtx_off, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, const uint64_t* d_bw_head,
                      const uint32_t* d_bw_csr, uint32_t* d_scc_id, const kspn_batch_options* base, uint32_t reps, kspn_batch_options* best, kspn_tune_report* report)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(count == 0 || (d_vtx_off && d_fw_head && d_fw_csr && d_bw_head && d_bw_csr && d_scc_id), "null pointer");
    require(best, "null pointer");
    require(n_total < 0xFFFFFFFFull, "n_total must be below 2^32 - 1");
    bind_device(ctx);
    kspn_batch_options o{};
    if (base) o = *base;
    uint32_t const R = reps ? reps : 3;
    tune_check     chk{ ctx, n_total };
    auto           run = [&](kspn_batch_options const& c) {
      scc_batched(ctx, count, n_total, d_vtx_off, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, d_scc_id, c, nullptr); // warm-up (and capture)
      chk.take(d_scc_id);
      float best_ms = 1e30f;
      for (uint32_t r = 0; r < R; ++r) {
        KSPN_CUDA(cudaEventRecord(ctx->ev[KSPN_PHASES], ctx->stream));
        scc_batched(ctx, count, n_total, d_vtx_off, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, d_scc_id, c, nullptr);
        KSPN_CUDA(cudaEventRecord(ctx->ev[KSPN_PHASES + 1], ctx->stream));
        KSPN_CUDA(cudaEventSynchronize(ctx->ev[KSPN_PHASES + 1]));
        float ms = 0;
        KSPN_CUDA(cudaEventElapsedTime(&ms, ctx->ev[KSPN_PHASES], ctx->ev[KSPN_PHASES + 1]));
        best_ms = std::min(best_ms, ms);
      }
      return best_ms;
    };
    using S = std::function<void(kspn_batch_options&)>;
    std::vector<std::vector<S>> axes;
    {
      std::vector<S> a;
      a.push_back([](kspn_batch_options& x) { x.cluster_size = 1, x.cluster_min = 0; });
      for (uint32_t cs : { 2u, 4u, 8u })
        for (uint64_t cm : { 1ull << 15, 1ull << 17 }) a.push_back([cs, cm](kspn_batch_options& x) { x.cluster_size = cs, x.cluster_min = cm; });
      axes.push_back(a);
    }
    axes.push_back({ [](kspn_batch_options& x) { x.search = 1; }, [](kspn_batch_options& x) { x.search = 2; } });
    {
      std::vector<S> a;
      for (uint32_t v : { 64u, 256u, 512u }) a.push_back([v](kspn_batch_options& x) { x.rem_tarjan = v; });
      axes.push_back(a);
    }
    {
      std::vector<S> a;
      for (uint32_t v : { 8u, 64u, 512u }) a.push_back([v](kspn_batch_options& x) { x.max_rounds = v; });
      axes.push_back(a);
    }
    kspn_batch_options const r = tune(o, axes, run, report);
    *best                      = r;
    scc_batched(ctx, count, n_total, d_vtx_off, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, d_scc_id, r, nullptr);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_manifest_read(const char* path, kspn_manifest* out)
{
  try {
    if (!path || !out) return KSPN_ERR_INVALID_ARGUMENT;
    manifest_read(path, out);
    return KSPN_OK;
  } catch (error const& e) {
    return e.code;
  } catch (...) {
    return KSPN_ERR_INTERNAL;
  }
}

int
kspn_manifest_load(kspn_context* ctx, const kspn_manifest* mf, uint64_t* d_fw_head, uint32_t* d_fw_csr, uint64_t* d_bw_head, uint32_t* d_bw_csr)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(mf && d_fw_head && d_bw_head && (mf->edge_count == 0 || (d_fw_csr && d_bw_csr)), "null pointer");
    bind_device(ctx);
    manifest_load(ctx, *mf, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr);
  });
}

int
kspn_manifest_write(const char* dir, const char* name, uint32_t n, uint64_t m, const uint64_t* fw_head, const uint32_t* fw_csr, const uint64_t* bw_head, const uint32_t* bw_csr,
                    uint32_t head_bytes, uint32_t csr_bytes, int big_endian, int self_loops, int duplicate_edges)
{
  try {
    if (!dir || !name || !fw_head || !bw_head || (m && (!fw_csr || !bw_csr))) return KSPN_ERR_INVALID_ARGUMENT;
    manifest_write(dir, name, n, m, fw_head, fw_csr, bw_head, bw_csr, head_bytes, csr_bytes, big_endian, self_loops, duplicate_edges);
    return KSPN_OK;
  } catch (error const& e) {
    return e.code;
  } catch (...) {
    return KSPN_ERR_INTERNAL;
  }
}

void
kspn_batch_shape(uint32_t count, uint64_t seed, uint32_t log2_min, uint32_t log2_max, float deg_min, float deg_max, uint32_t* n_out, uint64_t* draws_out)
{
  batch_shape(count, seed, log2_min, log2_max, deg_min, deg_max, n_out, draws_out);
}

int
kspn_gen_batch(kspn_context* ctx, uint32_t count, uint64_t seed, const uint64_t* d_vtx_off, const uint64_t* d_draw_off, const uint32_t* d_graph_ids, uint32_t* d_src, uint32_t* d_dst)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(count == 0 || (d_vtx_off && d_draw_off && d_src && d_dst), "null pointer");
    bind_device(ctx);
    uint64_t total = 0;
    if (count) {
      KSPN_CUDA(cudaMemcpyAsync(&total, d_draw_off + count, sizeof(total), cudaMemcpyDeviceToHost, ctx->stream));
      KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    gen_batch(ctx, count, seed, d_vtx_off, d_draw_off, d_graph_ids, total, d_src, d_dst);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_batch_localize(kspn_context* ctx, uint32_t count, uint64_t n_total, const uint64_t* d_vtx_off, const uint64_t* d_head, uint32_t* d_csr)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(count == 0 || (d_vtx_off && d_head && d_csr), "null pointer");
    bind_device(ctx);
    batch_localize(ctx, count, n_total, d_vtx_off, d_head, d_csr);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_normalise(kspn_context* ctx, uint32_t n, uint32_t* d_scc_id)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(n == 0 || d_scc_id, "null pointer");
    bind_device(ctx);
    ensure_workspace(ctx, n, 0);
    canonicalise(ctx, n, d_scc_id, ctx->ws.label, false);
  });
}

int
kspn_transpose(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* d_fw_head, const uint32_t* d_fw_csr, uint64_t* d_bw_head, uint32_t* d_bw_csr)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_fw_head && d_bw_head && (m == 0 || (d_fw_csr && d_bw_csr)), "null pointer");
    bind_device(ctx);
    transpose(ctx, n, m, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, nullptr);
  });
}

int
kspn_upload_transpose(kspn_context* ctx, uint32_t n, uint64_t m, const uint64_t* fw_head, const uint32_t* fw_csr, uint64_t* d_fw_head, uint32_t* d_fw_csr, uint64_t* d_bw_head, uint32_t* d_bw_csr, uint64_t chunk_edges)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(fw_head && d_fw_head && d_bw_head && (m == 0 || (fw_csr && d_fw_csr && d_bw_csr)), "null pointer");
    require(n < UNDECIDED, "n must be below 2^32 - 1");
    bind_device(ctx);
    upload_transpose(ctx, n, m, fw_head, fw_csr, d_fw_head, d_fw_csr, d_bw_head, d_bw_csr, chunk_edges);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_gen_gnm(kspn_context* ctx, uint32_t n, uint64_t draws, uint64_t seed, uint32_t* d_src, uint32_t* d_dst)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(draws == 0 || (d_src && d_dst), "null pointer");
    bind_device(ctx);
    gen_gnm(ctx, n, draws, seed, d_src, d_dst);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_gen_rmat(kspn_context* ctx, int scale, uint64_t draws, uint64_t seed, uint64_t t_a, uint64_t t_ab, uint64_t t_abc, int permute, uint32_t* d_src, uint32_t* d_dst)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(draws == 0 || (d_src && d_dst), "null pointer");
    require(scale >= 0 && scale <= 31, "scale must be in [0, 31]");
    bind_device(ctx);
    gen_rmat(ctx, scale, draws, seed, t_a, t_ab, t_abc, permute, d_src, d_dst);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_gen_rgg(kspn_context* ctx, uint32_t n, uint64_t seed, uint32_t g, uint64_t r2, uint32_t* d_src, uint32_t* d_dst, uint64_t capacity, uint64_t* m_out)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require((d_src == nullptr) == (d_dst == nullptr), "d_src and d_dst must both be given or both be NULL");
    bind_device(ctx);
    uint64_t const m = gen_rgg(ctx, n, seed, g, r2, d_src, d_dst, capacity);
    if (m_out) *m_out = m;
    require(!d_src || m <= capacity, "edge buffers smaller than the edge count");
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int
kspn_build_csr(kspn_context* ctx, uint32_t n, uint64_t m_raw, uint32_t* d_src, uint32_t* d_dst, uint64_t* d_head, uint32_t* d_csr, uint64_t* m_out)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return guard(ctx, [&] {
    require(d_head && (m_raw == 0 || (d_src && d_dst && d_csr)), "null pointer");
    bind_device(ctx);
    uint64_t const m = build_csr(ctx, n, m_raw, d_src, d_dst, d_head, d_csr);
    if (m_out) *m_out = m;
  });
}

} // extern "C"
