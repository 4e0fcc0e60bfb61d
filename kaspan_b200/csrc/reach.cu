// Single-pivot forward-backward search on the device.
//
// Reference: cache_forward_backward_search (kaspan/scc/cache_pivot_search.hpp:16-104),
// equal to forward_backward_search (pivot_search.hpp:15-85) at one rank:
//   FW  = vertices reachable from the pivot through undecided vertices
//   BW  = vertices of FW that reach the pivot through FW vertices
//   BW is the pivot's SCC; each member is decided with id = pivot.
// The reference walks a LIFO stack on one core; here each search is a
// level-synchronous, direction-optimising reachability:
//   top-down  : load-balanced expansion of the frontier's rows (expand.cuh),
//               visited set = a bitmap claimed with atomicOr;
//   bottom-up : every candidate scans its opposite-direction row and stops
//               at the first visited neighbour (used while the frontier is a
//               large share of the candidates).
// Only the reached SET matters, which neither order changes.
#include "expand.cuh"

namespace kspn {

namespace {

constexpr int      R_THREADS = 256;
constexpr int      CTR_NTILES = 8;
constexpr int      R_BIG      = 32;

unsigned
r_grid(uint64_t items)
{
  uint64_t const b = (items + R_THREADS - 1) / R_THREADS;
  return static_cast<unsigned>(b < 148ull * 8 ? (b ? b : 1) : 148ull * 8);
}

__global__ void
k_reach_seed(uint32_t* vis, uint32_t* q, uint32_t* qn, uint32_t pivot)
{
  q[0]  = pivot;
  *qn   = 1;
  vis[pivot >> 5] |= 1u << (pivot & 31);
}

// BW seed: the pivot leaves FW, joins BW, is decided with id = itself.
__global__ void
k_bw_seed(uint32_t* fwvis, uint32_t* bwvis, uint32_t* und, uint32_t* scc_id, uint32_t* q, uint32_t* qn, uint32_t pivot)
{
  uint32_t const mask = 1u << (pivot & 31);
  fwvis[pivot >> 5] &= ~mask;
  bwvis[pivot >> 5] |= mask;
  und[pivot >> 5] &= ~mask;
  scc_id[pivot] = pivot;
  q[0]          = pivot;
  *qn           = 1;
}

struct fw_td_op
{
  uint32_t const* und;
  uint32_t*       vis;
  uint32_t*       qout;
  uint32_t*       qout_n;
  __device__ __forceinline__ void operator()(uint32_t, uint32_t v, bool valid) const
  {
    bool const won = valid && bit_get(und, v) && !bit_get(vis, v) && bit_claim(vis, v);
    warp_push(won, v, qout, qout_n);
  }
};

struct bw_td_op
{
  uint32_t* fwvis;
  uint32_t* bwvis;
  uint32_t* und;
  uint32_t* scc_id;
  uint32_t  pivot;
  uint32_t* qout;
  uint32_t* qout_n;
  uint32_t* decided;
  __device__ __forceinline__ void operator()(uint32_t, uint32_t v, bool valid) const
  {
    bool const won = valid && bit_get(fwvis, v) && bit_take(fwvis, v);
    if (won) {
      bit_take(und, v);
      bit_claim(bwvis, v);
      scc_id[v] = pivot;
    }
    unsigned const b = __ballot_sync(0xFFFFFFFFu, won);
    if (b && (threadIdx.x & 31) == 0) atomicAdd(decided, static_cast<uint32_t>(__popc(b)));
    warp_push(won, v, qout, qout_n);
  }
};

// Bottom-up sweep.  Candidates: FW = undecided and not visited; BW =
// FW-visited (not yet BW-visited).  A candidate joins when a neighbour in
// `row` (FW: in-edges, BW: out-edges) is in `seen`.
template<bool BW>
__global__ void __launch_bounds__(R_THREADS)
k_bottom_up(uint32_t n,
            uint64_t const* __restrict__ head,
            uint32_t const* __restrict__ adj,
            uint32_t* __restrict__ und,
            uint32_t* __restrict__ cand_bm, // FW: vis (claimed into); BW: fwvis (taken from)
            uint32_t* __restrict__ seen,    // FW: vis;                  BW: bwvis
            uint32_t* __restrict__ scc_id,
            uint32_t pivot,
            uint32_t* __restrict__ qout,
            uint32_t* __restrict__ qout_n,
            uint32_t* __restrict__ decided,
            unsigned long long* __restrict__ edges)
{
  unsigned const lane  = threadIdx.x & 31u;
  uint64_t const span  = (static_cast<uint64_t>(n) + 31) & ~31ull;
  uint64_t       nedge = 0, ncand = 0;
  uint32_t       ndec  = 0;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * R_THREADS) {
    uint32_t const v = static_cast<uint32_t>(t);
    bool           cand;
    if (BW) cand = t < n && bit_get(cand_bm, v);
    else cand = t < n && bit_get(und, v) && !bit_get(cand_bm, v);
    uint64_t b = 0, e = 0;
    if (cand) b = head[v], e = head[v + 1], ++ncand;
    bool       found = false;
    bool const big   = cand && (e - b) >= R_BIG;
    if (cand && !big) {
      for (uint64_t x = b; x < e; ++x) {
        ++nedge;
        if (bit_get(seen, adj[x])) {
          found = true;
          break;
        }
      }
    }
    unsigned todo = __ballot_sync(0xFFFFFFFFu, big);
    while (todo) {
      unsigned const l = __ffs(todo) - 1;
      todo &= todo - 1;
      uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, b, l), e0 = __shfl_sync(0xFFFFFFFFu, e, l);
      bool           hit = false;
      for (uint64_t x = b0; x < e0; x += 32) {
        bool const mine = x + lane < e0 && bit_get(seen, adj[x + lane]);
        nedge += (x + lane < e0);
        if (__any_sync(0xFFFFFFFFu, mine)) {
          hit = true;
          break;
        }
      }
      if (lane == l) found = hit;
    }
    bool won = false;
    if (found) {
      if (BW) {
        won = bit_take(cand_bm, v);
        if (won) {
          bit_take(und, v);
          bit_claim(seen, v);
          scc_id[v] = pivot;
          ++ndec;
        }
      } else {
        won = bit_claim(cand_bm, v);
      }
    }
    warp_push(won, v, qout, qout_n);
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    nedge += __shfl_down_sync(0xFFFFFFFFu, nedge, s);
    ncand += __shfl_down_sync(0xFFFFFFFFu, ncand, s);
    ndec += __shfl_down_sync(0xFFFFFFFFu, ndec, s);
  }
  if (lane == 0) {
    if (nedge) atomicAdd(edges, static_cast<unsigned long long>(nedge));
    if (ncand) atomicAdd(edges + 1, static_cast<unsigned long long>(ncand));
    if (ndec) atomicAdd(decided, ndec);
  }
}

struct search_result
{
  uint32_t levels    = 0;
  uint32_t bottom_up = 0;
};

// Runs one search from the queue seeded in q0 (length in ctr[CTR_Q0]).
template<bool BW>
search_result
run_search(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t pivot, uint32_t n_cand, kspn_options const& opt)
{
  auto&          ws  = ctx->ws;
  search_result  res;
  uint32_t*      q[2]  = { ws.q0, ws.q1 };
  uint32_t*      qc[2] = { ws.ctr + CTR_Q0, ws.ctr + CTR_Q1 };
  auto*          edges = reinterpret_cast<unsigned long long*>(ws.ctr64);
  uint32_t const enter = opt.bu_enter_div ? opt.bu_enter_div : 1;
  uint32_t const leave = opt.bu_leave_div ? opt.bu_leave_div : 1;
  uint32_t const cap   = opt.max_levels ? opt.max_levels : g.n + 2;
  bool           bu    = false;
  int            cur   = 0;
  // top-down: FW expands out-rows, BW expands in-rows; bottom-up the opposite
  uint64_t const* td_head = BW ? g.bh : g.fh;
  uint32_t const* td_adj  = BW ? g.bc : g.fc;
  uint64_t const* bu_head = BW ? g.fh : g.bh;
  uint32_t const* bu_adj  = BW ? g.fc : g.bc;
  uint32_t qn_cur = 1;
  uint64_t e0 = ctx->h_ctr64[0], c0 = ctx->h_ctr64[1];
  for (;;) {
    if (res.levels >= cap) throw error{ KSPN_ERR_TIMEOUT, "reachability: level cap exceeded" };
    int const nxt = cur ^ 1;
    KSPN_CUDA(cudaMemsetAsync(qc[nxt], 0, sizeof(uint32_t), ctx->stream));
    if (!bu) {
      if (BW) {
        bw_td_op op{ ws.vis_a, ws.vis_b, und, scc_id, pivot, q[nxt], qc[nxt], ws.ctr + CTR_DECIDED };
        expand_level(ctx, td_head, td_adj, q[cur], qc[cur], ws.ctr + CTR_NTILES, edges, ws.tile_start, op);
      } else {
        fw_td_op op{ und, ws.vis_a, q[nxt], qc[nxt] };
        expand_level(ctx, td_head, td_adj, q[cur], qc[cur], ws.ctr + CTR_NTILES, edges, ws.tile_start, op);
      }
    } else {
      prof_start(ctx);
      k_bottom_up<BW><<<r_grid(g.n), R_THREADS, 0, ctx->stream>>>(g.n, bu_head, bu_adj, und, ws.vis_a, BW ? ws.vis_b : ws.vis_a, scc_id, pivot, q[nxt], qc[nxt], ws.ctr + CTR_DECIDED, edges);
      prof_stop(ctx);
      KSPN_CHECK_LAUNCH();
      ctx->launches += 1;
      res.bottom_up += 1;
    }
    res.levels += 1;
    read_counters(ctx);
    uint32_t const qn = ctx->h_ctr[CTR_Q0 + nxt];
    {
      uint64_t const de = ctx->h_ctr64[0] - e0, dc = ctx->h_ctr64[1] - c0;
      e0 = ctx->h_ctr64[0];
      c0 = ctx->h_ctr64[1];
      if (!bu) prof_add(ctx, KSPN_KERNEL_EXPAND, expand_bytes(qn_cur, de, qn, BW ? 4 : 0));
      // bottom-up: candidate sweep reads the bitmaps (n/8 B each), then per
      // candidate its offset pair, per edge id + probe, per join 4 B (+4 B BW id)
      else prof_add(ctx, KSPN_KERNEL_BOTTOM_UP, (BW ? 1 : 2) * (static_cast<uint64_t>(g.n) / 8) + 16 * dc + 8 * de + (BW ? 8 : 4) * static_cast<uint64_t>(qn));
    }
    qn_cur = qn;
    if (qn == 0) break;
    if (!bu && static_cast<uint64_t>(qn) * enter > n_cand) bu = true;
    else if (bu && static_cast<uint64_t>(qn) * leave < n_cand) bu = false;
    cur = nxt;
  }
  return res;
}

} // namespace

uint32_t
fw_bw(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t pivot, kspn_options const& opt, kspn_stats* st)
{
  auto&        ws    = ctx->ws;
  size_t const words = (static_cast<size_t>(g.n) + 31) / 32;
  if (pivot >= g.n) throw error{ KSPN_ERR_INVALID_ARGUMENT, "forward_backward_search: pivot >= n" };
  uint32_t const n_und = count_undecided(ctx, g.n, und);
  KSPN_CUDA(cudaMemsetAsync(ws.vis_a, 0, words * 4, ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.vis_b, 0, words * 4, ctx->stream));
  zero_counters(ctx);
  k_reach_seed<<<1, 1, 0, ctx->stream>>>(ws.vis_a, ws.q0, ws.ctr + CTR_Q0, pivot);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  search_result const fw = run_search<false>(ctx, g, und, scc_id, pivot, n_und, opt);

  KSPN_CUDA(cudaMemsetAsync(ws.ctr + CTR_DECIDED, 0, sizeof(uint32_t), ctx->stream));
  k_bw_seed<<<1, 1, 0, ctx->stream>>>(ws.vis_a, ws.vis_b, und, scc_id, ws.q0, ws.ctr + CTR_Q0, pivot);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  read_counters(ctx); // CTR_DECIDED was reset after the FW counters were read
  search_result const bw = run_search<true>(ctx, g, und, scc_id, pivot, n_und, opt);
  read_counters(ctx);
  uint32_t const decided = ctx->h_ctr[CTR_DECIDED] + 1; // + the pivot
  if (st) {
    if (st->levels_fw == 0 && st->levels_bw == 0) {
      st->levels_fw        = fw.levels;
      st->levels_bw        = bw.levels;
      st->levels_bottom_up = fw.bottom_up + bw.bottom_up;
    }
    st->edges_scanned = ctx->h_ctr64[0];
  }
  return decided;
}

} // namespace kspn
