// Multi-pivot label ("colour") search on the device.
//
// Reference: cache_label_search_pull (kaspan/scc/cache_multi_pivot_search_pull.hpp:40-244)
// with map = rotr(., rotation), unmap = rotl(., rotation)
// (cache_rot_label_search_pull, :246-266).  At one rank it computes:
//   FW    label[k] = min map(u) over k's undecided ancestors u (k included),
//         the fixpoint of pulling the minimum over undecided in-neighbours;
//   roots undecided k with label[k] == map(k): decided, id = k;
//   BW    an undecided k is decided (id = unmap(label[k])) when an
//         out-neighbour was decided with the same label.
// The fixpoint is unique, so the device may reach it in any order: here a
// push form over a worklist — every vertex whose label dropped offers it to
// its undecided out-neighbours with atomicMin, and joins the next level's
// worklist (a per-level claim bitmap keeps each vertex once per level).
// The backward closure pushes from newly decided vertices over in-edges.
#include "expand.cuh"

namespace kspn {

namespace {

constexpr int L_THREADS  = 256;
constexpr int CTR_NTILES = 8;

unsigned
l_grid(uint64_t items)
{
  uint64_t const b = (items + L_THREADS - 1) / L_THREADS;
  return static_cast<unsigned>(b < 148ull * 8 ? (b ? b : 1) : 148ull * 8);
}

// label = map(v) for undecided v (all queued), UNDECIDED otherwise.
__global__ void __launch_bounds__(L_THREADS)
k_label_init(uint32_t n, uint32_t const* __restrict__ und, uint32_t* __restrict__ label, int rot, uint32_t* __restrict__ q, uint32_t* __restrict__ qn)
{
  __shared__ uint32_t s_buf[DENSE_BUF];
  __shared__ uint32_t s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  block_queue    bq{ s_buf, &s_n };
  uint64_t const span = (static_cast<uint64_t>(n) + L_THREADS - 1) / L_THREADS * L_THREADS;
  for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * L_THREADS; base < span; base += static_cast<uint64_t>(gridDim.x) * L_THREADS) {
    uint64_t const t    = base + threadIdx.x;
    uint32_t const v    = static_cast<uint32_t>(t);
    bool const     live = t < n && bit_get(und, v);
    if (t < n) label[v] = live ? rotr32(v, rot) : UNDECIDED;
    bq.push(live, v);
    __syncthreads();
    if (s_n > DENSE_BUF - L_THREADS) bq.flush(q, qn, &s_base);
  }
  bq.flush(q, qn, &s_base);
}

struct label_fw_op
{
  uint32_t const* und;
  uint32_t*       label;
  uint32_t*       claim_next;
  __device__ __forceinline__ uint32_t probe(uint32_t v) const { return und[v >> 5]; }
  __device__ __forceinline__ bool     operator()(uint32_t u, uint32_t v, bool valid, uint32_t word) const
  {
    if (!valid || !((word >> (v & 31)) & 1u)) return false;
    uint32_t const lu = __ldcg(label + u);
    if (lu >= __ldcg(label + v)) return false;
    uint32_t const old = atomicMin(label + v, lu);
    return lu < old && bit_claim(claim_next, v);
  }
};

// Clears the claim bits of the queue about to be expanded (they were set
// when its entries were pushed); runs before the level that pushes into the
// other bitmap, so no push races with the clearing.
__global__ void
k_unclaim(uint32_t const* __restrict__ q, uint32_t const* __restrict__ qn_ptr, uint32_t* __restrict__ claim)
{
  uint32_t const qn = *qn_ptr;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < qn; i += gridDim.x * blockDim.x) {
    uint32_t const v = q[i];
    atomicAnd(claim + (v >> 5), ~(1u << (v & 31)));
  }
}

__global__ void __launch_bounds__(L_THREADS)
k_label_roots(uint32_t n, uint32_t* __restrict__ und, uint32_t const* __restrict__ label, uint32_t* __restrict__ scc_id, int rot, uint32_t* __restrict__ q, uint32_t* __restrict__ qn, uint32_t* __restrict__ decided)
{
  __shared__ uint32_t s_buf[DENSE_BUF];
  __shared__ uint32_t s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  block_queue    bq{ s_buf, &s_n };
  uint64_t const span = (static_cast<uint64_t>(n) + L_THREADS - 1) / L_THREADS * L_THREADS;
  uint32_t       dec  = 0;
  for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * L_THREADS; base < span; base += static_cast<uint64_t>(gridDim.x) * L_THREADS) {
    uint64_t const t    = base + threadIdx.x;
    uint32_t const v    = static_cast<uint32_t>(t);
    bool const     root = t < n && bit_get(und, v) && label[v] == rotr32(v, rot);
    bool const     won  = root && bit_take(und, v);
    if (won) {
      scc_id[v] = v;
      ++dec;
    }
    bq.push(won, v);
    __syncthreads();
    if (s_n > DENSE_BUF - L_THREADS) bq.flush(q, qn, &s_base);
  }
  bq.flush(q, qn, &s_base);
  if (dec) atomicAdd(decided, dec);
}

struct label_bw_op
{
  uint32_t*       und;
  uint32_t const* label;
  uint32_t*       scc_id;
  int             rot;
  // u = decided vertex, v = one of its in-neighbours; every push is a decision
  __device__ __forceinline__ uint32_t probe(uint32_t v) const { return und[v >> 5]; }
  __device__ __forceinline__ bool     operator()(uint32_t u, uint32_t v, bool valid, uint32_t word) const
  {
    if (!valid || !((word >> (v & 31)) & 1u)) return false;
    uint32_t const lu = label[u];
    if (label[v] != lu || !bit_take(und, v)) return false;
    scc_id[v] = rotl32(lu, rot);
    return true;
  }
};

} // namespace

uint32_t
label_search(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, int rotation, kspn_options const& opt, kspn_stats* st)
{
  auto&          ws    = ctx->ws;
  size_t const   words = (static_cast<size_t>(g.n) + 31) / 32;
  uint32_t*      q[2]  = { ws.q0, ws.q1 };
  uint32_t*      qc[2] = { ws.ctr + CTR_Q0, ws.ctr + CTR_Q1 };
  uint32_t*      claim[2] = { ws.vis_a, ws.vis_b };
  auto*          edges = reinterpret_cast<unsigned long long*>(ws.ctr64);
  uint32_t const cap   = opt.max_label_iters ? opt.max_label_iters : g.n + 2;

  zero_counters(ctx);
  KSPN_CUDA(cudaMemsetAsync(ws.vis_a, 0, words * 4, ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.vis_b, 0, words * 4, ctx->stream));
  k_label_init<<<l_grid(g.n), L_THREADS, 0, ctx->stream>>>(g.n, und, ws.label, rotation, q[0], qc[0]);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;

  // forward: min-label fixpoint
  read_counters(ctx);
  uint32_t qn_cur = ctx->h_ctr[CTR_Q0];
  uint64_t e0     = ctx->h_ctr64[0];
  int      cur    = 0;
  for (uint32_t level = 0;; ++level) {
    if (level >= cap) throw error{ KSPN_ERR_TIMEOUT, "label search: propagation cap exceeded" };
    int const nxt = cur ^ 1;
    KSPN_CUDA(cudaMemsetAsync(qc[nxt], 0, sizeof(uint32_t), ctx->stream));
    if (level > 0) {
      k_unclaim<<<l_grid(g.n), L_THREADS, 0, ctx->stream>>>(q[cur], qc[cur], claim[cur]);
      ctx->launches += 1;
    }
    expand_level(ctx, g.fh, g.fc, q[cur], qc[cur], ws.ctr + CTR_NTILES, edges, ws.tile_start, q[nxt], qc[nxt], label_fw_op{ und, ws.label, claim[nxt] });
    read_counters(ctx);
    uint32_t const qn = ctx->h_ctr[CTR_Q0 + nxt];
    prof_add(ctx, 0, KSPN_KERNEL_EXPAND, expand_bytes(qn_cur, ctx->h_ctr64[0] - e0, qn, 4)); // + label[u] read per row
    e0     = ctx->h_ctr64[0];
    qn_cur = qn;
    if (qn == 0) break;
    cur = nxt;
  }

  // roots, then the backward closure inside each label class
  KSPN_CUDA(cudaMemsetAsync(ws.ctr + CTR_Q0, 0, 2 * sizeof(uint32_t), ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.ctr + CTR_DECIDED, 0, sizeof(uint32_t), ctx->stream));
  k_label_roots<<<l_grid(g.n), L_THREADS, 0, ctx->stream>>>(g.n, und, ws.label, scc_id, rotation, q[0], qc[0], ws.ctr + CTR_DECIDED);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  read_counters(ctx);
  uint32_t decided = ctx->h_ctr[CTR_DECIDED];
  cur              = 0;
  for (uint32_t level = 0; ctx->h_ctr[CTR_Q0 + cur] > 0; ++level) {
    if (level >= cap) throw error{ KSPN_ERR_TIMEOUT, "label search: closure cap exceeded" };
    int const nxt = cur ^ 1;
    KSPN_CUDA(cudaMemsetAsync(qc[nxt], 0, sizeof(uint32_t), ctx->stream));
    uint32_t const fq = ctx->h_ctr[CTR_Q0 + cur];
    uint64_t const eb = ctx->h_ctr64[0];
    expand_level(ctx, g.bh, g.bc, q[cur], qc[cur], ws.ctr + CTR_NTILES, edges, ws.tile_start, q[nxt], qc[nxt], label_bw_op{ und, ws.label, scc_id, rotation });
    read_counters(ctx);
    uint32_t const pushed = ctx->h_ctr[CTR_Q0 + nxt];
    decided += pushed;
    prof_add(ctx, 0, KSPN_KERNEL_EXPAND, expand_bytes(fq, ctx->h_ctr64[0] - eb, pushed, 4));
    cur = nxt;
  }
  if (st) st->label_calls += 1;
  return decided;
}

} // namespace kspn
