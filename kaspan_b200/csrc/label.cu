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
//
// Learned seed order (kspn_options.learned_seeds, no reference
// counterpart): map(v) = bucket(v) << s | (v ^ mask), where s bits hold a
// vertex id, bucket(v) ranks the pivot model's score (a higher score, a
// smaller bucket, so the vertex wins the min-label propagation) and mask
// varies the order inside a bucket from call to call as the rotation does.
// map is injective on [0, n) and never UNDECIDED, so the fixpoint, the
// roots and the partition are those of any other seed order.
#include "expand.cuh"
#include "mlp.cuh"

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

// A search's seed order: the reference's rotated ids, or the learned order.
struct seed_map
{
  uint32_t const* bucket; // null: rotr(v, rot)
  int             rot;
  uint32_t        shift;  // id bits of a learned label
  uint32_t        mask;   // xor of the id bits (this call's order inside a bucket)
  __device__ __forceinline__ uint32_t map(uint32_t v) const { return bucket ? (__ldg(bucket + v) << shift) | (v ^ mask) : rotr32(v, rot); }
  __device__ __forceinline__ uint32_t unmap(uint32_t l) const { return bucket ? (l & ((1u << shift) - 1u)) ^ mask : rotl32(l, rot); }
};

// The pivot model's score of every undecided vertex as a bucket in
// [0, nbuckets - 1): sigmoid(logit) high -> bucket low.  One warp per vertex
// (the features sample its rows); the top bucket stays unused, so no label
// is UNDECIDED.
__global__ void __launch_bounds__(L_THREADS)
k_seed_buckets(uint32_t n, uint32_t const* __restrict__ und, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint64_t const* __restrict__ bh,
               uint32_t const* __restrict__ bc, float const* __restrict__ params, uint32_t nbuckets, uint32_t* __restrict__ bucket)
{
  unsigned const lane  = threadIdx.x & 31u;
  uint32_t const words = (n + 31) / 32;
  uint32_t const gw    = (blockIdx.x * L_THREADS + threadIdx.x) >> 5;
  uint32_t const nw    = (gridDim.x * L_THREADS) >> 5;
  // a warp takes 32 words at once (one per lane, one coalesced load), then
  // scores the set bits of the non-empty ones, one vertex at a time
  for (uint32_t wb = gw * 32; wb < words; wb += nw * 32) {
    uint32_t const w  = wb + lane;
    uint32_t       mw = w < words ? und[w] : 0u;
    if (w == words - 1 && (n & 31)) mw &= (1u << (n & 31)) - 1u;
    for (unsigned todo = __ballot_sync(0xFFFFFFFFu, mw != 0); todo; todo &= todo - 1) {
      unsigned const src  = __ffs(todo) - 1;
      uint32_t       word = __shfl_sync(0xFFFFFFFFu, mw, src);
      while (word) {
        uint32_t const v = (wb + src) * 32 + (__ffs(word) - 1);
        word &= word - 1;
        float f[MLP_IN], h1, h2;
        mlp_features(v, fh, fc, bh, bc, f);
        float const z = mlp_forward_w(mlp_weights_global{ params }, f, h1, h2);
        if (lane == 0) {
          float const    p = 1.f / (1.f + expf(-z));
          float const    q = (1.f - p) * static_cast<float>(nbuckets - 1);
          uint32_t const b = q >= static_cast<float>(nbuckets - 2) ? nbuckets - 2 : (q > 0.f ? static_cast<uint32_t>(q) : 0u);
          bucket[v]        = b;
        }
      }
    }
  }
}

// label = map(v) for undecided v (all queued), UNDECIDED otherwise.
__global__ void __launch_bounds__(L_THREADS)
k_label_init(uint32_t n, uint32_t const* __restrict__ und, uint32_t* __restrict__ label, seed_map sm, uint32_t* __restrict__ q, uint32_t* __restrict__ qn)
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
    if (t < n) label[v] = live ? sm.map(v) : UNDECIDED;
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
k_label_roots(uint32_t n, uint32_t* __restrict__ und, uint32_t const* __restrict__ label, uint32_t* __restrict__ scc_id, seed_map sm, uint32_t* __restrict__ q, uint32_t* __restrict__ qn, uint32_t* __restrict__ decided)
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
    bool const     root = t < n && bit_get(und, v) && label[v] == sm.map(v);
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
  seed_map        sm;
  // u = decided vertex, v = one of its in-neighbours; every push is a decision
  __device__ __forceinline__ uint32_t probe(uint32_t v) const { return und[v >> 5]; }
  __device__ __forceinline__ bool     operator()(uint32_t u, uint32_t v, bool valid, uint32_t word) const
  {
    if (!valid || !((word >> (v & 31)) & 1u)) return false;
    uint32_t const lu = label[u];
    if (label[v] != lu || !bit_take(und, v)) return false;
    scc_id[v] = sm.unmap(lu);
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

  seed_map sm{ nullptr, rotation, 0, 0 };
  if (opt.learned_seeds && ctx->pivot_model && g.n > 0 && g.n <= (1u << 31)) {
    // the learned order: every undecided vertex scored once per call
    uint32_t const shift = std::max<uint32_t>(1u, static_cast<uint32_t>(32 - __builtin_clz(g.n - 1 | 1u)));
    auto* const    bk    = static_cast<uint32_t*>(context_buffer(ctx, BUF_SEEDS, static_cast<size_t>(g.n) * 4));
    k_seed_buckets<<<l_grid(g.n / 8 + 1), L_THREADS, 0, ctx->stream>>>(g.n, und, g.fh, g.fc, g.bh, g.bc, ctx->pivot_model, 1u << (32 - shift), bk);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 1;
    sm = seed_map{ bk, rotation, shift, (static_cast<uint32_t>(rotation) * 0x9E3779B9u) & ((1u << shift) - 1u) };
  }
  zero_counters(ctx);
  KSPN_CUDA(cudaMemsetAsync(ws.vis_a, 0, words * 4, ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(ws.vis_b, 0, words * 4, ctx->stream));
  k_label_init<<<l_grid(g.n), L_THREADS, 0, ctx->stream>>>(g.n, und, ws.label, sm, q[0], qc[0]);
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
  k_label_roots<<<l_grid(g.n), L_THREADS, 0, ctx->stream>>>(g.n, und, ws.label, scc_id, sm, q[0], qc[0], ws.ctr + CTR_DECIDED);
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
    expand_level(ctx, g.bh, g.bc, q[cur], qc[cur], ws.ctr + CTR_NTILES, edges, ws.tile_start, q[nxt], qc[nxt], label_bw_op{ und, ws.label, scc_id, sm });
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
