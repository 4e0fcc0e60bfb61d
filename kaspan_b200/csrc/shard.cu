// One graph sharded over several GPUs: the device steps of one shard.
//
// Reference: the distributed kaspan::scc (kaspan/scc/scc.hpp:21-87) runs on
// a 1D vertex partition -- rank r owns the contiguous vertex range [lo, hi)
// and its rows of the forward CSR and of the transpose, neighbour ids
// global (kaspan/graph/bidi_graph_part.hpp:12-28,
// kaspan/graph/explicit_continuous_part.hpp); the forward and backward
// searches exchange frontier messages between ranks every iteration
// (frontier::comm, kaspan/scc/frontier.hpp:237-282: an all-to-all of the
// counts, then of the payload) and every phase ends with an all-reduce of
// the decided count (kaspan/util/mpi_basic.hpp).  These entry points are
// one rank's device work between those exchanges; kaspan_b200/shard.py
// drives them and runs the exchanges (torch.distributed, NCCL between GPUs).
//
// Shard layout on the device: n_loc = hi - lo local vertices; fw_head /
// bw_head u64[n_loc + 1] local offsets; fw_csr / bw_csr u32 GLOBAL ids;
// local state as bitmaps over the local range (bit v of word v/32 = local
// vertex v, i.e. global vertex lo + v); scc_id[n_loc] global ids.
#include "kspn_internal.cuh"
#include "prim.cuh"

#include <vector>

namespace kspn {

namespace {

constexpr int SH_THREADS = 256;

unsigned
sh_grid(uint64_t items)
{
  uint64_t const b = (items + SH_THREADS - 1) / SH_THREADS;
  return static_cast<unsigned>(b < 148ull * 8 ? (b ? b : 1) : 148ull * 8);
}

// Counters of one step (a 64-byte slot of ws.ctr is not used: the shard
// steps own their own small device block, shard_ctr below).
struct shard_ctr
{
  unsigned long long best_prod; // trim_1_first / pivot: largest in * out
  uint32_t           best_id;   // ... and its smallest global id
  uint32_t           decided;
  uint32_t           next_n;    // local frontier entries appended
  uint32_t           remote_n;  // remote ids appended
  uint32_t           min_id;    // smallest SCC member
  uint32_t           err;       // a list would have overflowed
  uint32_t           res_n;     // residual edges (low word) ...
  uint32_t           res_hi;    // ... high word
};

// trim_1_first on the local rows (kaspan/scc/trim_1_local.hpp:12-46): a
// local vertex with no in- or no out-edge is decided (id = its global id);
// und is written in full; the largest in * out of the rest goes to
// best_prod.  One warp per 32 local vertices (one und word).
__global__ void __launch_bounds__(SH_THREADS)
k_sh_trim_first(uint32_t n_loc, uint32_t lo, uint64_t const* __restrict__ fh, uint64_t const* __restrict__ bh, uint32_t* __restrict__ und, uint32_t* __restrict__ ids,
                shard_ctr* c)
{
  unsigned const lane  = threadIdx.x & 31u;
  uint32_t const words = (n_loc + 31) / 32;
  uint32_t       dec   = 0;
  unsigned long long best = 0;
  for (uint32_t w = (blockIdx.x * SH_THREADS + threadIdx.x) >> 5; w < words; w += (gridDim.x * SH_THREADS) >> 5) {
    uint32_t const v   = w * 32 + lane;
    bool           und_v = false;
    if (v < n_loc) {
      uint64_t const out = fh[v + 1] - fh[v], in = bh[v + 1] - bh[v];
      und_v              = out != 0 && in != 0;
      if (!und_v) ids[v] = lo + v, ++dec;
      else ids[v] = UNDECIDED;
      if (und_v && out * in > best) best = out * in;
    }
    unsigned const word = __ballot_sync(0xFFFFFFFFu, und_v);
    if (lane == 0) und[w] = word;
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) {
    unsigned long long const o = __shfl_xor_sync(0xFFFFFFFFu, best, sh);
    best                       = o > best ? o : best;
  }
  if (lane == 0 && best) atomicMax(&c->best_prod, best);
  dec = __reduce_add_sync(0xFFFFFFFFu, dec);
  if (lane == 0 && dec) atomicAdd(&c->decided, dec);
}

// Among the undecided local vertices whose in * out equals best_prod, the
// smallest global id (the reference's tie rule at one rank).
__global__ void __launch_bounds__(SH_THREADS)
k_sh_best_id(uint32_t n_loc, uint32_t lo, uint64_t const* __restrict__ fh, uint64_t const* __restrict__ bh, uint32_t const* __restrict__ und, shard_ctr* c)
{
  unsigned long long const best = c->best_prod;
  if (best == 0) return;
  for (uint32_t v = blockIdx.x * SH_THREADS + threadIdx.x; v < n_loc; v += gridDim.x * SH_THREADS)
    if (bit_get(und, v) && (fh[v + 1] - fh[v]) * (bh[v + 1] - bh[v]) == best) {
      atomicMin(&c->best_id, lo + v);
      break; // later vertices of this thread have larger ids
    }
}

// Largest in * out over the undecided local vertices (raw degrees, the
// reference's pivot rule on the remaining graph, kaspan/scc/pivot.hpp).
__global__ void __launch_bounds__(SH_THREADS)
k_sh_pivot(uint32_t n_loc, uint64_t const* __restrict__ fh, uint64_t const* __restrict__ bh, uint32_t const* __restrict__ und, shard_ctr* c)
{
  unsigned long long best = 0;
  for (uint32_t v = blockIdx.x * SH_THREADS + threadIdx.x; v < n_loc; v += gridDim.x * SH_THREADS)
    if (bit_get(und, v)) {
      unsigned long long const p = (fh[v + 1] - fh[v]) * (bh[v + 1] - bh[v]);
      if (p > best) best = p;
    }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) {
    unsigned long long const o = __shfl_xor_sync(0xFFFFFFFFu, best, sh);
    best                       = o > best ? o : best;
  }
  if ((threadIdx.x & 31u) == 0 && best) atomicMax(&c->best_prod, best);
}

// Search start: cand = und, vis = 0 for both searches, sent = 0.
__global__ void __launch_bounds__(SH_THREADS)
k_sh_search_init(uint32_t words, uint32_t gwords, uint32_t const* __restrict__ und, uint32_t* __restrict__ cand_f, uint32_t* __restrict__ cand_b, uint32_t* __restrict__ vis_f,
                 uint32_t* __restrict__ vis_b, uint32_t* __restrict__ sent_f, uint32_t* __restrict__ sent_b)
{
  for (uint32_t w = blockIdx.x * SH_THREADS + threadIdx.x; w < words; w += gridDim.x * SH_THREADS) {
    uint32_t const u = und[w];
    cand_f[w] = cand_b[w] = u;
    vis_f[w] = vis_b[w] = 0;
  }
  for (uint32_t w = blockIdx.x * SH_THREADS + threadIdx.x; w < gwords; w += gridDim.x * SH_THREADS) sent_f[w] = sent_b[w] = 0;
}

// Takes local vertex v (global lo + v) into the search: bit taken from
// cand, set in vis, appended to next.  All lanes call it.
__device__ __forceinline__ void
sh_take(bool pred, uint32_t v, uint32_t* cand, uint32_t* vis, uint32_t* next, uint32_t cap, shard_ctr* c)
{
  bool const     took   = pred && bit_take(cand, v);
  unsigned const ballot = __ballot_sync(0xFFFFFFFFu, took);
  if (!ballot) return;
  unsigned const lane   = threadIdx.x & 31u;
  unsigned const leader = __ffs(ballot) - 1;
  uint32_t       base   = 0;
  if (lane == leader) base = atomicAdd(&c->next_n, static_cast<uint32_t>(__popc(ballot)));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  if (took) {
    bit_set_async(vis, v);
    uint32_t const at = base + __popc(ballot & ((1u << lane) - 1u));
    if (at < cap) next[at] = v;
    else atomicExch(&c->err, 1u);
  }
}

// One top-down level of one search over the local rows (head/adj: fw for
// the forward search, bw for the backward one): one warp per frontier
// vertex, lanes over its row.  A local neighbour is taken (sh_take); a
// remote one is claimed once per search in the global bitmap `sent` and
// appended to `remote` (global ids) for the exchange.
__global__ void __launch_bounds__(SH_THREADS)
k_sh_expand(uint32_t n_loc, uint32_t lo, uint64_t const* __restrict__ head, uint32_t const* __restrict__ adj, uint32_t const* __restrict__ fq, uint32_t fn, uint32_t* cand, uint32_t* vis,
            uint32_t* sent, uint32_t* next, uint32_t next_cap, uint32_t* remote, uint32_t remote_cap, shard_ctr* c)
{
  unsigned const lane = threadIdx.x & 31u;
  for (uint32_t i = (blockIdx.x * SH_THREADS + threadIdx.x) >> 5; i < fn; i += (gridDim.x * SH_THREADS) >> 5) {
    uint32_t const v = fq[i];
    uint64_t const b = head[v], e = head[v + 1];
    for (uint64_t x = b; x < e; x += 32) {
      bool const     in    = x + lane < e;
      uint32_t const u     = in ? adj[x + lane] : 0u;
      uint32_t const lu    = u - lo;
      bool const     local = in && lu < n_loc;
      sh_take(local && bit_get(cand, lu), lu, cand, vis, next, next_cap, c);
      bool const     rem    = in && !local && bit_claim(sent, u);
      unsigned const ballot = __ballot_sync(0xFFFFFFFFu, rem);
      if (ballot) {
        unsigned const leader = __ffs(ballot) - 1;
        uint32_t       base   = 0;
        if (lane == leader) base = atomicAdd(&c->remote_n, static_cast<uint32_t>(__popc(ballot)));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (rem) {
          uint32_t const at = base + __popc(ballot & ((1u << lane) - 1u));
          if (at < remote_cap) remote[at] = u;
          else atomicExch(&c->err, 1u);
        }
      }
    }
  }
}

// Owner of global id u: the shard whose [bounds[r], bounds[r+1]) holds it.
__device__ __forceinline__ uint32_t
sh_owner(uint32_t u, uint32_t const* bounds, uint32_t parts)
{
  uint32_t lo = 0, hi = parts; // bounds[lo] <= u < bounds[hi]
  while (hi - lo > 1) {
    uint32_t const mid = (lo + hi) / 2;
    if (bounds[mid] <= u) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Remote ids grouped by owner (counting sort): counts[parts], then out in
// owner order.  cursor[parts] are the running offsets (zeroed by the host).
__global__ void __launch_bounds__(SH_THREADS)
k_sh_count(uint32_t const* __restrict__ remote, uint32_t rn, uint32_t const* __restrict__ bounds, uint32_t parts, uint32_t* __restrict__ counts)
{
  for (uint32_t i = blockIdx.x * SH_THREADS + threadIdx.x; i < rn; i += gridDim.x * SH_THREADS) atomicAdd(counts + sh_owner(remote[i], bounds, parts), 1u);
}
__global__ void __launch_bounds__(SH_THREADS)
k_sh_scatter(uint32_t const* __restrict__ remote, uint32_t rn, uint32_t const* __restrict__ bounds, uint32_t parts, uint32_t* __restrict__ cursor, uint32_t* __restrict__ out)
{
  for (uint32_t i = blockIdx.x * SH_THREADS + threadIdx.x; i < rn; i += gridDim.x * SH_THREADS) {
    uint32_t const u = remote[i];
    out[atomicAdd(cursor + sh_owner(u, bounds, parts), 1u)] = u;
  }
}

// Ids received from the other shards (all in [lo, hi)): taken locally.
__global__ void __launch_bounds__(SH_THREADS)
k_sh_receive(uint32_t n_loc, uint32_t lo, uint32_t const* __restrict__ recv, uint32_t rn, uint32_t* cand, uint32_t* vis, uint32_t* next, uint32_t next_cap, shard_ctr* c)
{
  for (uint32_t i0 = (blockIdx.x * SH_THREADS + threadIdx.x) & ~31u; i0 < rn; i0 += gridDim.x * SH_THREADS) {
    uint32_t const i  = i0 + (threadIdx.x & 31u);
    uint32_t const lu = i < rn ? recv[i] - lo : n_loc;
    bool const     ok = lu < n_loc;
    if (i < rn && !ok) atomicExch(&c->err, 2u);
    sh_take(ok && bit_get(cand, lu), ok ? lu : 0u, cand, vis, next, next_cap, c);
  }
}

// Smallest global id in vis_f & vis_b (the pivot's SCC on this shard).
__global__ void __launch_bounds__(SH_THREADS)
k_sh_scc_min(uint32_t words, uint32_t lo, uint32_t const* __restrict__ vis_f, uint32_t const* __restrict__ vis_b, shard_ctr* c)
{
  for (uint32_t w = blockIdx.x * SH_THREADS + threadIdx.x; w < words; w += gridDim.x * SH_THREADS) {
    uint32_t const s = vis_f[w] & vis_b[w];
    if (s) {
      atomicMin(&c->min_id, lo + w * 32 + (__ffs(s) - 1));
      break; // later words of this thread hold larger ids
    }
  }
}

// The SCC's local members leave und with id `id`.
__global__ void __launch_bounds__(SH_THREADS)
k_sh_finalize(uint32_t n_loc, uint32_t const* __restrict__ vis_f, uint32_t const* __restrict__ vis_b, uint32_t* __restrict__ und, uint32_t* __restrict__ ids, uint32_t id, shard_ctr* c)
{
  uint32_t const words = (n_loc + 31) / 32;
  uint32_t       dec   = 0;
  for (uint32_t w = blockIdx.x * SH_THREADS + threadIdx.x; w < words; w += gridDim.x * SH_THREADS) {
    uint32_t const s = vis_f[w] & vis_b[w] & und[w];
    if (!s) continue;
    und[w] &= ~s;
    for (uint32_t x = s; x; x &= x - 1) ids[w * 32 + __ffs(x) - 1] = id;
    dec += __popc(s);
  }
  dec = __reduce_add_sync(0xFFFFFFFFu, dec);
  if ((threadIdx.x & 31u) == 0 && dec) atomicAdd(&c->decided, dec);
}

// Edges of the residual sub-graph leaving this shard's rows: (lo + v, u)
// for every undecided local v and out-neighbour u undecided in the global
// bitmap gund (word u/32 of the whole graph).  Counted into res_n/res_hi
// (64 bits); written when the count stays below cap.
__global__ void __launch_bounds__(SH_THREADS)
k_sh_residual(uint32_t n_loc, uint32_t lo, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint32_t const* __restrict__ und, uint32_t const* __restrict__ gund,
              uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint64_t cap, shard_ctr* c)
{
  auto* const cnt  = reinterpret_cast<unsigned long long*>(&c->res_n);
  unsigned const lane = threadIdx.x & 31u;
  for (uint32_t v = (blockIdx.x * SH_THREADS + threadIdx.x) >> 5; v < n_loc; v += (gridDim.x * SH_THREADS) >> 5) {
    if (!bit_get(und, v)) continue; // warp-uniform
    uint64_t const b = fh[v], e = fh[v + 1];
    for (uint64_t x = b; x < e; x += 32) {
      bool const     in     = x + lane < e;
      uint32_t const u      = in ? fc[x + lane] : 0u;
      bool const     keep   = in && bit_get(gund, u);
      unsigned const ballot = __ballot_sync(0xFFFFFFFFu, keep);
      if (!ballot) continue;
      unsigned const     leader = __ffs(ballot) - 1;
      unsigned long long base   = 0;
      if (lane == leader) base = atomicAdd(cnt, static_cast<unsigned long long>(__popc(ballot)));
      base = __shfl_sync(0xFFFFFFFFu, base, leader);
      if (keep) {
        uint64_t const at = base + __popc(ballot & ((1u << lane) - 1u));
        if (at < cap) src[at] = lo + v, dst[at] = u;
      }
    }
  }
}

} // namespace

} // namespace kspn

using namespace kspn;

namespace {

void
sh_need(bool ok, char const* what)
{
  if (!ok) throw error{ KSPN_ERR_INVALID_ARGUMENT, what };
}

// The step's counter block, zeroed (min_id / best_id start at UNDECIDED).
shard_ctr*
sh_begin(kspn_context* ctx)
{
  KSPN_CUDA(cudaSetDevice(ctx->device));
  auto* c = static_cast<shard_ctr*>(context_buffer(ctx, BUF_SHARD, sizeof(shard_ctr)));
  KSPN_CUDA(cudaMemsetAsync(c, 0, sizeof(shard_ctr), ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(&c->best_id, 0xFF, sizeof(uint32_t), ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(&c->min_id, 0xFF, sizeof(uint32_t), ctx->stream));
  return c;
}

shard_ctr
sh_end(kspn_context* ctx, shard_ctr const* c)
{
  KSPN_CHECK_LAUNCH();
  shard_ctr h{};
  KSPN_CUDA(cudaMemcpyAsync(&h, c, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h.err == 1) throw error{ KSPN_ERR_INVALID_ARGUMENT, "shard step: an output list is too short" };
  if (h.err == 2) throw error{ KSPN_ERR_INVALID_ARGUMENT, "shard step: a received id lies outside this shard" };
  return h;
}

} // namespace

extern "C" int
kspn_shard_trim_first(kspn_context* ctx, uint32_t n_loc, uint32_t lo, uint64_t const* d_fw_head, uint64_t const* d_bw_head, uint32_t* d_und, uint32_t* d_scc_id, uint64_t* best_prod,
                      uint32_t* best_id, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(n_loc == 0 || (d_fw_head && d_bw_head && d_und && d_scc_id), "null device pointer");
    shard_ctr* c = sh_begin(ctx);
    if (n_loc) {
      k_sh_trim_first<<<sh_grid(n_loc), SH_THREADS, 0, ctx->stream>>>(n_loc, lo, d_fw_head, d_bw_head, d_und, d_scc_id, c);
      k_sh_best_id<<<sh_grid(n_loc), SH_THREADS, 0, ctx->stream>>>(n_loc, lo, d_fw_head, d_bw_head, d_und, c);
      ctx->launches += 2;
    }
    shard_ctr const h = sh_end(ctx, c);
    if (best_prod) *best_prod = h.best_prod;
    if (best_id) *best_id = h.best_prod ? h.best_id : UNDECIDED;
    if (decided) *decided = h.decided;
  });
}

extern "C" int
kspn_shard_pivot(kspn_context* ctx, uint32_t n_loc, uint32_t lo, uint64_t const* d_fw_head, uint64_t const* d_bw_head, uint32_t const* d_und, uint64_t* best_prod, uint32_t* best_id)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(n_loc == 0 || (d_fw_head && d_bw_head && d_und), "null device pointer");
    shard_ctr* c = sh_begin(ctx);
    if (n_loc) {
      k_sh_pivot<<<sh_grid(n_loc), SH_THREADS, 0, ctx->stream>>>(n_loc, d_fw_head, d_bw_head, d_und, c);
      k_sh_best_id<<<sh_grid(n_loc), SH_THREADS, 0, ctx->stream>>>(n_loc, lo, d_fw_head, d_bw_head, d_und, c);
      ctx->launches += 2;
    }
    shard_ctr const h = sh_end(ctx, c);
    if (best_prod) *best_prod = h.best_prod;
    if (best_id) *best_id = h.best_prod ? h.best_id : UNDECIDED;
  });
}

extern "C" int
kspn_shard_search_begin(kspn_context* ctx, uint32_t n_loc, uint32_t n, uint32_t const* d_und, uint32_t* d_cand_fw, uint32_t* d_cand_bw, uint32_t* d_vis_fw, uint32_t* d_vis_bw,
                        uint32_t* d_sent_fw, uint32_t* d_sent_bw)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(d_und && d_cand_fw && d_cand_bw && d_vis_fw && d_vis_bw && d_sent_fw && d_sent_bw, "null device pointer");
    KSPN_CUDA(cudaSetDevice(ctx->device));
    uint32_t const words = (n_loc + 31) / 32, gwords = (n + 31) / 32;
    k_sh_search_init<<<sh_grid(gwords > words ? gwords : words), SH_THREADS, 0, ctx->stream>>>(words, gwords, d_und, d_cand_fw, d_cand_bw, d_vis_fw, d_vis_bw, d_sent_fw, d_sent_bw);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 1;
  });
}

extern "C" int
kspn_shard_expand(kspn_context* ctx, uint32_t n_loc, uint32_t lo, uint64_t const* d_head, uint32_t const* d_adj, uint32_t const* d_frontier, uint32_t frontier_n, uint32_t* d_cand,
                  uint32_t* d_vis, uint32_t* d_sent, uint32_t* d_next, uint32_t next_cap, uint32_t* next_n, uint32_t* d_remote, uint32_t remote_cap, uint32_t parts,
                  uint32_t const* d_bounds, uint32_t* d_send, uint32_t* d_counts, uint32_t* counts)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(next_n && counts && parts >= 1 && parts <= 1024, "bad argument");
    sh_need(frontier_n == 0 || (d_head && d_adj && d_frontier && d_cand && d_vis && d_sent && d_next && d_remote && d_bounds && d_send && d_counts), "null device pointer");
    shard_ctr* c = sh_begin(ctx);
    KSPN_CUDA(cudaMemcpyAsync(&c->next_n, next_n, sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    if (frontier_n) {
      k_sh_expand<<<sh_grid(static_cast<uint64_t>(frontier_n) * 32), SH_THREADS, 0, ctx->stream>>>(n_loc, lo, d_head, d_adj, d_frontier, frontier_n, d_cand, d_vis, d_sent, d_next, next_cap,
                                                                                                   d_remote, remote_cap, c);
      ctx->launches += 1;
    }
    shard_ctr const h = sh_end(ctx, c);
    *next_n           = h.next_n;
    // the remote ids grouped by owning shard
    KSPN_CUDA(cudaMemsetAsync(d_counts, 0, 2 * parts * sizeof(uint32_t), ctx->stream));
    if (h.remote_n) {
      k_sh_count<<<sh_grid(h.remote_n), SH_THREADS, 0, ctx->stream>>>(d_remote, h.remote_n, d_bounds, parts, d_counts);
      KSPN_CHECK_LAUNCH();
    }
    KSPN_CUDA(cudaMemcpyAsync(counts, d_counts, parts * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    if (h.remote_n) {
      std::vector<uint32_t> start(parts);
      uint32_t              run = 0;
      for (uint32_t r = 0; r < parts; ++r) start[r] = run, run += counts[r];
      KSPN_CUDA(cudaMemcpyAsync(d_counts + parts, start.data(), parts * sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
      k_sh_scatter<<<sh_grid(h.remote_n), SH_THREADS, 0, ctx->stream>>>(d_remote, h.remote_n, d_bounds, parts, d_counts + parts, d_send);
      KSPN_CHECK_LAUNCH();
      KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
      ctx->launches += 2;
    }
  });
}

extern "C" int
kspn_shard_receive(kspn_context* ctx, uint32_t n_loc, uint32_t lo, uint32_t const* d_recv, uint32_t recv_n, uint32_t* d_cand, uint32_t* d_vis, uint32_t* d_next, uint32_t next_cap,
                   uint32_t* next_n)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(next_n != nullptr, "bad argument");
    sh_need(recv_n == 0 || (d_recv && d_cand && d_vis && d_next), "null device pointer");
    shard_ctr* c = sh_begin(ctx);
    KSPN_CUDA(cudaMemcpyAsync(&c->next_n, next_n, sizeof(uint32_t), cudaMemcpyHostToDevice, ctx->stream));
    if (recv_n) {
      k_sh_receive<<<sh_grid(recv_n), SH_THREADS, 0, ctx->stream>>>(n_loc, lo, d_recv, recv_n, d_cand, d_vis, d_next, next_cap, c);
      ctx->launches += 1;
    }
    *next_n = sh_end(ctx, c).next_n;
  });
}

extern "C" int
kspn_shard_scc_min(kspn_context* ctx, uint32_t n_loc, uint32_t lo, uint32_t const* d_vis_fw, uint32_t const* d_vis_bw, uint32_t* min_id)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(min_id && (n_loc == 0 || (d_vis_fw && d_vis_bw)), "null pointer");
    shard_ctr* c     = sh_begin(ctx);
    uint32_t   words = (n_loc + 31) / 32;
    if (words) {
      k_sh_scc_min<<<sh_grid(words), SH_THREADS, 0, ctx->stream>>>(words, lo, d_vis_fw, d_vis_bw, c);
      ctx->launches += 1;
    }
    *min_id = sh_end(ctx, c).min_id;
  });
}

extern "C" int
kspn_shard_finalize(kspn_context* ctx, uint32_t n_loc, uint32_t const* d_vis_fw, uint32_t const* d_vis_bw, uint32_t* d_und, uint32_t* d_scc_id, uint32_t id, uint32_t* decided)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(n_loc == 0 || (d_vis_fw && d_vis_bw && d_und && d_scc_id), "null device pointer");
    shard_ctr* c = sh_begin(ctx);
    if (n_loc) {
      k_sh_finalize<<<sh_grid((n_loc + 31) / 32), SH_THREADS, 0, ctx->stream>>>(n_loc, d_vis_fw, d_vis_bw, d_und, d_scc_id, id, c);
      ctx->launches += 1;
    }
    uint32_t const d = sh_end(ctx, c).decided;
    if (decided) *decided = d;
  });
}

extern "C" int
kspn_shard_residual(kspn_context* ctx, uint32_t n_loc, uint32_t lo, uint64_t const* d_fw_head, uint32_t const* d_fw_csr, uint32_t const* d_und, uint32_t const* d_global_und,
                    uint32_t* d_src, uint32_t* d_dst, uint64_t cap, uint64_t* count)
{
  if (!ctx) return KSPN_ERR_INVALID_ARGUMENT;
  return run_guarded(ctx, [&] {
    sh_need(count != nullptr, "bad argument");
    sh_need(n_loc == 0 || (d_fw_head && d_fw_csr && d_und && d_global_und), "null device pointer");
    sh_need(cap == 0 || (d_src && d_dst), "null output");
    shard_ctr* c = sh_begin(ctx);
    if (n_loc) {
      k_sh_residual<<<sh_grid(static_cast<uint64_t>(n_loc) * 32), SH_THREADS, 0, ctx->stream>>>(n_loc, lo, d_fw_head, d_fw_csr, d_und, d_global_und, d_src, d_dst, cap, c);
      ctx->launches += 1;
    }
    shard_ctr const h = sh_end(ctx, c);
    *count            = static_cast<uint64_t>(h.res_n) | (static_cast<uint64_t>(h.res_hi) << 32);
  });
}
