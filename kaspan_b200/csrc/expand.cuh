// Load-balanced frontier expansion (top-down step of reachability and label
// propagation).
//
// A level expands every edge of every queued vertex exactly once:
//   1. k_fs_reduce / k_fs_partials / k_fs_down: exclusive scan of the
//      queued vertices' degrees (prefix[i]) over a fixed grid that reads the
//      queue length from device memory, so a level never waits on the host
//      to size a launch.  k_fs_down also records, for every tile of
//      EX_TILE consecutive edges, the queue index whose row holds the tile's
//      first edge (tile_start[]).
//   2. k_expand: a persistent grid walks the tiles.  Per tile, the rows that
//      start inside it are flagged and a block max-scan gives every edge
//      slot its row, so hub rows are split across blocks and low-degree rows
//      are packed densely; neighbour ids are read coalesced.
// The per-edge operation is a functor called by every lane of the warp
// (with valid == false for padding lanes) so it may use warp-wide pushes;
// its probe(v) (one state word) is loaded for a batch of slots ahead.
#pragma once

#include "prim.cuh"

namespace kspn {

constexpr int FS_BLOCKS  = 296;
constexpr int FS_THREADS = 512;
constexpr int FS_ITEMS   = 8;
constexpr int FS_SUB     = FS_THREADS * FS_ITEMS;

constexpr int EX_THREADS = 256;
constexpr int EX_ITEMS   = 8;
constexpr int EX_TILE    = EX_THREADS * EX_ITEMS;
constexpr int EX_BLOCKS  = 148 * 8;

// Frontier in/out queues.  With cur == nullptr (host-driven levels) the
// input is (q0, n0) and the output (q1, n1); inside a device-driven loop
// `cur` selects which pair is the input this level, so a captured graph can
// alternate queues without host involvement.
struct fio
{
  uint32_t*       q0;
  uint32_t*       q1;
  uint32_t*       n0;
  uint32_t*       n1;
  uint32_t const* cur;
  __device__ __forceinline__ bool            sw() const { return cur && (*cur & 1u); }
  __device__ __forceinline__ uint32_t const* in() const { return sw() ? q1 : q0; }
  __device__ __forceinline__ uint32_t        in_n() const { return sw() ? *n1 : *n0; }
  __device__ __forceinline__ uint32_t*       out() const { return sw() ? q0 : q1; }
  __device__ __forceinline__ uint32_t*       out_n() const { return sw() ? n0 : n1; }
};

// A kernel whose gate is closed returns at once (device-chosen direction).
struct gate
{
  uint32_t const* word;
  uint32_t        want;
  __device__ __forceinline__ bool closed() const { return word && *word != want; }
};

__device__ __forceinline__ void
fs_chunk(uint32_t qn, uint32_t& beg, uint32_t& end)
{
  uint32_t const chunk = (qn + FS_BLOCKS - 1) / FS_BLOCKS;
  uint64_t const b     = static_cast<uint64_t>(blockIdx.x) * chunk;
  beg                  = static_cast<uint32_t>(b < qn ? b : qn);
  uint64_t const e     = b + chunk;
  end                  = static_cast<uint32_t>(e < qn ? e : qn);
}

static __global__ void __launch_bounds__(FS_THREADS)
k_fs_reduce(uint64_t const* __restrict__ head, fio f, uint64_t* __restrict__ partial, gate g)
{
  if (g.closed()) return;
  uint32_t const* q = f.in();
  uint32_t        beg, end;
  fs_chunk(f.in_n(), beg, end);
  uint64_t s = 0;
  for (uint32_t i = beg + threadIdx.x; i < end; i += FS_THREADS) {
    uint32_t const v = q[i];
    s += head[v + 1] - head[v];
  }
  uint64_t total;
  block_exclusive_scan<uint64_t, FS_THREADS>(s, &total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

// prefix[qn] = total; *ntiles = tiles; *edges += total (nullable);
// *last = total (nullable).
static __global__ void __launch_bounds__(1024)
k_fs_partials(uint64_t* __restrict__ partial, uint64_t* __restrict__ prefix, fio f, uint32_t* __restrict__ ntiles, unsigned long long* __restrict__ edges, unsigned long long* __restrict__ last, gate g)
{
  if (g.closed()) return;
  uint64_t const v = threadIdx.x < FS_BLOCKS ? partial[threadIdx.x] : 0;
  uint64_t       total;
  uint64_t const pre = block_exclusive_scan<uint64_t, 1024>(v, &total);
  if (threadIdx.x < FS_BLOCKS) partial[threadIdx.x] = pre;
  if (threadIdx.x == 0) {
    prefix[f.in_n()] = total;
    *ntiles          = static_cast<uint32_t>((total + EX_TILE - 1) / EX_TILE);
    if (edges) *edges += total;
    if (last) *last = total;
  }
}

static __global__ void __launch_bounds__(FS_THREADS)
k_fs_down(uint64_t const* __restrict__ head, fio f, uint64_t const* __restrict__ partial, uint64_t* __restrict__ prefix, uint32_t* __restrict__ tile_start, gate g)
{
  if (g.closed()) return;
  uint32_t const* q = f.in();
  uint32_t        beg, end;
  fs_chunk(f.in_n(), beg, end);
  uint64_t run = partial[blockIdx.x];
  for (uint32_t base = beg; base < end; base += FS_THREADS) {
    uint32_t const i   = base + threadIdx.x;
    uint64_t       deg = 0;
    if (i < end) {
      uint32_t const v = q[i];
      deg              = head[v + 1] - head[v];
    }
    uint64_t       total;
    uint64_t const p = run + block_exclusive_scan<uint64_t, FS_THREADS>(deg, &total);
    if (i < end) {
      prefix[i] = p;
      if (deg) {
        // tiles whose first edge lies in [p, p + deg)
        uint64_t const t0 = (p + EX_TILE - 1) / EX_TILE;
        uint64_t const t1 = (p + deg - 1) / EX_TILE;
        for (uint64_t t = t0; t <= t1; ++t) tile_start[t] = i;
      }
    }
    run += total;
  }
}

// Inclusive max-scan of s[0, EX_TILE) in place (EX_THREADS threads, each
// owning EX_ITEMS consecutive slots).
__device__ __forceinline__ void
tile_max_scan(uint32_t* s)
{
  __shared__ uint32_t warp_max[EX_THREADS / 32];
  unsigned const      t = threadIdx.x, lane = t & 31u, w = t >> 5;
  uint32_t            v[EX_ITEMS];
  uint32_t            m = 0;
#pragma unroll
  for (int k = 0; k < EX_ITEMS; ++k) {
    v[k] = s[t * EX_ITEMS + k];
    m    = max(m, v[k]);
    v[k] = m;
  }
  uint32_t x = m;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= static_cast<unsigned>(d)) x = max(x, y);
  }
  if (lane == 31) warp_max[w] = x;
  __syncthreads();
  uint32_t carry = 0;
  for (unsigned k = 0; k < w; ++k) carry = max(carry, warp_max[k]);
  uint32_t const excl = max(carry, __shfl_up_sync(0xFFFFFFFFu, x, 1) * (lane > 0));
#pragma unroll
  for (int k = 0; k < EX_ITEMS; ++k) s[t * EX_ITEMS + k] = max(v[k], excl);
  __syncthreads();
}

// Expands tile `tile` of a scanned queue (ntiles tiles, total edges):
// calls op on every edge slot of items [k_begin, k_end) (slot = item *
// EX_THREADS + thread) and appends the winners to bq.  All threads of the
// block call it.  Queue, prefix and tile starts are read through L2 (ld.cg):
// inside a persistent launch other blocks wrote them.
// s_j: EX_TILE words of shared memory; s_i: two words.
// Slots are processed EX_BATCH at a time, each stage's loads for all of
// them issued before any is used: row lookup, neighbour id, the op's state
// probe (op.probe(v)), then op(u, v, valid, probed_word).
constexpr int EX_BATCH = 4;

template<typename Op>
__device__ __forceinline__ void
expand_tile(uint32_t tile, uint32_t ntiles, uint32_t const* q, uint32_t qn, uint64_t total, uint64_t const* prefix, uint32_t const* tile_start, uint64_t const* __restrict__ head,
            uint32_t const* __restrict__ adj, uint32_t* s_j, uint32_t* s_i, block_queue& bq, Op const& op, int k_begin = 0, int k_end = EX_ITEMS,
            uint32_t* s_q = nullptr, uint64_t* s_p = nullptr)
{
  uint64_t const t0 = static_cast<uint64_t>(tile) * EX_TILE;
  uint64_t const t1 = t0 + EX_TILE < total ? t0 + EX_TILE : total;
  if (threadIdx.x == 0) {
    s_i[0] = __ldcg(tile_start + tile);
    s_i[1] = tile + 1 < ntiles ? __ldcg(tile_start + tile + 1) : qn - 1;
  }
#pragma unroll
  for (int k = 0; k < EX_ITEMS; ++k) s_j[k * EX_THREADS + threadIdx.x] = 0;
  __syncthreads();
  uint32_t const i0 = s_i[0], i1 = s_i[1];
  for (uint32_t j = i0 + 1 + threadIdx.x; j <= i1; j += EX_THREADS) {
    uint64_t const p = __ldcg(prefix + j);
    if (p < t1) atomicMax(&s_j[p - t0], j - i0);
  }
  __syncthreads();
  tile_max_scan(s_j);
  // the tile's frontier rows (queue entries and edge prefixes) staged in
  // shared memory when they fit (<= 512 rows): every slot's row lookup is
  // then a shared-memory read instead of two L2 reads
  bool const staged = s_q && i1 - i0 + 1 <= 512;
  if (staged) {
    for (uint32_t r = threadIdx.x; r <= i1 - i0; r += EX_THREADS) s_q[r] = __ldcg(q + i0 + r), s_p[r] = __ldcg(prefix + i0 + r);
    __syncthreads();
  }
  for (int k0 = k_begin; k0 < k_end; k0 += EX_BATCH) {
    uint32_t u[EX_BATCH], v[EX_BATCH], w[EX_BATCH];
    uint64_t idx[EX_BATCH];
    bool     ok[EX_BATCH];
#pragma unroll
    for (int h = 0; h < EX_BATCH; ++h) {
      uint32_t const slot = (k0 + h) * EX_THREADS + threadIdx.x;
      uint64_t const e    = t0 + slot;
      ok[h]               = k0 + h < k_end && e < t1;
      u[h]                = 0;
      idx[h]              = 0;
      if (ok[h]) {
        uint32_t const j  = i0 + s_j[slot];
        u[h]              = staged ? s_q[j - i0] : __ldcg(q + j);
        uint64_t const pj = staged ? s_p[j - i0] : __ldcg(prefix + j);
        ok[h]             = e >= pj;
        idx[h]            = e - pj; // offset in u's row
      }
    }
#pragma unroll
    for (int h = 0; h < EX_BATCH; ++h)
      if (ok[h]) {
        // the slot's edge lies in u's row by construction of prefix and
        // tile_start; a slot that does not is skipped, never read
        uint64_t const b = head[u[h]];
        ok[h]            = idx[h] < head[u[h] + 1] - b;
        idx[h] += b;
      }
#pragma unroll
    for (int h = 0; h < EX_BATCH; ++h) v[h] = ok[h] ? adj[idx[h]] : 0u;
#pragma unroll
    for (int h = 0; h < EX_BATCH; ++h) w[h] = ok[h] ? op.probe(v[h]) : 0u;
#pragma unroll
    for (int h = 0; h < EX_BATCH; ++h) bq.push(op(u[h], v[h], ok[h], w[h]), v[h]);
  }
}

// op(u, v, valid, word) -> bool: u = source (queued vertex), v = neighbour,
// word = op.probe(v) (the op's state word of v, loaded ahead); true appends
// v to the output queue.  Called by every lane (valid == false on padding
// lanes).
template<typename Op>
__global__ void __launch_bounds__(EX_THREADS)
k_expand(uint64_t const* __restrict__ head,
         uint32_t const* __restrict__ adj,
         fio f,
         uint64_t const* __restrict__ prefix,
         uint32_t const* __restrict__ tile_start,
         uint32_t const* __restrict__ ntiles_ptr,
         gate g,
         Op op)
{
  if (g.closed()) return;
  __shared__ uint32_t s_j[EX_TILE];
  __shared__ uint32_t s_out[EX_TILE];
  __shared__ uint32_t s_i[2], s_n, s_base;
  uint32_t const*     q      = f.in();
  uint32_t* const     qout   = f.out();
  uint32_t* const     qout_n = f.out_n();
  uint32_t const      qn     = f.in_n();
  uint32_t const      ntiles = *ntiles_ptr;
  uint64_t const      total  = prefix[qn];
  if (threadIdx.x == 0) s_n = 0;
  block_queue bq{ s_out, &s_n };
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    expand_tile(tile, ntiles, q, qn, total, prefix, tile_start, head, adj, s_j, s_i, bq, op);
    bq.flush(qout, qout_n, &s_base);
  }
}

// Algorithmic bytes of one expansion: per queued vertex its queue entry and
// offset pair (4 + 16 B), per edge the neighbour id and one state probe
// (4 + 4 B), per vertex pushed to the next queue 4 B (+ `extra` per push).
inline uint64_t
expand_bytes(uint64_t frontier, uint64_t edges, uint64_t pushed, uint64_t extra_per_push = 0)
{
  return 20 * frontier + 8 * edges + (4 + extra_per_push) * pushed;
}

// Host: one top-down level over queue q (length at qn_dev), partials /
// prefix / tile_start from the workspace.
// Scan of the queue's degrees (prefix, tile starts, tile count).  The edge
// total is added to *edges (nullable) and stored to *last (nullable).
inline void
frontier_scan(kspn_context* ctx, uint64_t const* head, fio f, uint32_t* ntiles_dev, unsigned long long* edges, unsigned long long* last, uint32_t* tile_start)
{
  auto&              ws = ctx->ws;
  cudaStream_t const s  = ctx->stream;
  gate const         open{ nullptr, 0 };
  k_fs_reduce<<<FS_BLOCKS, FS_THREADS, 0, s>>>(head, f, ws.blocks, open);
  k_fs_partials<<<1, 1024, 0, s>>>(ws.blocks, ws.prefix, f, ntiles_dev, edges, last, open);
  k_fs_down<<<FS_BLOCKS, FS_THREADS, 0, s>>>(head, f, ws.blocks, ws.prefix, tile_start, open);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 3;
}

// Expansion of a scanned queue; tiles_host bounds the grid (0: unknown,
// use the full persistent grid).
template<typename Op>
void
expand_scanned(kspn_context* ctx, uint64_t const* head, uint32_t const* adj, fio f, uint32_t* ntiles_dev, uint32_t* tile_start, uint64_t tiles_host, Op op)
{
  auto&          ws   = ctx->ws;
  unsigned const grid = tiles_host ? static_cast<unsigned>(tiles_host < EX_BLOCKS ? tiles_host : EX_BLOCKS) : EX_BLOCKS;
  prof_start(ctx);
  k_expand<Op><<<grid, EX_THREADS, 0, ctx->stream>>>(head, adj, f, ws.prefix, tile_start, ntiles_dev, gate{ nullptr, 0 }, op);
  prof_stop(ctx);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

// Host-driven level: input (q, *qn_in), output (qout, *qn_out).
template<typename Op>
void
expand_level(kspn_context* ctx, uint64_t const* head, uint32_t const* adj, uint32_t* q, uint32_t* qn_in, uint32_t* ntiles_dev, unsigned long long* edges_dev, uint32_t* tile_start, uint32_t* qout, uint32_t* qout_n, Op op)
{
  fio const f{ q, qout, qn_in, qout_n, nullptr };
  frontier_scan(ctx, head, f, ntiles_dev, edges_dev, nullptr, tile_start);
  expand_scanned(ctx, head, adj, f, ntiles_dev, tile_start, 0, op);
}

} // namespace kspn
