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
// (with valid == false for padding lanes) so it may use warp-wide pushes.
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

// counters used by an expansion (indices into a u32 device array)
struct ex_ctrs
{
  uint32_t const* qn;     // queue length (read)
  uint32_t*       ntiles; // written by k_fs_partials
  unsigned long long* edges; // running total of expanded edges (added)
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
k_fs_reduce(uint64_t const* __restrict__ head, uint32_t const* __restrict__ q, uint32_t const* __restrict__ qn_ptr, uint64_t* __restrict__ partial)
{
  uint32_t beg, end;
  fs_chunk(*qn_ptr, beg, end);
  uint64_t s = 0;
  for (uint32_t i = beg + threadIdx.x; i < end; i += FS_THREADS) {
    uint32_t const v = q[i];
    s += head[v + 1] - head[v];
  }
  uint64_t total;
  block_exclusive_scan<uint64_t, FS_THREADS>(s, &total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

static __global__ void __launch_bounds__(1024)
k_fs_partials(uint64_t* __restrict__ partial, uint64_t* __restrict__ prefix, uint32_t const* __restrict__ qn_ptr, uint32_t* __restrict__ ntiles, unsigned long long* __restrict__ edges)
{
  uint64_t const v = threadIdx.x < FS_BLOCKS ? partial[threadIdx.x] : 0;
  uint64_t       total;
  uint64_t const pre = block_exclusive_scan<uint64_t, 1024>(v, &total);
  if (threadIdx.x < FS_BLOCKS) partial[threadIdx.x] = pre;
  if (threadIdx.x == 0) {
    prefix[*qn_ptr] = total;
    *ntiles         = static_cast<uint32_t>((total + EX_TILE - 1) / EX_TILE);
    if (edges) *edges += total;
  }
}

static __global__ void __launch_bounds__(FS_THREADS)
k_fs_down(uint64_t const* __restrict__ head, uint32_t const* __restrict__ q, uint32_t const* __restrict__ qn_ptr, uint64_t const* __restrict__ partial, uint64_t* __restrict__ prefix, uint32_t* __restrict__ tile_start)
{
  uint32_t beg, end;
  fs_chunk(*qn_ptr, beg, end);
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

// op(u, v, valid): u = source (queued vertex), v = neighbour.
template<typename Op>
__global__ void __launch_bounds__(EX_THREADS)
k_expand(uint64_t const* __restrict__ head,
         uint32_t const* __restrict__ adj,
         uint32_t const* __restrict__ q,
         uint32_t const* __restrict__ qn_ptr,
         uint64_t const* __restrict__ prefix,
         uint32_t const* __restrict__ tile_start,
         uint32_t const* __restrict__ ntiles_ptr,
         Op op)
{
  __shared__ uint32_t s_j[EX_TILE];
  __shared__ uint32_t s_i0, s_i1;
  uint32_t const      qn     = *qn_ptr;
  uint32_t const      ntiles = *ntiles_ptr;
  uint64_t const      total  = prefix[qn];
  for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    uint64_t const t0 = static_cast<uint64_t>(tile) * EX_TILE;
    uint64_t const t1 = t0 + EX_TILE < total ? t0 + EX_TILE : total;
    if (threadIdx.x == 0) {
      s_i0 = tile_start[tile];
      s_i1 = tile + 1 < ntiles ? tile_start[tile + 1] : qn - 1;
    }
#pragma unroll
    for (int k = 0; k < EX_ITEMS; ++k) s_j[k * EX_THREADS + threadIdx.x] = 0;
    __syncthreads();
    uint32_t const i0 = s_i0, i1 = s_i1;
    for (uint32_t j = i0 + 1 + threadIdx.x; j <= i1; j += EX_THREADS) {
      uint64_t const p = prefix[j];
      if (p < t1) atomicMax(&s_j[p - t0], j - i0);
    }
    __syncthreads();
    tile_max_scan(s_j);
#pragma unroll 2
    for (int k = 0; k < EX_ITEMS; ++k) {
      uint32_t const slot  = k * EX_THREADS + threadIdx.x;
      uint64_t const e     = t0 + slot;
      bool const     valid = e < t1;
      uint32_t       u = 0, v = 0;
      if (valid) {
        uint32_t const j = i0 + s_j[slot];
        u                = q[j];
        v                = adj[head[u] + (e - prefix[j])];
      }
      op(u, v, valid);
    }
    __syncthreads();
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
template<typename Op>
void
expand_level(kspn_context* ctx, uint64_t const* head, uint32_t const* adj, uint32_t const* q, uint32_t const* qn_dev, uint32_t* ntiles_dev, unsigned long long* edges_dev, uint32_t* tile_start, Op op)
{
  auto&              ws = ctx->ws;
  cudaStream_t const s  = ctx->stream;
  k_fs_reduce<<<FS_BLOCKS, FS_THREADS, 0, s>>>(head, q, qn_dev, ws.blocks);
  k_fs_partials<<<1, 1024, 0, s>>>(ws.blocks, ws.prefix, qn_dev, ntiles_dev, edges_dev);
  k_fs_down<<<FS_BLOCKS, FS_THREADS, 0, s>>>(head, q, qn_dev, ws.blocks, ws.prefix, tile_start);
  prof_start(ctx);
  k_expand<Op><<<EX_BLOCKS, EX_THREADS, 0, s>>>(head, adj, q, qn_dev, ws.prefix, tile_start, ntiles_dev, op);
  prof_stop(ctx);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 4;
}

} // namespace kspn
