// Device-wide primitives used by several kspn phases: block and grid
// exclusive scans over a value functor.  Reduce-then-scan, three launches:
//   1. per-block sums        2. scan of the block sums (one block)
//   3. per-block rescan with the block's base, out[count] = total
#pragma once

#include "kspn_internal.cuh"

namespace kspn {

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS   = 8;
constexpr int SCAN_TILE    = SCAN_THREADS * SCAN_ITEMS;

// Exclusive scan of one value per thread across the block; returns the
// thread's prefix, *total = block sum.  All threads must call it.
template<typename T, int THREADS>
__device__ __forceinline__ T
block_exclusive_scan(T v, T* total)
{
  __shared__ T warp_sums[THREADS / 32];
  unsigned const lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  T              x    = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T const y = __shfl_up_sync(0xFFFFFFFFu, x, d);
    if (lane >= static_cast<unsigned>(d)) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T w = (lane < THREADS / 32) ? warp_sums[lane] : T(0);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      T const y = __shfl_up_sync(0xFFFFFFFFu, w, d);
      if (lane >= static_cast<unsigned>(d)) w += y;
    }
    if (lane < THREADS / 32) warp_sums[lane] = w; // inclusive
  }
  __syncthreads();
  T const base = warp ? warp_sums[warp - 1] : T(0);
  *total       = warp_sums[THREADS / 32 - 1];
  __syncthreads(); // warp_sums reusable by the next call
  return base + x - v;
}

template<typename T, typename F>
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_reduce(F f, uint64_t count, T* partial)
{
  uint64_t const base = static_cast<uint64_t>(blockIdx.x) * SCAN_TILE;
  T              s    = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    uint64_t const i = base + static_cast<uint64_t>(k) * SCAN_THREADS + threadIdx.x;
    if (i < count) s += f(i);
  }
  T total;
  block_exclusive_scan<T, SCAN_THREADS>(s, &total);
  if (threadIdx.x == 0) partial[blockIdx.x] = total;
}

template<typename T>
__global__ void __launch_bounds__(1024)
k_scan_partials(T* partial, uint32_t nb)
{
  // each thread owns a contiguous run of the block sums
  uint32_t const per = (nb + 1023) / 1024;
  uint32_t const beg = threadIdx.x * per;
  uint32_t const end = min(nb, beg + per);
  T              s   = 0;
  for (uint32_t i = beg; i < end; ++i) s += partial[i];
  T       total;
  T const pre = block_exclusive_scan<T, 1024>(s, &total);
  T       run = pre;
  for (uint32_t i = beg; i < end; ++i) {
    T const v  = partial[i];
    partial[i] = run;
    run += v;
  }
  if (threadIdx.x == 0) partial[nb] = total;
}

template<typename T, typename F>
__global__ void __launch_bounds__(SCAN_THREADS)
k_scan_down(F f, uint64_t count, T const* partial, T* out)
{
  // blocked arrangement: thread t owns items [t*ITEMS, (t+1)*ITEMS) of the tile
  uint64_t const base = static_cast<uint64_t>(blockIdx.x) * SCAN_TILE + static_cast<uint64_t>(threadIdx.x) * SCAN_ITEMS;
  T              v[SCAN_ITEMS];
  T              s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    uint64_t const i = base + k;
    v[k]             = (i < count) ? f(i) : T(0);
    s += v[k];
  }
  T total;
  T run = block_exclusive_scan<T, SCAN_THREADS>(s, &total) + partial[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    uint64_t const i = base + k;
    if (i < count) out[i] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[count] = partial[gridDim.x];
}

// out[i] = sum_{j<i} f(j) for i in [0, count], out[count] = total.
// partial must hold div_up(count, SCAN_TILE) + 1 entries.
template<typename T, typename F>
void
exclusive_scan(cudaStream_t s, F f, uint64_t count, T* out, T* partial, uint64_t* launches)
{
  if (count == 0) {
    KSPN_CUDA(cudaMemsetAsync(out, 0, sizeof(T), s));
    return;
  }
  unsigned const nb = div_up(count, SCAN_TILE);
  k_scan_reduce<T><<<nb, SCAN_THREADS, 0, s>>>(f, count, partial);
  k_scan_partials<T><<<1, 1024, 0, s>>>(partial, nb);
  k_scan_down<T><<<nb, SCAN_THREADS, 0, s>>>(f, count, partial, out);
  KSPN_CHECK_LAUNCH();
  if (launches) *launches += 3;
}

inline size_t
scan_partial_entries(uint64_t count)
{
  return div_up(count ? count : 1, SCAN_TILE) + 1;
}

// functors
struct f_array_u32
{
  uint32_t const* a;
  __device__ uint64_t operator()(uint64_t i) const { return a[i]; }
};
struct f_array_u32_as_u32
{
  uint32_t const* a;
  __device__ uint32_t operator()(uint64_t i) const { return a[i]; }
};
struct f_frontier_degree
{
  uint64_t const* head;
  uint32_t const* q;
  __device__ uint64_t operator()(uint64_t i) const
  {
    uint32_t const v = q[i];
    return head[v + 1] - head[v];
  }
};

// radix.cu: stable LSD radix sort of (key, value) u32 pairs on key bits
// [begin_bit, end_bit).  The result ends in keys/vals; keys_alt/vals_alt
// are scratch of the same size.  hist needs radix_hist_entries(count).
size_t radix_hist_entries(uint64_t count);
void   radix_sort_pairs(kspn_context* ctx, uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, uint64_t count, int begin_bit, int end_bit, uint32_t* hist, uint32_t* hist_partial);
// The same sort on key bits [0, end_bit) from read-only input (kin, vin) to
// (kout, vout); (ka, va) and (kb, vb) are scratch of `count` entries each
// (neither may alias the input or the output).
void   radix_sort_pairs_to(kspn_context* ctx, uint32_t const* kin, uint32_t const* vin, uint32_t* kout, uint32_t* vout, uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, uint64_t count, int end_bit, uint32_t* hist, uint32_t* hist_partial);

inline int
bits_for(uint64_t n) // bits needed to represent ids in [0, n)
{
  int b = 0;
  while ((1ull << b) < n) ++b;
  return b;
}

} // namespace kspn
