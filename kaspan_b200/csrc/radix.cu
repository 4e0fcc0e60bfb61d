// Stable LSD radix sort of (u32 key, u32 value) pairs, 8-bit digits.
//
// One pass = histogram per 4096-key tile (digit-major table), an exclusive
// scan of that table (global base of every (digit, tile)), and a scatter in
// which each tile ranks its keys stably: keys are visited in position order
// (16 rounds of 256 consecutive keys), __match_any_sync gives the rank among
// equal digits inside a warp, and a per-round scan over the 8 warps plus a
// running per-digit count give the rank inside the tile.
//
// Used by the device transpose (CSC build) and by the edge-list -> CSR build.
#include "prim.cuh"

namespace kspn {

namespace {

constexpr int RX_THREADS = 256;
constexpr int RX_ITEMS   = 16;
constexpr int RX_TILE    = RX_THREADS * RX_ITEMS;
constexpr int RX_WARPS   = RX_THREADS / 32;

__global__ void __launch_bounds__(RX_THREADS)
k_radix_hist(uint32_t const* __restrict__ keys, uint64_t count, int shift, uint32_t* __restrict__ hist, uint32_t num_tiles)
{
  __shared__ uint32_t cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  uint64_t const base = static_cast<uint64_t>(blockIdx.x) * RX_TILE;
#pragma unroll 4
  for (int r = 0; r < RX_ITEMS; ++r) {
    uint64_t const i = base + static_cast<uint64_t>(r) * RX_THREADS + threadIdx.x;
    if (i < count) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[static_cast<uint64_t>(threadIdx.x) * num_tiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void __launch_bounds__(RX_THREADS)
k_radix_scatter(uint32_t const* __restrict__ kin,
                uint32_t const* __restrict__ vin,
                uint32_t* __restrict__ kout,
                uint32_t* __restrict__ vout,
                uint64_t count,
                int      shift,
                uint32_t const* __restrict__ hist_scanned,
                uint32_t num_tiles)
{
  __shared__ uint32_t tile_base[256];
  __shared__ uint32_t local_off[256];
  __shared__ uint32_t run[256];
  __shared__ uint16_t wcnt[2][RX_WARPS][256];
  __shared__ uint32_t s_key[RX_TILE];
  __shared__ uint32_t s_val[RX_TILE];

  unsigned const t = threadIdx.x, w = t >> 5, lane = t & 31u;
  tile_base[t]     = hist_scanned[static_cast<uint64_t>(t) * num_tiles + blockIdx.x];
  run[t]           = 0;
#pragma unroll
  for (int ww = 0; ww < RX_WARPS; ++ww) wcnt[0][ww][t] = wcnt[1][ww][t] = 0;
  __syncthreads();

  uint64_t const base    = static_cast<uint64_t>(blockIdx.x) * RX_TILE;
  unsigned const lane_lt = (1u << lane) - 1u;
  uint32_t       key[RX_ITEMS], val[RX_ITEMS], pos[RX_ITEMS];
  // 1. stable rank of every key among the tile's keys of the same digit
#pragma unroll
  for (int r = 0; r < RX_ITEMS; ++r) {
    int const      buf   = r & 1;
    uint64_t const i     = base + static_cast<uint64_t>(r) * RX_THREADS + t;
    bool const     valid = i < count;
    key[r]               = valid ? kin[i] : 0u;
    val[r]               = valid ? vin[i] : 0u;
    uint32_t const d     = valid ? ((key[r] >> shift) & 255u) : 0x100u;
    unsigned const peers = __match_any_sync(0xFFFFFFFFu, d);
    unsigned const rank  = __popc(peers & lane_lt);
    if (valid && rank == 0) wcnt[buf][w][d] = static_cast<uint16_t>(__popc(peers));
    __syncthreads();
    {
      uint32_t acc = run[t];
#pragma unroll
      for (int ww = 0; ww < RX_WARPS; ++ww) {
        uint32_t const c     = wcnt[buf][ww][t];
        wcnt[buf][ww][t]     = static_cast<uint16_t>(acc);
        wcnt[buf ^ 1][ww][t] = 0;
        acc += c;
      }
      run[t] = acc;
    }
    __syncthreads();
    pos[r] = valid ? wcnt[buf][w][d] + rank : 0xFFFFFFFFu;
  }
  // 2. digit offsets inside the tile, keys staged in digit order
  {
    uint32_t const c = run[t];
    uint32_t       x = c;
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
      uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, x, dd);
      if (lane >= static_cast<unsigned>(dd)) x += y;
    }
    __shared__ uint32_t wsum[RX_WARPS];
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t carry = 0;
    for (unsigned k = 0; k < w; ++k) carry += wsum[k];
    local_off[t] = carry + x - c;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RX_ITEMS; ++r) {
    if (pos[r] != 0xFFFFFFFFu) {
      uint32_t const d   = (key[r] >> shift) & 255u;
      uint32_t const p   = local_off[d] + pos[r];
      s_key[p]           = key[r];
      s_val[p]           = val[r];
    }
  }
  __syncthreads();
  // 3. coalesced write-out: consecutive slots of one digit go to
  //    consecutive global positions
  uint64_t const left = count - base;
  uint32_t const n    = left < RX_TILE ? static_cast<uint32_t>(left) : RX_TILE;
  for (uint32_t p = t; p < n; p += RX_THREADS) {
    uint32_t const k = s_key[p];
    uint32_t const d = (k >> shift) & 255u;
    uint32_t const o = tile_base[d] + (p - local_off[d]);
    kout[o]          = k;
    vout[o]          = s_val[p];
  }
}

} // namespace

size_t
radix_hist_entries(uint64_t count)
{
  return static_cast<size_t>(256) * div_up(count ? count : 1, RX_TILE) + 1;
}

void
radix_sort_pairs(kspn_context* ctx, uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, uint64_t count, int begin_bit, int end_bit, uint32_t* hist, uint32_t* hist_partial)
{
  if (count <= 1 || end_bit <= begin_bit) return;
  cudaStream_t const s         = ctx->stream;
  uint32_t const     num_tiles = div_up(count, RX_TILE);
  uint64_t const     entries   = static_cast<uint64_t>(256) * num_tiles;
  uint32_t *         ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
  for (int shift = begin_bit; shift < end_bit; shift += 8) {
    k_radix_hist<<<num_tiles, RX_THREADS, 0, s>>>(ki, count, shift, hist, num_tiles);
    KSPN_CHECK_LAUNCH();
    exclusive_scan<uint32_t>(s, f_array_u32_as_u32{ hist }, entries, hist, hist_partial, &ctx->launches);
    k_radix_scatter<<<num_tiles, RX_THREADS, 0, s>>>(ki, vi, ko, vo, count, shift, hist, num_tiles);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 2;
    uint32_t* tk = ki;
    ki           = ko;
    ko           = tk;
    uint32_t* tv = vi;
    vi           = vo;
    vo           = tv;
  }
  if (ki != keys) {
    KSPN_CUDA(cudaMemcpyAsync(keys, ki, count * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    KSPN_CUDA(cudaMemcpyAsync(vals, vi, count * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
}

void
radix_sort_pairs_to(kspn_context* ctx, uint32_t const* kin, uint32_t const* vin, uint32_t* kout, uint32_t* vout, uint32_t* ka, uint32_t* va, uint32_t* kb, uint32_t* vb, uint64_t count, int end_bit, uint32_t* hist, uint32_t* hist_partial)
{
  cudaStream_t const s = ctx->stream;
  int const          passes = (end_bit + 7) / 8;
  if (count == 0) return;
  if (passes == 0 || count == 1) {
    KSPN_CUDA(cudaMemcpyAsync(kout, kin, count * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    KSPN_CUDA(cudaMemcpyAsync(vout, vin, count * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    return;
  }
  uint32_t const num_tiles = div_up(count, RX_TILE);
  uint64_t const entries   = static_cast<uint64_t>(256) * num_tiles;
  uint32_t const* ki = kin;
  uint32_t const* vi = vin;
  for (int p = 0; p < passes; ++p) {
    // the last pass lands in (kout, vout); the ones before alternate A / B
    // so that no pass reads and writes one buffer
    bool const last = p == passes - 1;
    uint32_t*  ko   = last ? kout : (((passes - 1 - p) & 1) ? ka : kb);
    uint32_t*  vo   = last ? vout : (((passes - 1 - p) & 1) ? va : vb);
    int const  shift = 8 * p;
    k_radix_hist<<<num_tiles, RX_THREADS, 0, s>>>(ki, count, shift, hist, num_tiles);
    KSPN_CHECK_LAUNCH();
    exclusive_scan<uint32_t>(s, f_array_u32_as_u32{ hist }, entries, hist, hist_partial, &ctx->launches);
    k_radix_scatter<<<num_tiles, RX_THREADS, 0, s>>>(ki, vi, ko, vo, count, shift, hist, num_tiles);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 2;
    ki = ko;
    vi = vo;
  }
}


} // namespace kspn
