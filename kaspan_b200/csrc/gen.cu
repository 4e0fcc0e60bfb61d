// Seeded synthetic edge lists (stand-ins for the KaGen generators the
// reference benchmarks with; no reference counterpart).
//
// Stream: draw i under key K is fmix(K + (i+1)*gamma) with SplitMix64's
// gamma and variant-13 finaliser (Steele, Lea, Flood, OOPSLA 2014); the key
// of seed s is fmix(s + gamma).
//  * G(n, draws): u = lo32 * n >> 32, v = hi32 * n >> 32.
//  * R-MAT(scale): `scale` levels, level l reads 32-bit half l&1 of draw
//    i*ceil(scale/2) + l/2 and picks a|b|c|d against integer thresholds;
//    ids then pass through a seeded bijection of [0, 2^scale).
//  * RGG(n, g, r2): point i is (draw(K, 2i) >> 34, draw(K, 2i+1) >> 34), 30-bit
//    fixed point in [0, 1)^2, in cell (x*g >> 30, y*g >> 30) of a g x g grid;
//    vertex ids number the points sorted by (cell, i).  Each pair i < j of
//    vertices in the same or adjacent cells at squared distance <= r2 (units
//    of 2^-60) takes the top two bits of draw(K2, i << 32 | j) (K2: the key
//    of seed ^ "RGGEDGES"): 0 i->j, 1 j->i, 2 both, 3 neither.
#include "kspn_internal.cuh"
#include "prim.cuh"

#include <cmath>

namespace kspn {

namespace {

constexpr uint64_t GAMMA = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ uint64_t
fmix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__host__ __device__ __forceinline__ uint64_t
seed_key(uint64_t seed)
{
  return fmix64(seed + GAMMA);
}
__host__ __device__ __forceinline__ uint64_t
draw(uint64_t key, uint64_t i)
{
  return fmix64(key + (i + 1) * GAMMA);
}

struct perm_keys
{
  uint32_t add[3];
  uint32_t mul[3];
};

__device__ __forceinline__ uint32_t
permute(uint32_t x, uint32_t mask, int sh, perm_keys const& pk)
{
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    x = (x + pk.add[r]) & mask;
    x = (x * pk.mul[r]) & mask;
    if (sh > 0) x ^= x >> sh;
  }
  return x & mask;
}

__global__ void
k_gen_gnm(uint32_t n, uint64_t draws, uint64_t key, uint32_t* __restrict__ src, uint32_t* __restrict__ dst)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < draws; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint64_t const r = draw(key, i);
    src[i]           = static_cast<uint32_t>(((r & 0xFFFFFFFFull) * n) >> 32);
    dst[i]           = static_cast<uint32_t>(((r >> 32) * n) >> 32);
  }
}

__global__ void
k_gen_rmat(int scale, uint64_t draws, uint64_t key, uint64_t ta, uint64_t tab, uint64_t tabc, int do_perm, perm_keys pk, uint32_t* __restrict__ src, uint32_t* __restrict__ dst)
{
  int const      words = (scale + 1) / 2;
  uint32_t const mask  = scale >= 32 ? 0xFFFFFFFFu : ((1u << scale) - 1u);
  int const      sh    = (scale + 1) / 2;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < draws; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t u = 0, v = 0;
    uint64_t r = 0;
    for (int l = 0; l < scale; ++l) {
      if ((l & 1) == 0) r = draw(key, i * static_cast<uint64_t>(words) + static_cast<uint64_t>(l >> 1));
      uint64_t const x  = (l & 1) ? (r >> 32) : (r & 0xFFFFFFFFull);
      uint32_t const bu = x >= tab;                    // c or d
      uint32_t const bv = (x >= ta && x < tab) || x >= tabc; // b or d
      u                 = (u << 1) | bu;
      v                 = (v << 1) | bv;
    }
    if (do_perm) {
      u = permute(u, mask, sh, pk);
      v = permute(v, mask, sh, pk);
    }
    src[i] = u;
    dst[i] = v;
  }
}

// ---------------------------------------------------------------- RGG
constexpr uint64_t RGG_EDGE_SALT = 0x5247474544474553ull; // "RGGEDGES"

__global__ void
k_rgg_points(uint32_t n, uint64_t key, uint32_t g, uint32_t* __restrict__ cell, uint32_t* __restrict__ idx)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint64_t const x = draw(key, 2 * i) >> 34, y = draw(key, 2 * i + 1) >> 34;
    cell[i]          = static_cast<uint32_t>(((y * g) >> 30) * g + ((x * g) >> 30));
    idx[i]           = static_cast<uint32_t>(i);
  }
}

// coordinates by new id (j = rank of the point in (cell, i) order)
__global__ void
k_rgg_gather(uint32_t n, uint64_t key, uint32_t const* __restrict__ idx, uint32_t* __restrict__ px, uint32_t* __restrict__ py)
{
  for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint64_t const i = idx[j];
    px[j]            = static_cast<uint32_t>(draw(key, 2 * i) >> 34);
    py[j]            = static_cast<uint32_t>(draw(key, 2 * i + 1) >> 34);
  }
}

// cell_start[c] = first vertex of cell c (sorted cell ids), cell_start[cells] = n
__global__ void
k_rgg_cells(uint64_t cells, uint32_t n, uint32_t const* __restrict__ cell, uint64_t* __restrict__ cell_start)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    int64_t const lo = i == 0 ? -1 : static_cast<int64_t>(cell[i - 1]);
    int64_t const hi = i == n ? static_cast<int64_t>(cells) : static_cast<int64_t>(cell[i]);
    for (int64_t c = lo + 1; c <= hi; ++c) cell_start[c] = i;
  }
}

// Edges of vertex i to partners j > i; written from src/dst[0] when src is
// given; returns their number.
__device__ __forceinline__ uint32_t
rgg_edges_of(uint32_t i, uint32_t const* __restrict__ px, uint32_t const* __restrict__ py, uint64_t const* __restrict__ cell_start, uint32_t g, uint64_t r2, uint64_t key2, uint32_t* src,
             uint32_t* dst)
{
  uint32_t       cnt = 0;
  int64_t const  xi = px[i], yi = py[i];
  int64_t const  cx = (xi * g) >> 30, cy = (yi * g) >> 30;
  for (int64_t yy = cy - 1; yy <= cy + 1; ++yy) {
    if (yy < 0 || yy >= static_cast<int64_t>(g)) continue;
    for (int64_t xx = cx - 1; xx <= cx + 1; ++xx) {
      if (xx < 0 || xx >= static_cast<int64_t>(g)) continue;
      uint64_t const c = static_cast<uint64_t>(yy) * g + static_cast<uint64_t>(xx);
      for (uint64_t j = cell_start[c]; j < cell_start[c + 1]; ++j) {
        if (j <= i) continue;
        int64_t const  dx = xi - static_cast<int64_t>(px[j]);
        int64_t const  dy = yi - static_cast<int64_t>(py[j]);
        uint64_t const d2 = static_cast<uint64_t>(dx * dx) + static_cast<uint64_t>(dy * dy);
        if (d2 > r2) continue;
        unsigned const dir = static_cast<unsigned>(draw(key2, (static_cast<uint64_t>(i) << 32) | j) >> 62);
        if (dir == 0 || dir == 2) {
          if (src) src[cnt] = i, dst[cnt] = static_cast<uint32_t>(j);
          ++cnt;
        }
        if (dir == 1 || dir == 2) {
          if (src) src[cnt] = static_cast<uint32_t>(j), dst[cnt] = i;
          ++cnt;
        }
      }
    }
  }
  return cnt;
}

__global__ void
k_rgg_count(uint32_t n, uint32_t const* __restrict__ px, uint32_t const* __restrict__ py, uint64_t const* __restrict__ cell_start, uint32_t g, uint64_t r2, uint64_t key2, uint32_t* __restrict__ cnt)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    cnt[i] = rgg_edges_of(static_cast<uint32_t>(i), px, py, cell_start, g, r2, key2, nullptr, nullptr);
}

__global__ void
k_rgg_write(uint32_t n, uint32_t const* __restrict__ px, uint32_t const* __restrict__ py, uint64_t const* __restrict__ cell_start, uint32_t g, uint64_t r2, uint64_t key2, uint64_t const* __restrict__ off,
            uint32_t* __restrict__ src, uint32_t* __restrict__ dst)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    rgg_edges_of(static_cast<uint32_t>(i), px, py, cell_start, g, r2, key2, src + off[i], dst + off[i]);
}

unsigned
gen_grid(uint64_t items)
{
  uint64_t const b = (items + 255) / 256;
  return static_cast<unsigned>(b < 148ull * 64 ? (b ? b : 1) : 148ull * 64);
}

} // namespace

void
gen_gnm(kspn_context* ctx, uint32_t n, uint64_t draws, uint64_t seed, uint32_t* src, uint32_t* dst)
{
  if (!draws) return;
  k_gen_gnm<<<gen_grid(draws), 256, 0, ctx->stream>>>(n, draws, seed_key(seed), src, dst);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

void
gen_rmat(kspn_context* ctx, int scale, uint64_t draws, uint64_t seed, uint64_t ta, uint64_t tab, uint64_t tabc, int do_perm, uint32_t* src, uint32_t* dst)
{
  if (!draws) return;
  uint64_t const pkey = seed_key(seed ^ 0x5045524D55544531ull);
  perm_keys      pk;
  for (int r = 0; r < 3; ++r) {
    uint64_t const k = draw(pkey, static_cast<uint64_t>(r));
    pk.add[r]        = static_cast<uint32_t>(k);
    pk.mul[r]        = static_cast<uint32_t>(k >> 32) | 1u;
  }
  k_gen_rmat<<<gen_grid(draws), 256, 0, ctx->stream>>>(scale, draws, seed_key(seed), ta, tab, tabc, do_perm, pk, src, dst);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

} // namespace kspn

namespace kspn {

uint64_t
gen_rgg(kspn_context* ctx, uint32_t n, uint64_t seed, uint32_t g, uint64_t r2, uint32_t* src, uint32_t* dst, uint64_t cap)
{
  cudaStream_t const s = ctx->stream;
  if (n == 0) return 0;
  if (g == 0) throw error{ KSPN_ERR_INVALID_ARGUMENT, "gen_rgg: g must be at least 1" };
  uint64_t const cells = static_cast<uint64_t>(g) * g;
  if (cells >= 0xFFFFFFFFull) throw error{ KSPN_ERR_INVALID_ARGUMENT, "gen_rgg: g * g must be below 2^32 - 1" };
  size_t const hist_n = radix_hist_entries(n);
  size_t const part_n = scan_partial_entries((hist_n > n + 1 ? hist_n : n + 1) + 1);
  // scratch: cell, idx (+ alternates), radix histogram + partials, points,
  // cell starts, per-vertex counts and edge offsets
  size_t const bytes = (6 * (static_cast<size_t>(n) + 64) + hist_n + part_n) * sizeof(uint32_t) + (cells + 1 + n + 1 + part_n + 256) * sizeof(uint64_t) + 16 * 256;
  char*        base  = static_cast<char*>(context_buffer(ctx, BUF_GEN, bytes));
  size_t       off   = 0;
  auto         take  = [&](size_t count, size_t elem) {
    off          = (off + 255) & ~size_t(255);
    char* const p = base + off;
    off += count * elem;
    return static_cast<void*>(p);
  };
  auto* cell      = static_cast<uint32_t*>(take(n + 1, 4));
  auto* idx       = static_cast<uint32_t*>(take(n + 1, 4));
  auto* cell_alt  = static_cast<uint32_t*>(take(n + 1, 4));
  auto* idx_alt   = static_cast<uint32_t*>(take(n + 1, 4));
  auto* px        = static_cast<uint32_t*>(take(n + 1, 4));
  auto* py        = static_cast<uint32_t*>(take(n + 1, 4));
  auto* hist      = static_cast<uint32_t*>(take(hist_n, 4));
  auto* part      = static_cast<uint32_t*>(take(part_n, 4));
  auto* cstart    = static_cast<uint64_t*>(take(cells + 1, 8));
  auto* offs      = static_cast<uint64_t*>(take(static_cast<size_t>(n) + 1, 8));
  auto* part64    = static_cast<uint64_t*>(take(part_n, 8));
  auto* cnt       = cell_alt; // free after the sort
  uint64_t const key  = seed_key(seed);
  uint64_t const key2 = seed_key(seed ^ RGG_EDGE_SALT);
  unsigned const grid = gen_grid(n);
  k_rgg_points<<<grid, 256, 0, s>>>(n, key, g, cell, idx);
  KSPN_CHECK_LAUNCH();
  if (cells > 1) radix_sort_pairs(ctx, cell, idx, cell_alt, idx_alt, n, 0, bits_for(cells), hist, part);
  k_rgg_gather<<<grid, 256, 0, s>>>(n, key, idx, px, py);
  k_rgg_cells<<<gen_grid(static_cast<uint64_t>(n) + 1), 256, 0, s>>>(cells, n, cell, cstart);
  k_rgg_count<<<grid, 256, 0, s>>>(n, px, py, cstart, g, r2, key2, cnt);
  KSPN_CHECK_LAUNCH();
  exclusive_scan<uint64_t>(s, f_array_u32{ cnt }, n, offs, part64, &ctx->launches);
  uint64_t m = 0;
  KSPN_CUDA(cudaMemcpyAsync(&m, offs + n, sizeof(m), cudaMemcpyDeviceToHost, s));
  KSPN_CUDA(cudaStreamSynchronize(s));
  ctx->launches += 5;
  if (src && m <= cap) {
    k_rgg_write<<<grid, 256, 0, s>>>(n, px, py, cstart, g, r2, key2, offs, src, dst);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 1;
  }
  return m;
}

// ---------------------------------------------------------------- batch mix
// Graph i's key is draw i of the stream of `seed`; its shape stream is
// that key's stream (draw 0: size, draw 1: mean degree), its edge stream
// the stream of key ^ "EDGE": draw k is edge k, (u, v) as in G(n, m).

namespace {

__host__ __device__ __forceinline__ uint64_t
batch_key(uint64_t seed, uint32_t g)
{
  return draw(seed_key(seed), g);
}

__global__ void
k_gen_batch(uint32_t count, uint64_t seed, uint64_t const* __restrict__ vtx_off, uint64_t const* __restrict__ draw_off, uint32_t const* __restrict__ ids, uint64_t total, uint32_t* __restrict__ src,
            uint32_t* __restrict__ dst)
{
  for (uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < total; j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    // graph of draw j: the last g with draw_off[g] <= j
    uint32_t lo = 0, hi = count;
    while (lo + 1 < hi) {
      uint32_t const mid = (lo + hi) / 2;
      if (draw_off[mid] <= j) lo = mid;
      else hi = mid;
    }
    uint64_t const vo = vtx_off[lo];
    uint64_t const n  = vtx_off[lo + 1] - vo;
    uint64_t const d  = draw(seed_key(batch_key(seed, ids ? ids[lo] : lo) ^ 0x45444745ull), j - draw_off[lo]);
    src[j]            = static_cast<uint32_t>(vo + ((d & 0xFFFFFFFFull) * n >> 32));
    dst[j]            = static_cast<uint32_t>(vo + ((d >> 32) * n >> 32));
  }
}

__global__ void
k_batch_localize(uint32_t count, uint64_t N, uint64_t const* __restrict__ vtx_off, uint64_t const* __restrict__ head, uint32_t* __restrict__ csr)
{
  for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < N; v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t lo = 0, hi = count;
    while (lo + 1 < hi) {
      uint32_t const mid = (lo + hi) / 2;
      if (vtx_off[mid] <= v) lo = mid;
      else hi = mid;
    }
    uint32_t const vo = static_cast<uint32_t>(vtx_off[lo]);
    for (uint64_t e = head[v], end = head[v + 1]; e < end; ++e) csr[e] -= vo;
  }
}

} // namespace

void
batch_shape(uint32_t count, uint64_t seed, uint32_t log2_min, uint32_t log2_max, float deg_min, float deg_max, uint32_t* n_out, uint64_t* draws_out)
{
  for (uint32_t g = 0; g < count; ++g) {
    uint64_t const k  = seed_key(batch_key(seed, g));
    double const   u1 = static_cast<double>(draw(k, 0) >> 11) * 0x1.0p-53;
    double const   u2 = static_cast<double>(draw(k, 1) >> 11) * 0x1.0p-53;
    double const   n  = std::nearbyint(std::exp2(log2_min + (static_cast<double>(log2_max) - log2_min) * u1));
    double const   d  = deg_min + (static_cast<double>(deg_max) - deg_min) * u2;
    n_out[g]          = static_cast<uint32_t>(n < 1 ? 1 : n);
    draws_out[g]      = static_cast<uint64_t>(std::nearbyint(n_out[g] * d));
  }
}

void
gen_batch(kspn_context* ctx, uint32_t count, uint64_t seed, uint64_t const* vtx_off, uint64_t const* draw_off, uint32_t const* ids, uint64_t total, uint32_t* src, uint32_t* dst)
{
  if (!total || !count) return;
  uint64_t const b = (total + 255) / 256;
  k_gen_batch<<<static_cast<unsigned>(b < 148ull * 64 ? b : 148ull * 64), 256, 0, ctx->stream>>>(count, seed, vtx_off, draw_off, ids, total, src, dst);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

void
batch_localize(kspn_context* ctx, uint32_t count, uint64_t N, uint64_t const* vtx_off, uint64_t const* head, uint32_t* csr)
{
  if (!N || !count) return;
  uint64_t const b = (N + 255) / 256;
  k_batch_localize<<<static_cast<unsigned>(b < 148ull * 64 ? b : 148ull * 64), 256, 0, ctx->stream>>>(count, N, vtx_off, head, csr);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

} // namespace kspn
