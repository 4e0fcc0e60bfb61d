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
#include "kspn_internal.cuh"

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
