// The pivot MLP's device pieces shared by the training / scoring kernels
// (mlp.cu) and the resident FW-BW launch (reach.cu), which scores its own
// pivot during its first level.
//
// Network: 8 FP32 features -> 32 (ReLU) -> 32 (ReLU) -> 1 logit.  Weights
// are kept FP32 for training and rounded to BF16 for every forward pass; all
// sums accumulate in FP32.  One warp evaluates one sample: lane j owns
// hidden unit j of both layers.
//
// Features of vertex v (raw degrees; the first MLP_SAMPLE neighbours of each
// row are sampled; "survives trim round 1" = both degrees > 0, the rule of
// trim_1_first, kaspan/scc/trim_1_local.hpp:12-46):
//   0 log2(1 + out(v)) / 16          1 log2(1 + in(v)) / 16
//   2 log2(1 + mean out(w), w out-neighbour) / 16
//   3 log2(1 + mean in(w), w in-neighbour) / 16
//   4 share of sampled out-neighbours that survive trim round 1
//   5 share of sampled in-neighbours that survive trim round 1
//   6 the trim round in which v is removed, judged from its samples, / 2:
//     0 = round 1 (a degree is 0), 0.5 = round 2 (no sampled out- or no
//     sampled in-neighbour survives round 1), 1 = later or never
//   7 log2(1 + mean out(w), w in-neighbour) / 16
//
// Parameter layout (KSPN_MLP_PARAMS floats): W1[32][8], b1[32], W2[32][32],
// b2[32], w3[32], b3.
#pragma once

#include "kspn_internal.cuh"

#include <cuda_bf16.h>

namespace kspn {

constexpr int MLP_IN     = 8;
constexpr int MLP_H      = 32;
constexpr int MLP_SAMPLE = 64;
constexpr int O_W1 = 0, O_B1 = O_W1 + MLP_H * MLP_IN, O_W2 = O_B1 + MLP_H, O_B2 = O_W2 + MLP_H * MLP_H, O_W3 = O_B2 + MLP_H, O_B3 = O_W3 + MLP_H;
constexpr int MLP_NPARAM = O_B3 + 1;
static_assert(MLP_NPARAM == KSPN_MLP_PARAMS, "parameter count");

__device__ __forceinline__ float
mlp_log2p(float x)
{
  return log2f(1.0f + x);
}

// Features of v into f[0..8) (all lanes of the warp call it; every lane
// gets the same values).
__device__ __forceinline__ void
mlp_features(uint32_t v, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint64_t const* __restrict__ bh, uint32_t const* __restrict__ bc, float (&f)[MLP_IN])
{
  unsigned const lane = threadIdx.x & 31u;
  uint64_t const ob = fh[v], oe = fh[v + 1], ib = bh[v], ie = bh[v + 1];
  float          so_out = 0, si_in = 0, si_out = 0, o_live = 0, i_live = 0;
  uint32_t const no = static_cast<uint32_t>(oe - ob < MLP_SAMPLE ? oe - ob : MLP_SAMPLE);
  uint32_t const ni = static_cast<uint32_t>(ie - ib < MLP_SAMPLE ? ie - ib : MLP_SAMPLE);
  for (uint32_t k = lane; k < no; k += 32) {
    uint32_t const w  = fc[ob + k];
    float const    ow = static_cast<float>(fh[w + 1] - fh[w]);
    float const    iw = static_cast<float>(bh[w + 1] - bh[w]);
    so_out += ow;
    o_live += ow > 0.f && iw > 0.f ? 1.f : 0.f;
  }
  for (uint32_t k = lane; k < ni; k += 32) {
    uint32_t const w  = bc[ib + k];
    float const    ow = static_cast<float>(fh[w + 1] - fh[w]);
    float const    iw = static_cast<float>(bh[w + 1] - bh[w]);
    si_in += iw;
    si_out += ow;
    i_live += ow > 0.f && iw > 0.f ? 1.f : 0.f;
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) {
    so_out += __shfl_xor_sync(0xFFFFFFFFu, so_out, sh);
    si_in += __shfl_xor_sync(0xFFFFFFFFu, si_in, sh);
    si_out += __shfl_xor_sync(0xFFFFFFFFu, si_out, sh);
    o_live += __shfl_xor_sync(0xFFFFFFFFu, o_live, sh);
    i_live += __shfl_xor_sync(0xFFFFFFFFu, i_live, sh);
  }
  float const inv_o = no ? 1.f / static_cast<float>(no) : 0.f;
  float const inv_i = ni ? 1.f / static_cast<float>(ni) : 0.f;
  f[0]              = mlp_log2p(static_cast<float>(oe - ob)) * (1.f / 16);
  f[1]              = mlp_log2p(static_cast<float>(ie - ib)) * (1.f / 16);
  f[2]              = mlp_log2p(so_out * inv_o) * (1.f / 16);
  f[3]              = mlp_log2p(si_in * inv_i) * (1.f / 16);
  f[4]              = o_live * inv_o;
  f[5]              = i_live * inv_i;
  f[6]              = (no == 0 || ni == 0) ? 0.f : ((o_live == 0.f || i_live == 0.f) ? 0.5f : 1.f);
  f[7]              = mlp_log2p(si_out * inv_i) * (1.f / 16);
}

// The weights as the forward pass reads them: BF16-rounded values already
// in shared memory, or FP32 parameters in global memory rounded on read.
struct mlp_weights_smem
{
  float const*                        w;
  __device__ __forceinline__ float operator()(int i) const { return w[i]; }
};
struct mlp_weights_global
{
  float const*                        p;
  __device__ __forceinline__ float operator()(int i) const { return __bfloat162float(__float2bfloat16_rn(__ldg(p + i))); }
};

// Forward pass of one sample by one warp: returns the logit (all lanes);
// h1, h2 = this lane's hidden units.
template<class W>
__device__ __forceinline__ float
mlp_forward_w(W const& w, float const (&x)[MLP_IN], float& h1, float& h2)
{
  unsigned const lane = threadIdx.x & 31u;
  float          a    = w(O_B1 + lane);
#pragma unroll
  for (int k = 0; k < MLP_IN; ++k) a += w(O_W1 + lane * MLP_IN + k) * x[k];
  h1      = a > 0.f ? a : 0.f;
  float b = w(O_B2 + lane);
#pragma unroll
  for (int i = 0; i < MLP_H; ++i) b += w(O_W2 + lane * MLP_H + i) * __shfl_sync(0xFFFFFFFFu, h1, i);
  h2      = b > 0.f ? b : 0.f;
  float z = w(O_W3 + lane) * h2;
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) z += __shfl_xor_sync(0xFFFFFFFFu, z, sh);
  return z + w(O_B3);
}

} // namespace kspn
