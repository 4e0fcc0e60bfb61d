// Learned pivot choice: a small MLP scores FW-BW pivot candidates.
//
// No reference counterpart.  The plain rule (trim_1_first's argmax of
// in-degree * out-degree, kaspan/scc/trim_1_local.hpp:12-46) stays the
// fallback; the model only changes WHICH vertex the FW-BW starts from, so
// the decomposition stays exact.  Candidates are the per-block best
// (in * out, id) pairs that k_trim_first leaves in ws.pivot (one per 1024
// vertices).
//
// Network, features and parameter layout: mlp.cuh.
#include "kspn_internal.cuh"
#include "mlp.cuh"
#include "prim.cuh"

#include <cuda_bf16.h>

#include <cmath>

namespace kspn {

namespace {

constexpr int MLP_WARPS = 8; // warps per block of the MLP kernels

// BF16-rounded weights of a block, in shared memory.
struct mlp_smem
{
  float w[MLP_NPARAM];
};

__device__ __forceinline__ void
mlp_load(mlp_smem& s, float const* __restrict__ params)
{
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) s.w[i] = __bfloat162float(__float2bfloat16_rn(params[i]));
  __syncthreads();
}

__device__ __forceinline__ float
mlp_forward(mlp_smem const& s, float const (&x)[MLP_IN], float& h1, float& h2)
{
  return mlp_forward_w(mlp_weights_smem{ s.w }, x, h1, h2);
}

// ordered key of a float (larger float -> larger unsigned)
__device__ __forceinline__ uint32_t
ordered(float x)
{
  uint32_t const u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Features of vertices vs[0, count) into feat[count][8].
// (ids >= n get zero features and raise *bad)
__global__ void __launch_bounds__(MLP_WARPS * 32)
k_mlp_features(uint32_t count, uint32_t n, uint32_t const* __restrict__ vs, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint64_t const* __restrict__ bh,
               uint32_t const* __restrict__ bc, float* __restrict__ feat, uint32_t* bad)
{
  unsigned const lane = threadIdx.x & 31u;
  for (uint32_t i = blockIdx.x * MLP_WARPS + (threadIdx.x >> 5); i < count; i += gridDim.x * MLP_WARPS) {
    float          f[MLP_IN] = {};
    uint32_t const v         = vs[i];
    if (v < n) mlp_features(v, fh, fc, bh, bc, f);
    else if (lane == 0) atomicExch(bad, 1u);
    if (lane < MLP_IN) {
      float x = 0;
#pragma unroll
      for (int k = 0; k < MLP_IN; ++k)
        if (static_cast<unsigned>(k) == lane) x = f[k];
      feat[static_cast<uint64_t>(i) * MLP_IN + lane] = x;
    }
  }
}

// Logits of feat[count][8].
__global__ void __launch_bounds__(MLP_WARPS * 32)
k_mlp_forward(uint32_t count, float const* __restrict__ feat, float const* __restrict__ params, float* __restrict__ out)
{
  __shared__ mlp_smem s;
  mlp_load(s, params);
  for (uint32_t i = blockIdx.x * MLP_WARPS + (threadIdx.x >> 5); i < count; i += gridDim.x * MLP_WARPS) {
    float x[MLP_IN];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) x[k] = feat[static_cast<uint64_t>(i) * MLP_IN + k];
    float      h1, h2;
    float const z = mlp_forward(s, x, h1, h2);
    if ((threadIdx.x & 31u) == 0) out[i] = z;
  }
}

// Mean binary cross-entropy of sigmoid(logit) against y over count samples
// and its gradient (FP32, with the BF16-rounded weights of the forward
// pass) added into grad[MLP_NPARAM]; loss added into *loss.  Each lane
// keeps its hidden unit's gradient rows; the block sums them in shared
// memory, then adds them to global memory once.
__global__ void __launch_bounds__(MLP_WARPS * 32)
k_mlp_grad(uint32_t count, float const* __restrict__ feat, float const* __restrict__ y, float const* __restrict__ params, float* __restrict__ grad, float* __restrict__ loss)
{
  __shared__ mlp_smem s;
  __shared__ float    g[MLP_NPARAM];
  __shared__ float    s_loss;
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) g[i] = 0.f;
  if (threadIdx.x == 0) s_loss = 0.f;
  mlp_load(s, params);
  unsigned const lane = threadIdx.x & 31u;
  float const    inv  = 1.f / static_cast<float>(count);
  float          gw1[MLP_IN] = {}, gw2[MLP_H] = {}, gb1 = 0, gb2 = 0, gw3 = 0, gb3 = 0, lsum = 0;
  for (uint32_t i = blockIdx.x * MLP_WARPS + (threadIdx.x >> 5); i < count; i += gridDim.x * MLP_WARPS) {
    float x[MLP_IN];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) x[k] = feat[static_cast<uint64_t>(i) * MLP_IN + k];
    float       h1, h2;
    float const z  = mlp_forward(s, x, h1, h2);
    float const yi = y[i];
    // loss = max(z, 0) - z y + log(1 + exp(-|z|)); dloss/dz = sigmoid(z) - y
    lsum += lane == 0 ? (fmaxf(z, 0.f) - z * yi + log1pf(expf(-fabsf(z)))) : 0.f;
    float const dz = (1.f / (1.f + expf(-z)) - yi) * inv;
    gb3 += lane == 0 ? dz : 0.f;
    gw3 += dz * h2;
    float const d2 = h2 > 0.f ? dz * s.w[O_W3 + lane] : 0.f; // d logit / d (pre-activation of unit lane, layer 2)
    gb2 += d2;
    float d1 = 0; // sum_j d2_j * W2[j][lane]
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
      float const d2j = __shfl_sync(0xFFFFFFFFu, d2, j);
      float const h1j = __shfl_sync(0xFFFFFFFFu, h1, j);
      gw2[j] += d2 * h1j;
      d1 += d2j * s.w[O_W2 + j * MLP_H + lane];
    }
    d1 = h1 > 0.f ? d1 : 0.f;
    gb1 += d1;
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) gw1[k] += d1 * x[k];
  }
  // block sums in shared memory, then one global add per parameter
#pragma unroll
  for (int k = 0; k < MLP_IN; ++k) atomicAdd(&g[O_W1 + lane * MLP_IN + k], gw1[k]);
#pragma unroll
  for (int j = 0; j < MLP_H; ++j) atomicAdd(&g[O_W2 + lane * MLP_H + j], gw2[j]);
  atomicAdd(&g[O_B1 + lane], gb1);
  atomicAdd(&g[O_B2 + lane], gb2);
  atomicAdd(&g[O_W3 + lane], gw3);
  if (lane == 0) {
    atomicAdd(&g[O_B3], gb3);
    atomicAdd(&s_loss, lsum);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x)
    if (g[i] != 0.f) atomicAdd(grad + i, g[i]);
  if (threadIdx.x == 0) atomicAdd(loss, s_loss * inv);
}

// One Adam step (Kingma and Ba, 2015) on the FP32 master weights.
__global__ void
k_mlp_adam(float* __restrict__ params, float const* __restrict__ grad, float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps, float b1t, float b2t)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_NPARAM; i += gridDim.x * blockDim.x) {
    float const gi = grad[i];
    float const mi = b1 * m[i] + (1.f - b1) * gi;
    float const vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i]           = mi;
    v[i]           = vi;
    params[i] -= lr * (mi / (1.f - b1t)) / (sqrtf(vi / (1.f - b2t)) + eps);
  }
}

// Learned pivot: every per-block candidate of k_trim_first is scored.  The
// model acts as a filter on the plain rule: among the candidates it accepts
// (logit >= 0: "in the largest SCC") the largest in * out wins, so the plain
// pivot stays whenever the model accepts it; when it accepts none, the
// largest logit wins.  Ties: smallest id.  Key for atomicMax: bit 63 =
// accepted, bits 62..32 = the product's float bits (accepted) or the
// logit's order key >> 1 (not accepted), low word = ~id.
// The plain pivot first (one warp): when the model accepts it, it is the
// answer of the rule below (the largest in * out among accepted
// candidates), so the full scan is skipped (*done = 1).
__global__ void __launch_bounds__(32)
k_pivot_check(uint64_t const* __restrict__ pv_prod, uint32_t const* __restrict__ pv_id, uint32_t n, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc,
              uint64_t const* __restrict__ bh, uint32_t const* __restrict__ bc, float const* __restrict__ params, uint32_t* done)
{
  __shared__ mlp_smem s;
  mlp_load(s, params);
  uint32_t const v = *pv_id;
  if (*pv_prod == 0 || v >= n) return; // no pivot: the scan decides
  float f[MLP_IN];
  mlp_features(v, fh, fc, bh, bc, f);
  float      h1, h2;
  float const z = mlp_forward(s, f, h1, h2);
  if (threadIdx.x == 0 && z >= 0.f) *done = 1u;
}

__global__ void __launch_bounds__(MLP_WARPS * 32)
k_pivot_score(uint32_t nb, uint64_t const* __restrict__ cand_prod, uint32_t const* __restrict__ cand_id, uint32_t n, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc,
              uint64_t const* __restrict__ bh, uint32_t const* __restrict__ bc, float const* __restrict__ params, unsigned long long* best, uint32_t const* done)
{
  if (*done) return; // the plain pivot was accepted
  __shared__ mlp_smem s;
  mlp_load(s, params);
  for (uint32_t i = blockIdx.x * MLP_WARPS + (threadIdx.x >> 5); i < nb; i += gridDim.x * MLP_WARPS) {
    uint32_t const v = cand_id[i];
    if (cand_prod[i] == 0 || v >= n) continue; // a block whose vertices were all trimmed
    float f[MLP_IN];
    mlp_features(v, fh, fc, bh, bc, f);
    float      h1, h2;
    float const z = mlp_forward(s, f, h1, h2);
    bool const               ok = z >= 0.f;
    unsigned long long const hi = ok ? (0x80000000ull | __float_as_uint(static_cast<float>(cand_prod[i]))) : static_cast<unsigned long long>(ordered(z) >> 1);
    if ((threadIdx.x & 31u) == 0) atomicMax(best, (hi << 32) | (0xFFFFFFFFu - v));
  }
}

// The chosen candidate into the pivot slot k_fwbw reads (left as it was
// when no candidate qualified).
__global__ void
k_pivot_pick(unsigned long long const* best, uint64_t* pv_prod, uint32_t* pv_id, uint32_t const* done)
{
  unsigned long long const b = *best;
  if (*done || b == 0) return;
  *pv_id   = 0xFFFFFFFFu - static_cast<uint32_t>(b & 0xFFFFFFFFu);
  *pv_prod = 1; // any non-zero product: a pivot exists
}

unsigned
mlp_grid(uint64_t samples)
{
  uint64_t const b = (samples + MLP_WARPS - 1) / MLP_WARPS;
  return static_cast<unsigned>(b < 148ull * 8 ? (b ? b : 1) : 148ull * 8);
}

} // namespace

void
mlp_features(kspn_context* ctx, dgraph const& g, uint32_t count, uint32_t const* vs, float* feat)
{
  if (!count) return;
  zero_counters(ctx);
  k_mlp_features<<<mlp_grid(count), MLP_WARPS * 32, 0, ctx->stream>>>(count, g.n, vs, g.fh, g.fc, g.bh, g.bc, feat, ctx->ws.ctr + CTR_ERR);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  read_counters(ctx);
  if (ctx->h_ctr[CTR_ERR]) throw error{ KSPN_ERR_INVALID_ARGUMENT, "mlp_features: a vertex id >= n" };
}

void
mlp_forward(kspn_context* ctx, uint32_t count, float const* feat, float const* params, float* out)
{
  if (!count) return;
  k_mlp_forward<<<mlp_grid(count), MLP_WARPS * 32, 0, ctx->stream>>>(count, feat, params, out);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

void
mlp_grad(kspn_context* ctx, uint32_t count, float const* feat, float const* y, float const* params, float* grad, float* loss)
{
  KSPN_CUDA(cudaMemsetAsync(grad, 0, MLP_NPARAM * sizeof(float), ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), ctx->stream));
  if (!count) return;
  k_mlp_grad<<<mlp_grid(count), MLP_WARPS * 32, 0, ctx->stream>>>(count, feat, y, params, grad, loss);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

void
mlp_adam(kspn_context* ctx, float* params, float const* grad, float* m, float* v, float lr, int step)
{
  float const b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float const b1t = static_cast<float>(std::pow(static_cast<double>(b1), step));
  float const b2t = static_cast<float>(std::pow(static_cast<double>(b2), step));
  k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, ctx->stream>>>(params, grad, m, v, lr, b1, b2, eps, b1t, b2t);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

// Rewrites the pivot slot that k_trim_first filled (trim_1_first_async)
// with the model's choice among its per-block candidates.  With check, the
// plain pivot in the slot is scored first and kept if the model accepts it;
// without, every candidate is scored (the resident launch has already
// scored the plain pivot and rejected it).
void
learned_pivot(kspn_context* ctx, dgraph const& g, float const* params, bool check)
{
  auto&          ws   = ctx->ws;
  unsigned const nb   = pivot_candidates(g.n);
  auto*          best = reinterpret_cast<unsigned long long*>(ws.ctr64 + 14); // [14] best key, [15] done flag (low word)
  auto*          done = reinterpret_cast<uint32_t*>(ws.ctr64 + 15);
  KSPN_CUDA(cudaMemsetAsync(best, 0, 2 * sizeof(unsigned long long), ctx->stream));
  uint32_t const* ids = reinterpret_cast<uint32_t const*>(ws.pivot + 4096);
  if (check) {
    k_pivot_check<<<1, 32, 0, ctx->stream>>>(ws.pivot + PV_FINAL, ids + PV_FINAL, g.n, g.fh, g.fc, g.bh, g.bc, params, done);
    ctx->launches += 1;
  }
  k_pivot_score<<<mlp_grid(nb), MLP_WARPS * 32, 0, ctx->stream>>>(nb, ws.pivot, ids, g.n, g.fh, g.fc, g.bh, g.bc, params, best, done);
  k_pivot_pick<<<1, 1, 0, ctx->stream>>>(best, ws.pivot + PV_FINAL, reinterpret_cast<uint32_t*>(ws.pivot + 4096) + PV_FINAL, done);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 2;
}

} // namespace kspn
