// Learned pivot choice: a small MLP scores FW-BW pivot candidates.
//
// No reference counterpart.  The plain rule (trim_1_first's argmax of
// in-degree * out-degree, kaspan/scc/trim_1_local.hpp:12-46) stays the
// fallback; the model only changes WHICH vertex the FW-BW starts from, so
// the decomposition stays exact.  Candidates are the per-block best
// (in * out, id) pairs that k_trim_first leaves in ws.pivot (one per 1024
// vertices).
//
// Network: 8 FP32 features -> 32 (ReLU) -> 32 (ReLU) -> 1 (logit of "the
// vertex lies in the largest SCC").  Weights are kept FP32 for training and
// rounded to BF16 for every forward pass; all sums accumulate in FP32.  One
// warp evaluates one sample: lane j owns hidden unit j of both layers.
//
// Features of vertex v (raw degrees; the first MLP_SAMPLE neighbours of each
// row are sampled):
//   0 log2(1 + out(v)) / 16          1 log2(1 + in(v)) / 16
//   2 log2(1 + mean out(w), w out-neighbour) / 16
//   3 log2(1 + mean in(w), w in-neighbour) / 16
//   4 share of sampled out-neighbours with out(w) = 0 (dead ends)
//   5 share of sampled in-neighbours with in(w) = 0 (pure sources)
//   6 log2(1 + mean in(w), w out-neighbour) / 16
//   7 log2(1 + mean out(w), w in-neighbour) / 16
//
// Parameter layout (MLP_PARAMS floats): W1[32][8], b1[32], W2[32][32],
// b2[32], w3[32], b3.
#include "kspn_internal.cuh"
#include "prim.cuh"

#include <cuda_bf16.h>

#include <cmath>

namespace kspn {

namespace {

constexpr int MLP_IN     = 8;
constexpr int MLP_H      = 32;
constexpr int MLP_SAMPLE = 64;
constexpr int O_W1 = 0, O_B1 = O_W1 + MLP_H * MLP_IN, O_W2 = O_B1 + MLP_H, O_B2 = O_W2 + MLP_H * MLP_H, O_W3 = O_B2 + MLP_H, O_B3 = O_W3 + MLP_H;
constexpr int MLP_NPARAM = O_B3 + 1;
static_assert(MLP_NPARAM == KSPN_MLP_PARAMS, "parameter count");
constexpr int MLP_WARPS = 8; // warps per block of the MLP kernels

__device__ __forceinline__ float
log2p(float x)
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
  float          so_out = 0, so_in = 0, si_in = 0, si_out = 0, sinks = 0, srcs = 0;
  uint32_t const no = static_cast<uint32_t>(oe - ob < MLP_SAMPLE ? oe - ob : MLP_SAMPLE);
  uint32_t const ni = static_cast<uint32_t>(ie - ib < MLP_SAMPLE ? ie - ib : MLP_SAMPLE);
  for (uint32_t k = lane; k < no; k += 32) {
    uint32_t const w  = fc[ob + k];
    float const    ow = static_cast<float>(fh[w + 1] - fh[w]);
    float const    iw = static_cast<float>(bh[w + 1] - bh[w]);
    so_out += ow;
    so_in += iw;
    sinks += ow == 0.f ? 1.f : 0.f;
  }
  for (uint32_t k = lane; k < ni; k += 32) {
    uint32_t const w  = bc[ib + k];
    float const    ow = static_cast<float>(fh[w + 1] - fh[w]);
    float const    iw = static_cast<float>(bh[w + 1] - bh[w]);
    si_in += iw;
    si_out += ow;
    srcs += iw == 0.f ? 1.f : 0.f;
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) {
    so_out += __shfl_xor_sync(0xFFFFFFFFu, so_out, sh);
    so_in += __shfl_xor_sync(0xFFFFFFFFu, so_in, sh);
    si_in += __shfl_xor_sync(0xFFFFFFFFu, si_in, sh);
    si_out += __shfl_xor_sync(0xFFFFFFFFu, si_out, sh);
    sinks += __shfl_xor_sync(0xFFFFFFFFu, sinks, sh);
    srcs += __shfl_xor_sync(0xFFFFFFFFu, srcs, sh);
  }
  float const inv_o = no ? 1.f / static_cast<float>(no) : 0.f;
  float const inv_i = ni ? 1.f / static_cast<float>(ni) : 0.f;
  f[0]              = log2p(static_cast<float>(oe - ob)) * (1.f / 16);
  f[1]              = log2p(static_cast<float>(ie - ib)) * (1.f / 16);
  f[2]              = log2p(so_out * inv_o) * (1.f / 16);
  f[3]              = log2p(si_in * inv_i) * (1.f / 16);
  f[4]              = sinks * inv_o;
  f[5]              = srcs * inv_i;
  f[6]              = log2p(so_in * inv_o) * (1.f / 16);
  f[7]              = log2p(si_out * inv_i) * (1.f / 16);
}

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

// Forward pass of one sample by one warp: returns the logit (all lanes);
// h1, h2 = this lane's hidden units.
__device__ __forceinline__ float
mlp_forward(mlp_smem const& s, float const (&x)[MLP_IN], float& h1, float& h2)
{
  unsigned const lane = threadIdx.x & 31u;
  float          a    = s.w[O_B1 + lane];
#pragma unroll
  for (int k = 0; k < MLP_IN; ++k) a += s.w[O_W1 + lane * MLP_IN + k] * x[k];
  h1      = a > 0.f ? a : 0.f;
  float b = s.w[O_B2 + lane];
#pragma unroll
  for (int i = 0; i < MLP_H; ++i) b += s.w[O_W2 + lane * MLP_H + i] * __shfl_sync(0xFFFFFFFFu, h1, i);
  h2      = b > 0.f ? b : 0.f;
  float z = s.w[O_W3 + lane] * h2;
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) z += __shfl_xor_sync(0xFFFFFFFFu, z, sh);
  return z + s.w[O_B3];
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
// with the model's choice among its per-block candidates.
void
learned_pivot(kspn_context* ctx, dgraph const& g, float const* params)
{
  auto&          ws   = ctx->ws;
  unsigned const nb   = pivot_candidates(g.n);
  auto*          best = reinterpret_cast<unsigned long long*>(ws.ctr64 + 14); // [14] best key, [15] done flag (low word)
  auto*          done = reinterpret_cast<uint32_t*>(ws.ctr64 + 15);
  KSPN_CUDA(cudaMemsetAsync(best, 0, 2 * sizeof(unsigned long long), ctx->stream));
  uint32_t const* ids = reinterpret_cast<uint32_t const*>(ws.pivot + 4096);
  k_pivot_check<<<1, 32, 0, ctx->stream>>>(ws.pivot + PV_FINAL, ids + PV_FINAL, g.n, g.fh, g.fc, g.bh, g.bc, params, done);
  k_pivot_score<<<mlp_grid(nb), MLP_WARPS * 32, 0, ctx->stream>>>(nb, ws.pivot, ids, g.n, g.fh, g.fc, g.bh, g.bc, params, best, done);
  k_pivot_pick<<<1, 1, 0, ctx->stream>>>(best, ws.pivot + PV_FINAL, reinterpret_cast<uint32_t*>(ws.pivot + 4096) + PV_FINAL, done);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 3;
}

} // namespace kspn
