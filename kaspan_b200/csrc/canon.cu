// Canonical relabel on the device: every component id becomes the minimum
// vertex carrying it.  Same result as normalise_scc_id
// (kaspan/test/normalise_scc.hpp:10-25), which names each id after the
// first vertex in id order holding it.  Three streaming passes:
//   scratch[r] = UNDECIDED;  atomicMin(scratch[id[v]], v);  id[v] = scratch[id[v]].
#include "kspn_internal.cuh"

namespace kspn {

namespace {

constexpr int C_THREADS = 256;

unsigned
c_grid(uint64_t items)
{
  uint64_t const b = (items + C_THREADS - 1) / C_THREADS;
  return static_cast<unsigned>(b < 148ull * 16 ? (b ? b : 1) : 148ull * 16);
}

__global__ void
k_canon_min(uint32_t n, uint32_t const* __restrict__ id, uint32_t* __restrict__ scratch, uint32_t* __restrict__ err)
{
  for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t const r = id[v];
    if (r >= n) {
      atomicOr(err, 1u);
      continue;
    }
    atomicMin(scratch + r, static_cast<uint32_t>(v));
  }
}

__global__ void
k_canon_apply(uint32_t n, uint32_t* __restrict__ id, uint32_t const* __restrict__ scratch)
{
  for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t const r = id[v];
    if (r < n) id[v] = scratch[r];
  }
}

} // namespace

void
canonicalise(kspn_context* ctx, uint32_t n, uint32_t* scc_id, uint32_t* scratch)
{
  if (n == 0) return;
  cudaStream_t const s = ctx->stream;
  KSPN_CUDA(cudaMemsetAsync(scratch, 0xFF, static_cast<size_t>(n) * 4, s));
  KSPN_CUDA(cudaMemsetAsync(ctx->ws.ctr + CTR_ERR, 0, 4, s));
  k_canon_min<<<c_grid(n), C_THREADS, 0, s>>>(n, scc_id, scratch, ctx->ws.ctr + CTR_ERR);
  k_canon_apply<<<c_grid(n), C_THREADS, 0, s>>>(n, scc_id, scratch);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 2;
  read_counters(ctx);
  if (ctx->h_ctr[CTR_ERR]) throw error{ KSPN_ERR_INTERNAL, "canonical relabel: an id was >= n (vertex left undecided?)" };
}

} // namespace kspn
