// Canonical relabel on the device: every component id becomes the minimum
// vertex carrying it.  Same result as normalise_scc_id
// (kaspan/test/normalise_scc.hpp:10-25), which names each id after the
// first vertex in id order holding it.  Three streaming passes:
//   scratch[r] = r;  scratch[id[v]] = min(scratch[id[v]], v);  id[v] = scratch[id[v]].
// Every id is a member of its own component (trim: the vertex itself;
// FW-BW: the pivot; label search: the root), so the identity start is exact.
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
k_canon_init(uint32_t n, uint32_t* __restrict__ scratch, bool members)
{
  for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < n; v += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    scratch[v] = members ? static_cast<uint32_t>(v) : UNDECIDED;
}

// scratch[r] = min over members.  With `members` the ids are members of
// their own class and scratch starts as the identity (r already counted);
// otherwise (arbitrary ids, normalise_scc_id) it starts at UNDECIDED.  Lanes of a warp holding the
// same r combine first (one atomic per group), and the atomic is skipped
// when the stored minimum is already smaller -- the giant component's
// representative is read by every warp but written by very few.
__global__ void
k_canon_min(uint32_t n, uint32_t const* __restrict__ id, uint32_t* __restrict__ scratch, uint32_t* __restrict__ err, bool members)
{
  uint64_t const span = (static_cast<uint64_t>(n) + 31) & ~31ull;
  unsigned const lane = threadIdx.x & 31u;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t const v  = static_cast<uint32_t>(t);
    uint32_t       r  = t < n ? id[v] : UNDECIDED;
    if (t < n && r >= n) {
      atomicOr(err, 1u);
      r = UNDECIDED;
    }
    unsigned const peers  = __match_any_sync(0xFFFFFFFFu, r);
    uint32_t const mn     = __reduce_min_sync(peers, t < n ? v : UNDECIDED);
    bool const     leader = lane == static_cast<unsigned>(__ffs(peers) - 1);
    if (leader && r != UNDECIDED && (!members || mn < r) && mn < __ldcg(scratch + r)) atomicMin(scratch + r, mn);
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
canonicalise(kspn_context* ctx, uint32_t n, uint32_t* scc_id, uint32_t* scratch, bool members)
{
  if (n == 0) return;
  cudaStream_t const s = ctx->stream;
  KSPN_CUDA(cudaMemsetAsync(ctx->ws.ctr + CTR_ERR, 0, 4, s));
  k_canon_init<<<c_grid(n), C_THREADS, 0, s>>>(n, scratch, members);
  k_canon_min<<<c_grid(n), C_THREADS, 0, s>>>(n, scc_id, scratch, ctx->ws.ctr + CTR_ERR, members);
  k_canon_apply<<<c_grid(n), C_THREADS, 0, s>>>(n, scc_id, scratch);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 3;
  read_counters(ctx);
  if (ctx->h_ctr[CTR_ERR]) throw error{ KSPN_ERR_INTERNAL, "canonical relabel: an id was >= n (vertex left undecided?)" };
}

} // namespace kspn
