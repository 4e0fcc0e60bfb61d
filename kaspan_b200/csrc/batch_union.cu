// The batch mix as ONE graph (kspn_batch_options.route = 1; no reference
// counterpart: the reference decomposes one graph per `scc` call,
// kaspan/scc/scc.hpp:21-87).
//
// The graphs of a batch are disjoint, so the SCCs of their union are the
// graphs' SCCs.  The union gets global ids (each row entry shifted by its
// graph's first vertex) and one extra vertex s = n_total whose out-row AND
// in-row list one pivot per graph (the graph's largest in * out, smallest id
// on ties).  From s, FW(s) meets graph g exactly in FW(p_g) and BW(s) in
// BW(p_g) (a path from s enters a graph only through its pivot and never
// leaves it: s appears in no graph's rows), so the SCC of s is s plus every
// pivot's SCC -- one FW-BW of the single-graph pipeline decides one SCC in
// every graph at once.  s has in * out = P^2 (P pivots); where that beats
// every real vertex's in * out (checked on the host, else the mix takes the
// per-graph route) the pipeline's own pivot rule picks s, and s is decided
// by the first FW-BW, before any phase could read the rows s is missing
// from (its edges appear only in its own rows).  The rest of the
// single-graph pipeline (trim, residual, label
// searches) never looks at graph boundaries and is exact on the union as
// it is.  Afterwards the members of s's SCC are renamed graph by graph to
// the smallest member in their graph, and every id is made local.
#include "kspn_internal.cuh"

namespace kspn {

namespace {

constexpr int U_THREADS = 256;
constexpr uint64_t U_CHUNK = 1u << 16; // row entries per block of k_union_rows

// pivot of graph g: (in * out, id) with the larger product, then the
// smaller id; NONE (UNDECIDED) when every product is 0.
__global__ void __launch_bounds__(U_THREADS)
k_union_pivots(uint32_t count, uint64_t const* __restrict__ vtx_off, uint64_t const* __restrict__ fh, uint64_t const* __restrict__ bh, uint32_t* __restrict__ piv,
               unsigned long long* __restrict__ maxprod)
{
  __shared__ unsigned long long s_p[U_THREADS / 32];
  __shared__ uint32_t           s_v[U_THREADS / 32];
  uint32_t const                g = blockIdx.x;
  if (g >= count) return;
  uint64_t const     v0 = vtx_off[g], v1 = vtx_off[g + 1];
  unsigned long long bp = 0;
  uint32_t           bv = UNDECIDED;
  for (uint64_t v = v0 + threadIdx.x; v < v1; v += U_THREADS) {
    unsigned long long const p = (fh[v + 1] - fh[v]) * (bh[v + 1] - bh[v]);
    if (p > bp) bp = p, bv = static_cast<uint32_t>(v); // ascending v: the first strict max wins
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    unsigned long long const op = __shfl_down_sync(0xFFFFFFFFu, bp, s);
    uint32_t const           ov = __shfl_down_sync(0xFFFFFFFFu, bv, s);
    if (op > bp || (op == bp && ov < bv)) bp = op, bv = ov;
  }
  if ((threadIdx.x & 31) == 0) s_p[threadIdx.x >> 5] = bp, s_v[threadIdx.x >> 5] = bv;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < U_THREADS / 32; ++w)
      if (s_p[w] > bp || (s_p[w] == bp && s_v[w] < bv)) bp = s_p[w], bv = s_v[w];
    piv[g] = bp ? bv : UNDECIDED;
    if (bp) atomicMax(maxprod, bp);
  }
}

// Row entries [b * U_CHUNK, (b + 1) * U_CHUNK) shifted to global ids: the
// block finds the graph of its first entry (binary search over the graphs'
// first edges), each thread then walks its entries in order and moves on to
// later graphs as it crosses their first edges.
__global__ void __launch_bounds__(U_THREADS)
k_union_rows(uint32_t count, uint64_t m, uint64_t const* __restrict__ vtx_off, uint64_t const* __restrict__ head, uint32_t const* __restrict__ local,
             uint32_t* __restrict__ global)
{
  __shared__ uint32_t s_g;
  uint64_t const      e0 = static_cast<uint64_t>(blockIdx.x) * U_CHUNK;
  if (e0 >= m) return;
  uint64_t const e1 = e0 + U_CHUNK < m ? e0 + U_CHUNK : m;
  if (threadIdx.x == 0) {
    // the last graph whose first edge is <= e0 (graphs may have no edges)
    uint32_t lo = 0, hi = count; // invariant: first edge of lo <= e0; answer in [lo, hi)
    while (hi - lo > 1) {
      uint32_t const mid = (lo + hi) / 2;
      if (head[vtx_off[mid]] <= e0) lo = mid;
      else hi = mid;
    }
    s_g = lo;
  }
  __syncthreads();
  uint32_t g    = s_g;
  uint64_t next = g + 1 < count ? head[vtx_off[g + 1]] : m; // first edge of the next graph
  uint64_t base = vtx_off[g];
  for (uint64_t e = e0 + threadIdx.x; e < e1; e += U_THREADS) {
    while (e >= next) {
      ++g;
      base = vtx_off[g];
      next = g + 1 < count ? head[vtx_off[g + 1]] : m;
    }
    global[e] = static_cast<uint32_t>(base + local[e]);
  }
}

// The super-source's rows: the graphs' pivots, compacted in graph order, at
// [m, m + P) of both row arrays; both heads of s's successor slot n + 1.
// One block.
__global__ void __launch_bounds__(1024)
k_union_super(uint32_t count, uint64_t n, uint64_t m, uint32_t const* __restrict__ piv, uint64_t* __restrict__ fh, uint32_t* __restrict__ fc, uint64_t* __restrict__ bh,
              uint32_t* __restrict__ bc, uint32_t* __restrict__ p_out)
{
  __shared__ uint32_t s_base;
  __shared__ uint32_t s_w[32];
  if (threadIdx.x == 0) s_base = 0;
  __syncthreads();
  for (uint32_t b = 0; b < count; b += 1024) {
    uint32_t const g   = b + threadIdx.x;
    bool const     has = g < count && piv[g] != UNDECIDED;
    unsigned const bal = __ballot_sync(0xFFFFFFFFu, has);
    uint32_t const ws  = __popc(bal);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = ws;
    __syncthreads();
    uint32_t off = 0, tot = 0;
    for (uint32_t w = 0; w < 32; ++w) {
      if (w < (threadIdx.x >> 5)) off += s_w[w];
      tot += s_w[w];
    }
    off += __popc(bal & ((1u << (threadIdx.x & 31)) - 1u));
    if (has) {
      uint64_t const at = m + s_base + off;
      fc[at]            = piv[g];
      bc[at]            = piv[g];
    }
    __syncthreads();
    if (threadIdx.x == 0) s_base += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    fh[n + 1] = m + s_base;
    bh[n + 1] = m + s_base;
    *p_out    = s_base;
  }
}

// Graph g's ids made local; members of the super-source's SCC (id ==
// super) take the smallest such member of g.
__global__ void __launch_bounds__(U_THREADS)
k_union_rename(uint32_t count, uint64_t n, uint64_t const* __restrict__ vtx_off, uint32_t const* __restrict__ uid, uint32_t* __restrict__ scc_id)
{
  __shared__ uint32_t s_min;
  uint32_t const      g = blockIdx.x;
  if (g >= count) return;
  uint32_t const super = uid[n];
  uint64_t const v0 = vtx_off[g], v1 = vtx_off[g + 1];
  if (threadIdx.x == 0) s_min = UNDECIDED;
  __syncthreads();
  uint32_t mine = UNDECIDED;
  for (uint64_t v = v0 + threadIdx.x; v < v1; v += U_THREADS)
    if (uid[v] == super) {
      mine = static_cast<uint32_t>(v); // ascending v: the first is this thread's smallest
      break;
    }
  mine = __reduce_min_sync(0xFFFFFFFFu, mine);
  if ((threadIdx.x & 31) == 0 && mine != UNDECIDED) atomicMin(&s_min, mine);
  __syncthreads();
  uint32_t const gmin = s_min;
  for (uint64_t v = v0 + threadIdx.x; v < v1; v += U_THREADS) {
    uint32_t const u = uid[v];
    scc_id[v]        = static_cast<uint32_t>((u == super ? gmin : u) - v0);
  }
}

} // namespace

// Builds the union: heads copied (global edge positions already), rows
// shifted to global ids, the super-source's rows appended.  Buffers: fh, bh
// hold n + 2 entries, fc, bc m + count.  Returns P (pivots) and, in
// *maxprod, the largest in * out of a real vertex; synchronises.
uint32_t
union_build(kspn_context* ctx, uint32_t count, uint64_t n, uint64_t m, uint64_t const* vtx_off, uint64_t const* fh_in, uint32_t const* fc_in, uint64_t const* bh_in,
            uint32_t const* bc_in, uint64_t* fh, uint32_t* fc, uint64_t* bh, uint32_t* bc, uint32_t* piv, uint32_t* p_dev, unsigned long long* maxprod_dev,
            unsigned long long* maxprod)
{
  cudaStream_t const s = ctx->stream;
  KSPN_CUDA(cudaMemsetAsync(maxprod_dev, 0, sizeof(unsigned long long), s));
  KSPN_CUDA(cudaMemcpyAsync(fh, fh_in, (n + 1) * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
  KSPN_CUDA(cudaMemcpyAsync(bh, bh_in, (n + 1) * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
  k_union_pivots<<<count, U_THREADS, 0, s>>>(count, vtx_off, fh_in, bh_in, piv, maxprod_dev);
  unsigned const blocks = static_cast<unsigned>((m + U_CHUNK - 1) / U_CHUNK);
  if (blocks) {
    k_union_rows<<<blocks, U_THREADS, 0, s>>>(count, m, vtx_off, fh_in, fc_in, fc);
    k_union_rows<<<blocks, U_THREADS, 0, s>>>(count, m, vtx_off, bh_in, bc_in, bc);
  }
  k_union_super<<<1, 1024, 0, s>>>(count, n, m, piv, fh, fc, bh, bc, p_dev);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 3 + (blocks ? 2 : 0);
  uint32_t P = 0;
  KSPN_CUDA(cudaMemcpyAsync(&P, p_dev, sizeof(P), cudaMemcpyDeviceToHost, s));
  KSPN_CUDA(cudaMemcpyAsync(maxprod, maxprod_dev, sizeof(*maxprod), cudaMemcpyDeviceToHost, s));
  KSPN_CUDA(cudaStreamSynchronize(s));
  return P;
}

void
union_rename(kspn_context* ctx, uint32_t count, uint64_t n, uint64_t const* vtx_off, uint32_t const* uid, uint32_t* scc_id)
{
  k_union_rename<<<count, U_THREADS, 0, ctx->stream>>>(count, n, vtx_off, uid, scc_id);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

} // namespace kspn
