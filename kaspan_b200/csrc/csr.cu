// Graph construction on the device:
//  * transpose (CSC build): the reference's backward_complement_graph
//    (kaspan/scc/backward_complement.hpp:22-68) is a counting sort that
//    leaves each in-row ascending; here a stable radix sort of the
//    (target, source) pairs, taken in CSR order, gives the same rows.
//  * build_csr: edge list -> CSR with self-loops and duplicates removed and
//    rows ascending (two stable sorts, then an adjacent-difference compact).
//  * validate: monotone offsets, head[0] == 0, head[n] == m, ids < n.
#include "prim.cuh"

namespace kspn {

namespace {

// src[e] = u for every edge e of row u.  Small rows by their own lane,
// rows of 64+ entries by the whole warp.
__global__ void
k_expand_rows(uint32_t n, uint64_t const* __restrict__ head, uint32_t* __restrict__ src)
{
  uint64_t const tid  = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  unsigned const lane = threadIdx.x & 31u;
  uint64_t const wbase = tid - lane; // first vertex of this warp's group
  if (wbase >= n) return;
  uint32_t const u   = static_cast<uint32_t>(tid);
  bool const     ok  = tid < n;
  uint64_t const beg = ok ? head[u] : 0, end = ok ? head[u + 1] : 0;
  bool const     big = (end - beg) >= 64;
  if (!big)
    for (uint64_t e = beg; e < end; ++e) src[e] = u;
  unsigned todo = __ballot_sync(0xFFFFFFFFu, big);
  while (todo) {
    unsigned const l  = __ffs(todo) - 1;
    todo &= todo - 1;
    uint64_t const b  = __shfl_sync(0xFFFFFFFFu, beg, l);
    uint64_t const e_ = __shfl_sync(0xFFFFFFFFu, end, l);
    uint32_t const uu = static_cast<uint32_t>(wbase + l);
    for (uint64_t e = b + lane; e < e_; e += 32) src[e] = uu;
  }
}

// head[v] = first index of key v in the ascending keys[0, m) (= m past the
// last key): every boundary between two different keys writes the heads of
// the ids it spans, so each head is written exactly once, without atomics.
__global__ void
k_heads_from_sorted(uint32_t n, uint64_t m, uint32_t const* __restrict__ keys, uint64_t* __restrict__ head)
{
  uint64_t const stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i <= m; i += stride) {
    int64_t const lo = i == 0 ? -1 : static_cast<int64_t>(keys[i - 1]);
    int64_t const hi = i == m ? static_cast<int64_t>(n) : static_cast<int64_t>(keys[i]);
    for (int64_t v = lo + 1; v <= hi; ++v) head[v] = i;
  }
}

// keep[i] = 1 for the first copy of each (src, dst) with src != dst
struct f_keep
{
  uint32_t const* s;
  uint32_t const* d;
  __device__ uint32_t operator()(uint64_t i) const
  {
    if (s[i] == d[i]) return 0u;
    if (i > 0 && s[i - 1] == s[i] && d[i - 1] == d[i]) return 0u;
    return 1u;
  }
};

__global__ void
k_compact_edges(uint64_t m_raw, uint32_t const* __restrict__ s, uint32_t const* __restrict__ d, uint32_t const* __restrict__ pos, uint32_t* __restrict__ csr, uint32_t* __restrict__ src_kept)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m_raw; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    if (pos[i + 1] != pos[i]) {
      csr[pos[i]]      = d[i];
      src_kept[pos[i]] = s[i];
    }
  }
}

__global__ void
k_validate(uint32_t n, uint64_t m, uint64_t const* __restrict__ head, uint32_t const* __restrict__ csr, uint32_t* __restrict__ err)
{
  uint64_t const stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    if (head[i] > head[i + 1]) atomicOr(err, 1u);
  if (blockIdx.x == 0 && threadIdx.x == 0 && (head[0] != 0 || head[n] != m)) atomicOr(err, 2u);
  for (uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < m; e += stride)
    if (csr[e] >= n) atomicOr(err, 4u);
}

unsigned
grid_for(uint64_t items, int threads)
{
  uint64_t const b = (items + threads - 1) / threads;
  return static_cast<unsigned>(b < 148ull * 32 ? (b ? b : 1) : 148ull * 32);
}

struct scratch
{
  void*  p     = nullptr;
  size_t bytes = 0;
  template<typename T>
  T* carve(size_t& off, size_t count)
  {
    off      = (off + 255) & ~size_t(255);
    T* ptr   = reinterpret_cast<T*>(static_cast<char*>(p) + off);
    off += count * sizeof(T);
    return ptr;
  }
};

void
alloc_scratch(kspn_context* ctx, scratch& s, size_t bytes)
{
  s.p     = context_buffer(ctx, BUF_BUILD, bytes);
  s.bytes = bytes;
}

} // namespace

void
transpose(kspn_context* ctx, uint32_t n, uint64_t m, uint64_t const* fh, uint32_t const* fc, uint64_t* bh, uint32_t* bc, uint32_t* /*unused*/)
{
  cudaStream_t const s = ctx->stream;
  if (n == 0) {
    KSPN_CUDA(cudaMemsetAsync(bh, 0, sizeof(uint64_t), s));
    return;
  }
  size_t const hist_n = radix_hist_entries(m);
  size_t const part_n = scan_partial_entries(hist_n > n + 1 ? hist_n : n + 1);
  scratch      sc;
  alloc_scratch(ctx, sc, 3 * (m + 64) * sizeof(uint32_t) + (hist_n + part_n + n + 64) * sizeof(uint64_t) + 4096);
  size_t    off   = 0;
  uint32_t* keys  = sc.carve<uint32_t>(off, m + 1);
  uint32_t* kalt  = sc.carve<uint32_t>(off, m + 1);
  uint32_t* valt  = sc.carve<uint32_t>(off, m + 1);
  uint32_t* hist  = sc.carve<uint32_t>(off, hist_n);
  uint32_t* part  = sc.carve<uint32_t>(off, part_n);
  uint32_t* cnt   = sc.carve<uint32_t>(off, n + 1);
  uint64_t* part64 = sc.carve<uint64_t>(off, part_n);

  if (m) {
    KSPN_CUDA(cudaMemcpyAsync(keys, fc, m * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    k_expand_rows<<<div_up(n, 256), 256, 0, s>>>(n, fh, bc);
    KSPN_CHECK_LAUNCH();
    radix_sort_pairs(ctx, keys, bc, kalt, valt, m, 0, bits_for(n), hist, part);
  }
  k_heads_from_sorted<<<grid_for(m + 1, 256), 256, 0, s>>>(n, m, keys, bh);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 2;
  (void)cnt;
  (void)part64;
}

uint64_t
build_csr(kspn_context* ctx, uint32_t n, uint64_t m_raw, uint32_t* src, uint32_t* dst, uint64_t* head, uint32_t* csr)
{
  cudaStream_t const s = ctx->stream;
  if (m_raw >= 0xFFFFFFFFull) throw error{ KSPN_ERR_INVALID_ARGUMENT, "build_csr: edge lists of 2^32-1 or more entries are not supported" };
  size_t const hist_n = radix_hist_entries(m_raw);
  size_t const part_n = scan_partial_entries((hist_n > m_raw + 1 ? hist_n : m_raw + 1) + n + 1);
  scratch      sc;
  alloc_scratch(ctx, sc, 3 * (m_raw + 64) * sizeof(uint32_t) + (hist_n + part_n + n + 64) * sizeof(uint64_t) + 4096);
  size_t    off    = 0;
  uint32_t* kalt   = sc.carve<uint32_t>(off, m_raw + 1);
  uint32_t* valt   = sc.carve<uint32_t>(off, m_raw + 1);
  uint32_t* pos    = sc.carve<uint32_t>(off, m_raw + 1);
  uint32_t* hist   = sc.carve<uint32_t>(off, hist_n);
  uint32_t* part   = sc.carve<uint32_t>(off, part_n);
  uint32_t* rowcnt = sc.carve<uint32_t>(off, n + 1);
  uint64_t* part64 = sc.carve<uint64_t>(off, part_n);

  int const b = bits_for(n);
  // (dst, src) stably by dst, then (src, dst) stably by src => sorted by (src, dst)
  radix_sort_pairs(ctx, dst, src, kalt, valt, m_raw, 0, b, hist, part);
  radix_sort_pairs(ctx, src, dst, kalt, valt, m_raw, 0, b, hist, part);
  exclusive_scan<uint32_t>(s, f_keep{ src, dst }, m_raw, pos, part, &ctx->launches);
  uint32_t m32 = 0;
  KSPN_CUDA(cudaMemcpyAsync(&m32, pos + m_raw, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  KSPN_CUDA(cudaStreamSynchronize(s));
  uint64_t const m = m32;
  if (m_raw) {
    k_compact_edges<<<grid_for(m_raw, 256), 256, 0, s>>>(m_raw, src, dst, pos, csr, kalt);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 1;
  }
  k_heads_from_sorted<<<grid_for(m + 1, 256), 256, 0, s>>>(n, m, kalt, head);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  (void)rowcnt;
  (void)part64;
  KSPN_CUDA(cudaStreamSynchronize(s));
  return m;
}

void
validate(kspn_context* ctx, dgraph const& g)
{
  cudaStream_t const s = ctx->stream;
  uint32_t*          err = ctx->ws.ctr + CTR_ERR;
  KSPN_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), s));
  uint64_t const items = g.m > g.n ? g.m : g.n;
  k_validate<<<grid_for(items, 256), 256, 0, s>>>(g.n, g.m, g.fh, g.fc, err);
  if (g.bh != g.fh) k_validate<<<grid_for(items, 256), 256, 0, s>>>(g.n, g.m, g.bh, g.bc, err);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 2;
  read_counters(ctx);
  uint32_t const e = ctx->h_ctr[CTR_ERR];
  if (e) {
    std::string what = "invalid graph:";
    if (e & 1u) what += " offsets decrease;";
    if (e & 2u) what += " head[0] != 0 or head[n] != m;";
    if (e & 4u) what += " neighbour id >= n;";
    throw error{ KSPN_ERR_INVALID_GRAPH, what };
  }
}

} // namespace kspn
