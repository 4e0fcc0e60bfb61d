// Graph construction on the device:
//  * transpose (CSC build): the reference's backward_complement_graph
//    (kaspan/scc/backward_complement.hpp:22-68) is a counting sort that
//    leaves each in-row ascending; here a stable radix sort of the
//    (target, source) pairs, taken in CSR order, gives the same rows.
//  * build_csr: edge list -> CSR with self-loops and duplicates removed and
//    rows ascending (two stable sorts, then an adjacent-difference compact).
//  * validate: monotone offsets, head[0] == 0, head[n] == m, ids < n.
#include "prim.cuh"

#include <algorithm>

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
    // ids >= n (an invalid graph, reported by validation afterwards) are
    // clamped so that no head beyond n is written
    int64_t const lo = i == 0 ? -1 : static_cast<int64_t>(min(keys[i - 1], n));
    int64_t const hi = i == m ? static_cast<int64_t>(n) : static_cast<int64_t>(min(keys[i], n));
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

// src[e - e0] = u for the edges e in [e0, e1) of rows [u_lo, u_hi) (rows
// clipped to the range).  Small rows by their own lane, rows of 64+
// entries by the whole warp.
__global__ void
k_expand_range(uint32_t u_lo, uint32_t u_hi, uint64_t const* __restrict__ head, uint64_t e0, uint64_t e1, uint32_t* __restrict__ src)
{
  uint64_t const tid   = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  unsigned const lane  = threadIdx.x & 31u;
  uint64_t const wbase = u_lo + tid - lane;
  if (wbase >= u_hi) return;
  uint64_t const uu  = u_lo + tid;
  bool const     ok  = uu < u_hi;
  uint64_t       beg = ok ? head[uu] : 0, end = ok ? head[uu + 1] : 0;
  beg                = beg < e0 ? e0 : beg;
  end                = end > e1 ? e1 : end;
  end                = end < beg ? beg : end;
  bool const big = (end - beg) >= 64;
  if (!big)
    for (uint64_t e = beg; e < end; ++e) src[e - e0] = static_cast<uint32_t>(uu);
  for (unsigned todo = __ballot_sync(0xFFFFFFFFu, big); todo; todo &= todo - 1) {
    unsigned const l  = __ffs(todo) - 1;
    uint64_t const b  = __shfl_sync(0xFFFFFFFFu, beg, l);
    uint64_t const e_ = __shfl_sync(0xFFFFFFFFu, end, l);
    uint32_t const u  = static_cast<uint32_t>(wbase + l);
    for (uint64_t e = b + lane; e < e_; e += 32) src[e - e0] = u;
  }
}

// Offsets of one sorted chunk's entries inside their CSC rows, one block per
// RO_THREADS * RO_ITEMS consecutive entries (each thread RO_ITEMS of them):
// an entry's run of equal keys (one target) starts at the largest run start
// at or before it (a block-wide max-scan; a run that began in an earlier
// block is found by a binary search over the sorted keys), the run's start
// reads the target's placed count once and shares it in shared memory, and
// off[i] = that count + i's rank in the run.  One random read per run
// instead of two per entry.
constexpr int RO_THREADS = 256, RO_ITEMS = 8;
__global__ void __launch_bounds__(RO_THREADS)
k_run_offsets(uint32_t n, uint32_t const* __restrict__ keys, uint32_t cnt, uint32_t const* __restrict__ indeg, uint32_t* __restrict__ off)
{
  __shared__ uint32_t s_base[RO_THREADS * RO_ITEMS];
  __shared__ uint32_t s_wmax[RO_THREADS / 32];
  __shared__ uint32_t s_pre, s_prebase;
  uint32_t const b0 = blockIdx.x * (RO_THREADS * RO_ITEMS);
  if (b0 >= cnt) return;
  uint32_t const i0 = b0 + threadIdx.x * RO_ITEMS;
  uint32_t       key[RO_ITEMS];
  uint32_t       last = 0; // largest run start among this thread's items (0: none)
  bool           has  = false;
#pragma unroll
  for (int k = 0; k < RO_ITEMS; ++k) {
    uint32_t const i = i0 + k;
    key[k]           = i < cnt ? keys[i] : UNDECIDED;
    bool const start = i < cnt && (i == 0 || keys[i - 1] != key[k]);
    if (start) last = i, has = true;
  }
  if (threadIdx.x == 0) {
    // the run holding the block's first entry may have started earlier
    uint32_t const v = keys[b0];
    uint32_t       lo = 0, hi = b0; // first index in [0, b0] whose key is v
    if (b0 > 0 && keys[b0 - 1] == v) {
      while (lo < hi) {
        uint32_t const mid = lo + (hi - lo) / 2;
        if (keys[mid] >= v) hi = mid;
        else lo = mid + 1;
      }
    } else lo = b0;
    s_pre     = lo;
    s_prebase = v < n ? indeg[v] : 0u;
  }
  // block-wide inclusive max-scan of the threads' last run starts
  uint32_t incl = has ? last : 0u;
  unsigned const lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
    if (lane >= static_cast<unsigned>(d)) incl = max(incl, y);
  }
  if (lane == 31) s_wmax[wid] = incl;
  __syncthreads();
  uint32_t prev = s_pre; // starts before this thread's first item
  for (uint32_t w = 0; w < wid; ++w) prev = max(prev, s_wmax[w]);
  uint32_t const wexcl = __shfl_up_sync(0xFFFFFFFFu, incl, 1);
  if (lane > 0) prev = max(prev, wexcl);
  // run starts in this block publish their target's placed count
  uint32_t gstart[RO_ITEMS];
  uint32_t cur = prev;
#pragma unroll
  for (int k = 0; k < RO_ITEMS; ++k) {
    uint32_t const i = i0 + k;
    if (i < cnt && (i == 0 || keys[i - 1] != key[k])) {
      cur                = i;
      s_base[i - b0]     = key[k] < n ? indeg[key[k]] : 0u;
    }
    gstart[k] = cur;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < RO_ITEMS; ++k) {
    uint32_t const i = i0 + k;
    if (i >= cnt || key[k] >= n) continue;
    uint32_t const base = gstart[k] >= b0 ? s_base[gstart[k] - b0] : s_prebase;
    off[i]              = base + (i - gstart[k]);
  }
}

// placed count of each run's target, after the chunk: its last entry's
// offset + 1
__global__ void
k_run_ends(uint32_t n, uint32_t const* __restrict__ keys, uint32_t cnt, uint32_t const* __restrict__ off, uint32_t* __restrict__ indeg)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
    uint32_t const v = keys[i];
    if (v < n && (i + 1 == cnt || keys[i + 1] != v)) indeg[v] = off[i] + 1;
  }
}

// Placement in bands: band b holds the vertices [bv[b], bv[b+1]) whose CSC
// rows fill about 1/nb of bc; bv[b] = first vertex whose head reaches
// b * m / nb.
__global__ void
k_band_vertices(uint32_t n, uint64_t m, uint64_t const* __restrict__ head, uint32_t nb, uint32_t* __restrict__ bv)
{
  uint32_t const b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b > nb) return;
  uint64_t const target = b == nb ? m + 1 : (m / nb) * b + (m % nb) * b / nb;
  uint32_t       lo = 0, hi = n; // first v in [0, n] with head[v] >= target (n if none)
  while (lo < hi) {
    uint32_t const mid = lo + (hi - lo) / 2;
    if (head[mid] >= target) hi = mid;
    else lo = mid + 1;
  }
  bv[b] = b == 0 ? 0u : (b == nb ? n : lo);
}

// seg[b * nc + c] = first entry of sorted chunk c with key >= bv[b]
__global__ void
k_band_segments(uint32_t const* __restrict__ skeys, uint64_t m, uint64_t chunk, uint32_t nc, uint32_t nb, uint32_t const* __restrict__ bv, uint32_t* __restrict__ seg)
{
  uint32_t const t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (nb + 1) * nc) return;
  uint32_t const  b = t / nc, c = t % nc;
  uint64_t const  e0  = c * chunk;
  uint32_t const  cnt = static_cast<uint32_t>((e0 + chunk < m ? e0 + chunk : m) - e0);
  uint32_t const* k   = skeys + e0;
  uint32_t const  key = bv[b];
  uint32_t        lo = 0, hi = cnt;
  while (lo < hi) {
    uint32_t const mid = lo + (hi - lo) / 2;
    if (k[mid] >= key) hi = mid;
    else lo = mid + 1;
  }
  seg[t] = b == nb ? cnt : lo;
}

// bc[head[v] + off[i]] = source of entry i.  A neighbour id >= n (an
// invalid graph, which validation reports afterwards) splits runs, so
// positions are bounded here instead of trusted.
__global__ void
k_place(uint32_t n, uint64_t m, uint32_t const* __restrict__ keys, uint32_t const* __restrict__ off, uint32_t const* __restrict__ vals, uint64_t const* __restrict__ head, uint32_t* __restrict__ bc)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint32_t const v = keys[i];
    if (v >= n) continue;
    uint64_t const p = head[v] + off[i];
    if (p < m) bc[p] = vals[i];
  }
}

// The same placement, band by band: block x of the grid works on band
// x / (nc * per) and chunk (x / per) % nc, so the blocks resident at one
// time write into one or two bands' rows and L2 merges their sectors.
__global__ void
k_place_banded(uint32_t n, uint64_t m, uint64_t chunk, uint32_t nc, uint32_t per, uint32_t const* __restrict__ seg, uint32_t const* __restrict__ keys, uint32_t const* __restrict__ off, uint32_t const* __restrict__ vals, uint64_t const* __restrict__ head, uint32_t* __restrict__ bc)
{
  uint32_t const b = blockIdx.x / (nc * per), c = (blockIdx.x / per) % nc, part = blockIdx.x % per;
  uint32_t const lo = seg[b * nc + c], hi = seg[(b + 1) * nc + c];
  uint64_t const e0 = c * chunk;
  for (uint32_t j = lo + part * blockDim.x + threadIdx.x; j < hi; j += per * blockDim.x) {
    uint64_t const i = e0 + j;
    uint32_t const v = keys[i];
    if (v >= n) continue;
    uint64_t const p = head[v] + off[i];
    if (p < m) bc[p] = vals[i];
  }
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

namespace {
constexpr uint64_t PLACE_BAND_BYTES = 32ull << 20; // a quarter of L2
constexpr uint64_t BAND_MAX         = 4096;
} // namespace

void
upload_transpose(kspn_context* ctx, uint32_t n, uint64_t m, uint64_t const* h_fh, uint32_t const* h_fc, uint64_t* dfh, uint32_t* dfc, uint64_t* dbh, uint32_t* dbc, uint64_t chunk)
{
  cudaStream_t const s = ctx->stream;
  if (!ctx->copy_stream) {
    KSPN_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    KSPN_CUDA(cudaEventCreateWithFlags(&ctx->copy_ev, cudaEventDisableTiming));
  }
  cudaStream_t const cs = ctx->copy_stream;
  if (chunk == 0) chunk = UPLOAD_CHUNK;
  chunk = chunk < m ? chunk : (m ? m : 1);
  // the copies start after the work already queued on the context's stream
  KSPN_CUDA(cudaEventRecord(ctx->copy_ev, s));
  KSPN_CUDA(cudaStreamWaitEvent(cs, ctx->copy_ev, 0));
  KSPN_CUDA(cudaMemcpyAsync(dfh, h_fh, (static_cast<size_t>(n) + 1) * 8, cudaMemcpyHostToDevice, cs));
  if (n == 0 || m == 0) {
    KSPN_CUDA(cudaMemsetAsync(dbh, 0, (static_cast<size_t>(n) + 1) * 8, s));
    KSPN_CUDA(cudaEventRecord(ctx->copy_ev, cs));
    KSPN_CUDA(cudaStreamWaitEvent(s, ctx->copy_ev, 0));
    return;
  }
  if (m >= 0xFFFFFFFFull) throw error{ KSPN_ERR_INVALID_ARGUMENT, "upload_transpose: 2^32-1 or more edges are not supported" };
  // the chunk row ranges come from binary searches over the host offsets
  if (h_fh[0] != 0 || h_fh[n] != m) throw error{ KSPN_ERR_INVALID_GRAPH, "invalid graph: head[0] != 0 or head[n] != m;" };
  size_t const hist_n = radix_hist_entries(chunk);
  size_t const part_n = scan_partial_entries((hist_n > n + 1 ? hist_n : n + 1));
  scratch      sc;
  size_t const band_cap = (BAND_MAX + 1) * ((m + chunk - 1) / chunk);
  alloc_scratch(ctx, sc, (3 * (m + 64) + 5 * (chunk + 64) + (static_cast<size_t>(n) + 64) + BAND_MAX + 64 + band_cap + 64) * sizeof(uint32_t) + (hist_n + part_n) * sizeof(uint32_t) + part_n * sizeof(uint64_t) + 16384);
  size_t    off    = 0;
  uint32_t* skeys  = sc.carve<uint32_t>(off, m);     // chunk-sorted targets
  uint32_t* svals  = sc.carve<uint32_t>(off, m);     // their sources
  uint32_t* roff   = sc.carve<uint32_t>(off, m);     // offset inside the CSC row
  uint32_t* src    = sc.carve<uint32_t>(off, chunk); // sources of the chunk, CSR order
  uint32_t* ka     = sc.carve<uint32_t>(off, chunk);
  uint32_t* va     = sc.carve<uint32_t>(off, chunk);
  uint32_t* kb     = sc.carve<uint32_t>(off, chunk);
  uint32_t* vb     = sc.carve<uint32_t>(off, chunk);
  uint32_t* indeg  = sc.carve<uint32_t>(off, n);
  uint32_t* hist   = sc.carve<uint32_t>(off, hist_n);
  uint32_t* part   = sc.carve<uint32_t>(off, part_n);
  uint64_t* part64 = sc.carve<uint64_t>(off, part_n);
  uint32_t* bv     = sc.carve<uint32_t>(off, BAND_MAX + 1);
  uint32_t* seg    = sc.carve<uint32_t>(off, band_cap);
  KSPN_CUDA(cudaMemsetAsync(indeg, 0, static_cast<size_t>(n) * 4, s));
  int const bits = bits_for(n);
  for (uint64_t e0 = 0; e0 < m; e0 += chunk) {
    uint64_t const e1  = e0 + chunk < m ? e0 + chunk : m;
    uint32_t const cnt = static_cast<uint32_t>(e1 - e0);
    KSPN_CUDA(cudaMemcpyAsync(dfc + e0, h_fc + e0, static_cast<size_t>(cnt) * 4, cudaMemcpyHostToDevice, cs));
    KSPN_CUDA(cudaEventRecord(ctx->copy_ev, cs));
    KSPN_CUDA(cudaStreamWaitEvent(s, ctx->copy_ev, 0)); // the wait binds this record
    // rows holding [e0, e1): the host has the offsets
    uint32_t const u_lo = static_cast<uint32_t>(std::upper_bound(h_fh, h_fh + n + 1, e0) - h_fh - 1);
    uint32_t const u_hi = static_cast<uint32_t>(std::lower_bound(h_fh + u_lo, h_fh + n + 1, e1) - h_fh);
    k_expand_range<<<div_up(static_cast<uint64_t>(u_hi - u_lo), 256), 256, 0, s>>>(u_lo, u_hi, dfh, e0, e1, src);
    KSPN_CHECK_LAUNCH();
    radix_sort_pairs_to(ctx, dfc + e0, src, skeys + e0, svals + e0, ka, va, kb, vb, cnt, bits, hist, part);
    unsigned const g = grid_for(cnt, 256);
    k_run_offsets<<<div_up(cnt, RO_THREADS * RO_ITEMS), RO_THREADS, 0, s>>>(n, skeys + e0, cnt, indeg, roff + e0);
    k_run_ends<<<g, 256, 0, s>>>(n, skeys + e0, cnt, roff + e0, indeg);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 3;
  }
  exclusive_scan<uint64_t>(s, f_array_u32{ indeg }, n, dbh, part64, &ctx->launches);
  // bands of about PLACE_BAND_BYTES of CSC rows; `per` blocks per (band, chunk)
  uint64_t const nc  = (m + chunk - 1) / chunk;
  uint64_t const nb  = std::max<uint64_t>(1, std::min<uint64_t>((m * 4 + PLACE_BAND_BYTES - 1) / PLACE_BAND_BYTES, n));
  uint32_t const per = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(64, m / (nb * nc * 8192))));
  if ((nb + 1) * nc > band_cap || nb * nc * per > 0x7FFFFFFFull) {
    k_place<<<grid_for(m, 256), 256, 0, s>>>(n, m, skeys, roff, svals, dbh, dbc);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 1;
    return;
  }
  k_band_vertices<<<div_up(nb + 1, 256), 256, 0, s>>>(n, m, dbh, static_cast<uint32_t>(nb), bv);
  k_band_segments<<<div_up((nb + 1) * nc, 256), 256, 0, s>>>(skeys, m, chunk, static_cast<uint32_t>(nc), static_cast<uint32_t>(nb), bv, seg);
  k_place_banded<<<static_cast<unsigned>(nb * nc * per), 256, 0, s>>>(n, m, chunk, static_cast<uint32_t>(nc), per, seg, skeys, roff, svals, dbh, dbc);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 3;
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
