// Residual device finish: Tarjan on the undecided sub-graph.
//
// Reference: the residual step of variant/scc_trim_ex_residual.hpp:110-127
// (also scc_ispan_like.hpp, scc_trim_ex_light_residual.hpp):
// allgather_fw_sub_graph (kaspan/scc/allgather_sub_graph.hpp:253-301)
// gathers the sub-graph induced by the undecided vertices, tarjan
// (kaspan/scc/tarjan.hpp:20-136) decomposes it on one core, and each SCC is
// named by its smallest original vertex id.
//
// On the device the sub-graph splits into weakly connected pieces (an SCC
// never spans two), and one warp decomposes each small piece in shared
// memory:
//   1. union-find over the undecided vertices' out-edges to undecided
//      vertices (hooking the larger root under the smaller with atomicCAS,
//      path halving), then every entry set to its root by a pass in which
//      only v's own thread writes parent[v]; every loop bounded;
//   2. the undecided vertices in id order (ordered compaction), stably
//      radix-sorted by root: each piece is a segment, ascending inside;
//   3. a warp per segment of at most RS_MAXV vertices and RS_MAXE internal
//      edges builds the piece's CSR in shared memory (local ids by binary
//      search in the sorted segment), lane 0 runs an iterative Tarjan with
//      explicit stacks, and the warp writes each member's SCC id (its
//      smallest member: the smallest local index, since the segment is
//      ascending) and clears it from und.
// Larger pieces stay undecided; the pipeline's label rounds finish them.
#include "kspn_internal.cuh"
#include "prim.cuh"
#include "tarjan_smem.cuh"

namespace kspn {

namespace {

constexpr int      RS_THREADS = 256;
constexpr int      RS_WARPS   = 4;    // warps per block of the Tarjan kernel
constexpr uint32_t RS_FIND    = 1u << 20; // bound on one find / unite loop

unsigned
rs_grid(uint64_t items)
{
  uint64_t const b = (items + RS_THREADS - 1) / RS_THREADS;
  return static_cast<unsigned>(b < 148ull * 16 ? (b ? b : 1) : 148ull * 16);
}

__device__ __forceinline__ bool
und_has(uint32_t const* und, uint32_t v)
{
  return (und[v >> 5] >> (v & 31)) & 1u;
}

// root of x with path halving; UNDECIDED when the bound was reached
__device__ __forceinline__ uint32_t
rs_find(uint32_t* parent, uint32_t x)
{
  for (uint32_t it = 0; it < RS_FIND; ++it) {
    uint32_t const p = __ldcg(parent + x);
    if (p == x) return x;
    uint32_t const gp = __ldcg(parent + p);
    if (gp != p) parent[x] = gp; // halving (a lost race only skips a shortcut)
    x = gp;
  }
  return UNDECIDED;
}

__global__ void __launch_bounds__(RS_THREADS)
k_res_init(uint32_t n, uint32_t const* __restrict__ und, uint32_t* __restrict__ parent)
{
  for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * RS_THREADS + threadIdx.x; v < n; v += static_cast<uint64_t>(gridDim.x) * RS_THREADS)
    if (und_has(und, static_cast<uint32_t>(v))) parent[v] = static_cast<uint32_t>(v);
}

// u ~ v (both undecided); false when a loop bound was reached
__device__ __forceinline__ bool
rs_unite(uint32_t* parent, uint32_t u, uint32_t v)
{
  uint32_t a = u, b = v;
  for (uint32_t it = 0; it < RS_FIND; ++it) {
    a = rs_find(parent, a);
    b = rs_find(parent, b);
    if (a == UNDECIDED || b == UNDECIDED) return false;
    if (a == b) return true;
    if (a < b) {
      uint32_t const s = a;
      a = b, b = s;
    }
    // hook the larger root under the smaller
    if (atomicCAS(parent + a, a, b) == a) return true;
  }
  return false;
}

__device__ __forceinline__ void
rs_edge(uint32_t const* und, uint32_t* parent, uint32_t* err, uint32_t u, uint32_t v)
{
  if (v != u && und_has(und, v) && !rs_unite(parent, u, v)) atomicExch(err, 1u);
}

// u ~ v for every edge between undecided vertices.  A lane walks a row of
// up to 32 edges, the warp one of up to HEAVY_ROW; longer rows are listed
// for k_res_hook_heavy.
__global__ void __launch_bounds__(RS_THREADS)
k_res_hook(uint32_t n, uint32_t const* __restrict__ und, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint32_t* parent, uint32_t* err, uint32_t* heavy, uint32_t* heavy_n)
{
  unsigned const lane = threadIdx.x & 31u;
  uint64_t const span = (static_cast<uint64_t>(n) + 31) & ~31ull;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * RS_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * RS_THREADS) {
    uint32_t const u    = static_cast<uint32_t>(t);
    bool const     have = t < n && und_has(und, u);
    uint64_t       b = 0, e = 0;
    if (have) b = fh[u], e = fh[u + 1];
    uint64_t const len = e - b;
    if (have && len <= 32)
      for (uint64_t x = b; x < e; ++x) rs_edge(und, parent, err, u, fc[x]);
    for (unsigned todo = __ballot_sync(0xFFFFFFFFu, have && len > 32 && len <= HEAVY_ROW); todo; todo &= todo - 1) {
      unsigned const l  = __ffs(todo) - 1;
      uint32_t const ul = __shfl_sync(0xFFFFFFFFu, u, l);
      uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, b, l), e0 = __shfl_sync(0xFFFFFFFFu, e, l);
      for (uint64_t x = b0 + lane; x < e0; x += 32) rs_edge(und, parent, err, ul, fc[x]);
    }
    warp_push(have && len > HEAVY_ROW, u, heavy, heavy_n);
  }
}

// The listed rows, in slices over every warp of the grid.
__global__ void __launch_bounds__(RS_THREADS)
k_res_hook_heavy(uint32_t const* __restrict__ und, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint32_t* parent, uint32_t* err, uint32_t const* heavy, uint32_t const* heavy_n)
{
  unsigned const lane = threadIdx.x & 31u;
  heavy_slices(heavy, *heavy_n, fh, [&](uint32_t, uint32_t u, uint64_t b, uint64_t e) {
    for (uint64_t x = b + lane; x < e; x += 32) rs_edge(und, parent, err, u, fc[x]);
  });
}

// Shortens the trees (path halving; another thread's halving store may
// overwrite a root written here with an older ancestor, so k_res_flatten
// finishes the job).
__global__ void __launch_bounds__(RS_THREADS)
k_res_compress(uint32_t n, uint32_t const* __restrict__ und, uint32_t* parent, uint32_t* err)
{
  for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * RS_THREADS + threadIdx.x; v < n; v += static_cast<uint64_t>(gridDim.x) * RS_THREADS) {
    if (!und_has(und, static_cast<uint32_t>(v))) continue;
    uint32_t const r = rs_find(parent, static_cast<uint32_t>(v));
    if (r == UNDECIDED) atomicExch(err, 1u);
    else parent[v] = r;
  }
}

// parent[v] = root of v, each entry written only by v's own thread (the
// walk itself writes nothing), so every entry ends at its root.
__global__ void __launch_bounds__(RS_THREADS)
k_res_flatten(uint32_t n, uint32_t const* __restrict__ und, uint32_t* parent, uint32_t* err)
{
  for (uint64_t v = static_cast<uint64_t>(blockIdx.x) * RS_THREADS + threadIdx.x; v < n; v += static_cast<uint64_t>(gridDim.x) * RS_THREADS) {
    if (!und_has(und, static_cast<uint32_t>(v))) continue;
    uint32_t x  = static_cast<uint32_t>(v);
    bool     ok = false;
    for (uint32_t it = 0; it < RS_FIND; ++it) {
      uint32_t const p = __ldcg(parent + x);
      if (p == x) {
        ok = true;
        break;
      }
      x = p;
    }
    if (!ok) atomicExch(err, 1u);
    else parent[v] = x;
  }
}

struct f_und_popc
{
  uint32_t const* und;
  uint32_t        n;
  __device__ uint32_t operator()(uint64_t w) const
  {
    uint32_t x = und[w];
    if ((w + 1) * 32 > n) x &= (n & 31) ? (1u << (n & 31)) - 1u : 0xFFFFFFFFu;
    return __popc(x);
  }
};

// (root, vertex) of every undecided vertex, in vertex order
__global__ void __launch_bounds__(RS_THREADS)
k_res_list(uint32_t n, uint32_t const* __restrict__ und, uint32_t const* __restrict__ pos, uint32_t const* __restrict__ parent, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
  uint32_t const words = (n + 31) / 32;
  for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * RS_THREADS + threadIdx.x; w < words; w += static_cast<uint64_t>(gridDim.x) * RS_THREADS) {
    uint32_t x = und[w];
    if ((w + 1) * 32 > n) x &= (n & 31) ? (1u << (n & 31)) - 1u : 0xFFFFFFFFu;
    uint32_t j = pos[w];
    for (; x; x &= x - 1, ++j) {
      uint32_t const v = static_cast<uint32_t>(w) * 32 + __ffs(x) - 1;
      keys[j]          = parent[v];
      vals[j]          = v;
    }
  }
}

struct f_seg_head
{
  uint32_t const* keys;
  __device__ uint32_t operator()(uint64_t i) const { return i == 0 || keys[i] != keys[i - 1] ? 1u : 0u; }
};

__global__ void __launch_bounds__(RS_THREADS)
k_res_segments(uint64_t k, uint32_t const* __restrict__ keys, uint32_t const* __restrict__ spos, uint32_t* __restrict__ seg_start)
{
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * RS_THREADS + threadIdx.x; i < k; i += static_cast<uint64_t>(gridDim.x) * RS_THREADS)
    if (i == 0 || keys[i] != keys[i - 1]) seg_start[spos[i]] = static_cast<uint32_t>(i);
  if (blockIdx.x == 0 && threadIdx.x == 0) seg_start[spos[k]] = static_cast<uint32_t>(k);
}

// One warp per piece of at most RS_MAXV vertices and RS_MAXE internal edges.
__global__ void __launch_bounds__(RS_WARPS * 32)
k_res_tarjan(uint32_t const* __restrict__ seg_count,
             uint32_t const* __restrict__ seg_start,
             uint32_t const* __restrict__ vals,
             uint64_t const* __restrict__ fh,
             uint32_t const* __restrict__ fc,
             uint32_t* und,
             uint32_t* __restrict__ scc_id,
             uint32_t* decided,
             uint32_t* big)
{
  extern __shared__ __align__(16) unsigned char rs_smem[];
  unsigned const  lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  rs_piece&       p    = reinterpret_cast<rs_piece*>(rs_smem)[wid];
  uint32_t const  S    = *seg_count;
  uint32_t        dec  = 0;
  for (uint32_t sgi = blockIdx.x * RS_WARPS + wid; sgi < S; sgi += gridDim.x * RS_WARPS) {
    uint32_t const b = seg_start[sgi], k = seg_start[sgi + 1] - b;
    if (k > RS_MAXV) {
      if (lane == 0) atomicAdd(big, 1u);
      continue;
    }
    bool heavy_row = false;
    for (uint32_t i = lane; i < k; i += 32) {
      uint32_t const v = vals[b + i];
      p.vid[i]         = v;
      heavy_row |= fh[v + 1] - fh[v] > HEAVY_ROW;
    }
    if (__any_sync(0xFFFFFFFFu, heavy_row)) {
      // a member's row is too long for one lane: left to the later rounds
      if (lane == 0) atomicAdd(big, 1u);
      __syncwarp();
      continue;
    }
    __syncwarp();
    // internal out-degrees; lane l owns local vertices [l*per, l*per + per)
    uint32_t const per = (k + 31) / 32;
    uint32_t       cnt = 0;
    for (uint32_t i = lane * per; i < k && i < lane * per + per; ++i) {
      uint32_t const v = p.vid[i];
      uint32_t       c = 0;
      for (uint64_t e = fh[v], end = fh[v + 1]; e < end; ++e) {
        uint32_t const w = fc[e];
        c += und_has(und, w) ? 1u : 0u; // undecided neighbours lie in this piece
      }
      p.comp[i] = static_cast<uint16_t>(c < RS_MAXE ? c : RS_MAXE); // clamped; the total decides
      cnt += c;
    }
    uint32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= static_cast<unsigned>(d)) incl += y;
    }
    uint32_t const total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (total > RS_MAXE) {
      if (lane == 0) atomicAdd(big, 1u);
      __syncwarp();
      continue;
    }
    // offsets, then the local adjacency
    uint32_t run = incl - cnt;
    for (uint32_t i = lane * per; i < k && i < lane * per + per; ++i) {
      p.off[i] = static_cast<uint16_t>(run);
      run += p.comp[i];
    }
    if (lane == 0) p.off[k] = static_cast<uint16_t>(total);
    __syncwarp();
    for (uint32_t i = lane * per; i < k && i < lane * per + per; ++i) {
      uint32_t const v = p.vid[i];
      uint32_t       o = p.off[i];
      for (uint64_t e = fh[v], end = fh[v + 1]; e < end; ++e) {
        uint32_t const w = fc[e];
        if (und_has(und, w)) p.adj[o++] = static_cast<uint16_t>(rs_local(p, k, w));
      }
    }
    __syncwarp();
    if (lane == 0) rs_tarjan(p, k);
    __syncwarp();
    // ids and und; each vertex's word cleared by an atomic (pieces share words)
    for (uint32_t i = lane; i < k; i += 32) {
      uint32_t const v = p.vid[i];
      scc_id[v]        = p.vid[p.comp[i]];
      atomicAnd(und + (v >> 5), ~(1u << (v & 31)));
    }
    dec += lane == 0 ? k : 0;
    __syncwarp();
  }
  if (lane == 0 && dec) atomicAdd(decided, dec);
}

} // namespace

// Decides every undecided piece (weakly connected component of the
// undecided sub-graph) that fits a warp's shared memory; returns the
// vertices decided.  *pieces_left (nullable) = pieces left undecided.
uint32_t
residual(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t* pieces_left)
{
  cudaStream_t const s = ctx->stream;
  auto&              ws = ctx->ws;
  if (pieces_left) *pieces_left = 0;
  if (g.n == 0) return 0;
  uint32_t const words  = (g.n + 31) / 32;
  size_t const   hist_n = radix_hist_entries(g.n);
  size_t const   part_n = scan_partial_entries((hist_n > g.n + 1 ? hist_n : g.n + 1) + words + 1);
  size_t const   hcap   = heavy_capacity(g.n, g.m);
  size_t const   bytes  = (6 * (static_cast<size_t>(g.n) + 64) + words + 64 + hist_n + part_n + hcap) * sizeof(uint32_t) + 32 * 256;
  char*          base   = static_cast<char*>(context_buffer(ctx, BUF_BUILD, bytes));
  size_t         off    = 0;
  auto           take   = [&](size_t count) {
    off          = (off + 255) & ~size_t(255);
    auto* const p = reinterpret_cast<uint32_t*>(base + off);
    off += count * sizeof(uint32_t);
    return p;
  };
  uint32_t* keys = take(g.n + 1);
  uint32_t* vals = take(g.n + 1);
  uint32_t* kalt = take(g.n + 1);
  uint32_t* valt = take(g.n + 1);
  uint32_t* spos = take(g.n + 2);
  uint32_t* seg  = take(g.n + 2);
  uint32_t* wpos = take(words + 1);
  uint32_t* hist = take(hist_n);
  uint32_t* part = take(part_n);
  uint32_t* hlist = take(hcap);
  uint32_t* parent = ws.label;

  zero_counters(ctx);
  unsigned const grid = rs_grid(g.n);
  k_res_init<<<grid, RS_THREADS, 0, s>>>(g.n, und, parent);
  k_res_hook<<<grid, RS_THREADS, 0, s>>>(g.n, und, g.fh, g.fc, parent, ws.ctr + CTR_ERR, hlist, ws.ctr + CTR_RES_HEAVY);
  k_res_hook_heavy<<<148 * 8, RS_THREADS, 0, s>>>(und, g.fh, g.fc, parent, ws.ctr + CTR_ERR, hlist, ws.ctr + CTR_RES_HEAVY);
  k_res_compress<<<grid, RS_THREADS, 0, s>>>(g.n, und, parent, ws.ctr + CTR_ERR);
  k_res_flatten<<<grid, RS_THREADS, 0, s>>>(g.n, und, parent, ws.ctr + CTR_ERR);
  KSPN_CHECK_LAUNCH();
  // the undecided vertices in id order, then stably by root
  exclusive_scan<uint32_t>(s, f_und_popc{ und, g.n }, words, wpos, part, &ctx->launches);
  k_res_list<<<rs_grid(words), RS_THREADS, 0, s>>>(g.n, und, wpos, parent, keys, vals);
  KSPN_CHECK_LAUNCH();
  uint32_t k = 0;
  KSPN_CUDA(cudaMemcpyAsync(&k, wpos + words, sizeof(k), cudaMemcpyDeviceToHost, s));
  KSPN_CUDA(cudaStreamSynchronize(s));
  ctx->launches += 6;
  if (k == 0) return 0;
  radix_sort_pairs(ctx, keys, vals, kalt, valt, k, 0, bits_for(g.n), hist, part);
  exclusive_scan<uint32_t>(s, f_seg_head{ keys }, k, spos, part, &ctx->launches);
  k_res_segments<<<rs_grid(k), RS_THREADS, 0, s>>>(k, keys, spos, seg);
  // pieces: spos[k] of them, starts in seg
  size_t const smem = sizeof(rs_piece) * RS_WARPS;
  KSPN_CUDA(cudaFuncSetAttribute(k_res_tarjan, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  k_res_tarjan<<<148 * 4, RS_WARPS * 32, smem, s>>>(spos + k, seg, vals, g.fh, g.fc, und, scc_id, ws.ctr + CTR_DECIDED, ws.ctr + CTR_AUX);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 2;
  read_counters(ctx);
  if (ctx->h_ctr[CTR_ERR]) throw error{ KSPN_ERR_INTERNAL, "residual: union-find loop bound reached" };
  if (pieces_left) *pieces_left = ctx->h_ctr[CTR_AUX];
  return ctx->h_ctr[CTR_DECIDED];
}

} // namespace kspn
