// Single-pivot forward-backward search on the device.
//
// Reference: cache_forward_backward_search (kaspan/scc/cache_pivot_search.hpp:16-104),
// equal to forward_backward_search (pivot_search.hpp:15-85) at one rank:
//   FW  = vertices reachable from the pivot through undecided vertices
//   BW  = vertices of FW that reach the pivot through FW vertices
//   BW is the pivot's SCC; each member is decided with id = pivot.
// The reference walks a LIFO stack on one core; here each search is a
// level-synchronous, direction-optimising reachability (Beamer, Asanovic,
// Patterson, SC'12), of which only the reached SET matters:
//   top-down  : load-balanced expansion of the frontier's rows (expand.cuh);
//   bottom-up : every candidate scans its opposite-direction row and stops
//               at the first visited neighbour.
// Before each level the frontier's edge count m_f is known (frontier scan);
// the level runs bottom-up when m_f > m_u / alpha (m_u: edges not yet
// explored) and returns top-down when the frontier holds fewer than
// n_candidates / beta vertices.
//
// Vertex state per search, one bit each (u32 words, atomics on words):
//   FW: cand = undecided and not yet reached (a copy of und, bits taken on
//       discovery), vis_a = reached;
//   BW: vis_a = FW-reached and not yet BW-reached (bits taken on discovery),
//       vis_b = BW-reached.
// Each edge costs at most one probe and each discovery two atomics; the
// undecided set and ids are written once at the end, a word at a time.
//
// Level control lives on the device (reach_state): a `decide` kernel picks
// the direction from the scan, both expansion kernels are launched and the
// one whose gate is closed returns at once, and an `advance` kernel flips the
// queues and sets the loop condition.  The whole FW-BW is ONE CUDA graph
// launch with two conditional while-nodes (one per search); with profiling
// on, the same kernels run from a host loop with CUDA events around the
// expansion kernels.
#include "expand.cuh"

#include <cstring>
#include <tuple>

namespace kspn {

namespace {

constexpr int R_THREADS = 256;
constexpr int R_BIG     = 32;
constexpr int BU_BUF    = 2048;
constexpr int BU_ILP    = 4;

unsigned
r_grid(uint64_t items)
{
  uint64_t const b = (items + R_THREADS - 1) / R_THREADS;
  return static_cast<unsigned>(b < 148ull * 8 ? (b ? b : 1) : 148ull * 8);
}

// bottom-up: one block per chunk of R_THREADS bitmap words, capped at the
// resident-block count
unsigned
bu_grid(uint32_t n)
{
  uint64_t const chunks = ((static_cast<uint64_t>(n) + 31) / 32 + R_THREADS - 1) / R_THREADS;
  return static_cast<unsigned>(chunks < 148ull * 4 ? (chunks ? chunks : 1) : 148ull * 4);
}

// Device-side control block of one FW-BW (lives in the workspace).
struct reach_state
{
  uint32_t           cur;      // frontier selector (fio)
  uint32_t           qn[2];    // queue lengths
  uint32_t           mode;     // 0 top-down, 1 bottom-up
  uint32_t           level;    // levels of the running search
  uint32_t           cap;      // level cap per search
  uint32_t           err;      // 1: a search hit the cap
  uint32_t           ntiles;   // frontier tiles (scan)
  uint32_t           bu;       // bottom-up levels of the running search
  uint32_t           pivot;
  uint32_t           n_und;    // undecided vertices (candidates of FW)
  uint32_t           id;       // id given to the SCC
  uint32_t           decided;  // SCC size
  uint32_t           min_ids;  // 1: id = smallest member, 0: id = pivot
  uint32_t           scan;     // 1: this level scans its frontier
  uint32_t           levels_fw, bu_fw, levels_bw, bu_bw;
  unsigned long long m_u, m_out, m_in, m_f, alpha, beta;
  unsigned long long edges_td, edges_bu, cands_bu;
};
static_assert(sizeof(reach_state) <= 512, "reach_state must fit its workspace slot");

__global__ void __launch_bounds__(R_THREADS)
k_r_init(uint32_t words, uint32_t const* __restrict__ und, uint32_t* __restrict__ cand, uint32_t* __restrict__ vis_a, uint32_t* __restrict__ vis_b, reach_state* st)
{
  for (uint32_t w = blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) {
    cand[w]  = und[w];
    vis_a[w] = 0;
    vis_b[w] = 0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->n_und = 0;
    st->m_out = st->m_in = 0;
    st->edges_td = st->edges_bu = st->cands_bu = 0;
    st->err                                    = 0;
    st->decided                                = 0;
    st->levels_fw = st->bu_fw = st->levels_bw = st->bu_bw = 0;
  }
}

// n_und, and the out-/in-degree sums of undecided vertices.
__global__ void __launch_bounds__(R_THREADS)
k_und_degrees(uint32_t n, uint32_t const* __restrict__ und, uint64_t const* __restrict__ fh, uint64_t const* __restrict__ bh, reach_state* st)
{
  uint64_t       so = 0, si = 0;
  uint32_t       c  = 0;
  unsigned const lane = threadIdx.x & 31u;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; t < n; t += static_cast<uint64_t>(gridDim.x) * R_THREADS) {
    uint32_t const v = static_cast<uint32_t>(t);
    if (!bit_get(und, v)) continue;
    ++c;
    so += fh[v + 1] - fh[v];
    si += bh[v + 1] - bh[v];
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    c += __shfl_down_sync(0xFFFFFFFFu, c, s);
    so += __shfl_down_sync(0xFFFFFFFFu, so, s);
    si += __shfl_down_sync(0xFFFFFFFFu, si, s);
  }
  if (lane == 0) {
    if (c) atomicAdd(&st->n_und, c);
    if (so) atomicAdd(&st->m_out, static_cast<unsigned long long>(so));
    if (si) atomicAdd(&st->m_in, static_cast<unsigned long long>(si));
  }
}

// Starts a search at the pivot: taken from `avail`, set in `mark`.
template<bool BW>
__global__ void
k_r_seed(uint32_t* avail, uint32_t* mark, uint32_t* q0, reach_state* st)
{
  uint32_t const p = st->pivot;
  uint32_t const m = 1u << (p & 31);
  avail[p >> 5] &= ~m;
  mark[p >> 5] |= m;
  q0[0]     = p;
  st->qn[0] = 1;
  st->qn[1] = 0;
  st->cur   = 0;
  st->level = 0;
  st->bu    = 0;
  st->mode  = 0;
  st->m_u   = BW ? st->m_in : st->m_out;
}

// Before the frontier scan: a bottom-up search whose frontier is still
// large stays bottom-up and needs no scan (scan = 0); otherwise scan = 1 and
// the direction is settled after the scan by k_r_decide.
__global__ void
k_r_prescan(reach_state* st)
{
  uint32_t const qn = st->qn[st->cur & 1u];
  st->scan          = !(st->mode == 1 && static_cast<unsigned long long>(qn) * st->beta >= st->n_und);
  st->m_f           = 0;
  st->qn[(st->cur & 1u) ^ 1u] = 0;
}

__global__ void
k_r_decide(reach_state* st)
{
  if (!st->scan) return; // stays bottom-up
  unsigned long long const mf = st->m_f;
  if (st->mode == 0 && mf * st->alpha > st->m_u) st->mode = 1;
  else if (st->mode == 1) st->mode = 0; // frontier fell below n_und / beta
  if (st->mode == 0) st->edges_td += mf;
}

template<bool BW>
__global__ void
k_r_advance(reach_state* st, cudaGraphConditionalHandle h, int in_graph)
{
  unsigned long long const mf = st->m_f;
  st->m_u                     = st->m_u > mf ? st->m_u - mf : 0;
  st->level += 1;
  st->bu += st->mode;
  st->cur ^= 1u;
  unsigned cond = st->qn[st->cur & 1u] > 0;
  if (cond && st->level >= st->cap) {
    st->err = 1;
    cond    = 0;
  }
  if (!cond) {
    if (BW) st->levels_bw = st->level, st->bu_bw = st->bu;
    else st->levels_fw = st->level, st->bu_fw = st->bu;
  }
  if (in_graph) cudaGraphSetConditional(h, cond);
}

// top-down, both directions: v joins when its bit in `avail` is taken
struct take_op
{
  uint32_t* avail; // FW: cand; BW: vis_a
  uint32_t* mark;  // FW: vis_a; BW: vis_b
  __device__ __forceinline__ bool operator()(uint32_t, uint32_t v, bool valid) const
  {
    if (!valid || !bit_get(avail, v) || !bit_take(avail, v)) return false;
    bit_claim(mark, v);
    return true;
  }
};

// Bottom-up sweep: candidates are the set bits of `avail`; a candidate
// joins (taken from avail, set in mark, queued) when a neighbour in its
// `head/adj` row is in `mark`.
//  * Compaction: a block reads BU_WORDS bitmap words (one per thread), and a
//    block scan of their popcounts packs the candidate ids into shared
//    memory, so a sweep over few candidates costs about one pass over the
//    bitmap and lanes never idle on non-candidates.
//  * Each thread then carries BU_ILP candidates at once (interleaved row
//    walks) so their dependent loads overlap; a row with no visited
//    neighbour among its first R_BIG entries is finished by the whole warp.
constexpr int BU_WORDS = R_THREADS;

__global__ void __launch_bounds__(R_THREADS)
k_bottom_up(uint32_t n,
            uint64_t const* __restrict__ head,
            uint32_t const* __restrict__ adj,
            uint32_t* __restrict__ avail,
            uint32_t* __restrict__ mark,
            fio f,
            gate g,
            reach_state* st)
{
  if (g.closed()) return;
  __shared__ uint32_t s_cand[BU_WORDS * 32];
  __shared__ uint32_t s_found[BU_WORDS];
  __shared__ uint32_t s_buf[BU_BUF];
  __shared__ uint32_t s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  uint32_t* const qout   = f.out();
  uint32_t* const qout_n = f.out_n();
  block_queue     bq{ s_buf, &s_n };
  unsigned const  lane  = threadIdx.x & 31u;
  uint32_t const  words = (n + 31) / 32;
  uint64_t        nedge = 0, ncand = 0;
  for (uint32_t wbase = blockIdx.x * BU_WORDS; wbase < words; wbase += gridDim.x * BU_WORDS) {
    // 1. pack this chunk's candidates
    uint32_t const w    = wbase + threadIdx.x;
    uint32_t       word = w < words ? avail[w] : 0u;
    s_found[threadIdx.x] = 0;
    if (w == words - 1 && (n & 31)) word &= (1u << (n & 31)) - 1u;
    uint32_t       total;
    uint32_t       j = block_exclusive_scan<uint32_t, R_THREADS>(static_cast<uint32_t>(__popc(word)), &total);
    while (word) {
      uint32_t const b = __ffs(word) - 1;
      word &= word - 1;
      s_cand[j++] = w * 32 + b;
    }
    __syncthreads();
    ncand += threadIdx.x == 0 ? total : 0;
    // 2. walk the packed candidates, BU_ILP per thread
    for (uint32_t r = 0; r < total; r += R_THREADS * BU_ILP) {
      uint32_t v[BU_ILP];
      uint64_t b[BU_ILP], e[BU_ILP];
      bool     live[BU_ILP], found[BU_ILP];
#pragma unroll
      for (int k = 0; k < BU_ILP; ++k) {
        uint32_t const i = r + k * R_THREADS + threadIdx.x;
        live[k]          = i < total;
        v[k]             = live[k] ? s_cand[i] : 0u;
        b[k] = e[k] = 0;
        if (live[k]) b[k] = head[v[k]], e[k] = head[v[k] + 1];
        found[k] = false;
      }
      // interleaved walks: every candidate checks up to R_BIG neighbours
      // itself (most meet a visited one within the first few)
      for (int step_i = 0; step_i < R_BIG; ++step_i) {
        bool any = false;
#pragma unroll
        for (int k = 0; k < BU_ILP; ++k) {
          if (live[k] && b[k] < e[k]) {
            uint32_t const x = adj[b[k]++];
            ++nedge;
            if (bit_get(mark, x)) found[k] = true, live[k] = false;
            any = true;
          } else {
            live[k] = false;
          }
        }
        if (!any) break;
      }
      // rows still open after R_BIG neighbours: the whole warp, one at a time
#pragma unroll
      for (int k = 0; k < BU_ILP; ++k) {
        bool const open = live[k] && b[k] < e[k];
        unsigned   todo = __ballot_sync(0xFFFFFFFFu, open);
        while (todo) {
          unsigned const l = __ffs(todo) - 1;
          todo &= todo - 1;
          uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, b[k], l), e0 = __shfl_sync(0xFFFFFFFFu, e[k], l);
          bool           hit = false;
          for (uint64_t x = b0; x < e0; x += 32) {
            bool const in   = x + lane < e0;
            bool const mine = in && bit_get(mark, adj[x + lane]);
            nedge += in;
            if (__any_sync(0xFFFFFFFFu, mine)) {
              hit = true;
              break;
            }
          }
          if (lane == l) found[k] = hit;
        }
      }
      // a candidate belongs to this block's chunk only, so its bits can be
      // collected in shared memory and written once per word below
#pragma unroll
      for (int k = 0; k < BU_ILP; ++k) {
        if (found[k]) atomicOr(&s_found[(v[k] >> 5) - wbase], 1u << (v[k] & 31));
        bq.push(found[k], v[k]);
      }
      __syncthreads();
      if (s_n > BU_BUF - R_THREADS * BU_ILP) bq.flush(qout, qout_n, &s_base);
    }
    __syncthreads(); // s_found complete; s_cand is rewritten by the next chunk
    if (w < words && s_found[threadIdx.x]) {
      // word w is written by this thread only (chunks are disjoint); other
      // blocks may read it concurrently, which only delays their hits
      avail[w] &= ~s_found[threadIdx.x];
      mark[w] |= s_found[threadIdx.x];
    }
  }
  bq.flush(qout, qout_n, &s_base);
#pragma unroll
  for (int s = 16; s; s >>= 1) nedge += __shfl_down_sync(0xFFFFFFFFu, nedge, s);
  if (lane == 0 && nedge) atomicAdd(&st->edges_bu, static_cast<unsigned long long>(nedge));
  if (threadIdx.x == 0 && ncand) atomicAdd(&st->cands_bu, static_cast<unsigned long long>(ncand));
}

__global__ void
k_r_setid(reach_state* st)
{
  st->id = st->min_ids ? UNDECIDED : st->pivot;
}

// Smallest member of the SCC (first set bit of vis_b) into st->id when
// min_ids is set; one atomic per block.
__global__ void __launch_bounds__(R_THREADS)
k_bitmap_min(uint32_t n, uint32_t const* __restrict__ bm, reach_state* st)
{
  if (!st->min_ids) return;
  __shared__ uint32_t s_min;
  if (threadIdx.x == 0) s_min = UNDECIDED;
  __syncthreads();
  uint32_t const words = (n + 31) / 32;
  uint32_t       best  = UNDECIDED;
  for (uint32_t w = blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) {
    uint32_t const s = bm[w];
    if (s) {
      best = min(best, w * 32 + (__ffs(s) - 1));
      break; // later words of this thread only hold larger ids
    }
  }
  best = __reduce_min_sync(0xFFFFFFFFu, best);
  if ((threadIdx.x & 31) == 0 && best != UNDECIDED) atomicMin(&s_min, best);
  __syncthreads();
  if (threadIdx.x == 0 && s_min != UNDECIDED) atomicMin(&st->id, s_min);
}

// The SCC is vis_b: it leaves the undecided set with id st->id.  One
// thread per bitmap word, so no atomics on und.
__global__ void __launch_bounds__(R_THREADS)
k_fwbw_finalize(uint32_t n, uint32_t const* __restrict__ vis_b, uint32_t* __restrict__ und, uint32_t* __restrict__ scc_id, reach_state* st)
{
  uint32_t const words = (n + 31) / 32;
  uint32_t const id    = st->id;
  uint32_t       c     = 0;
  for (uint32_t w = blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) {
    uint32_t s = vis_b[w];
    if (!s) continue;
    und[w] &= ~s;
    c += __popc(s);
    while (s) {
      uint32_t const b = __ffs(s) - 1;
      s &= s - 1;
      scc_id[w * 32 + b] = id;
    }
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, sh);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&st->decided, c);
}

// ---------------------------------------------------------------- graph building
// Adds kernel `fn` with arguments `vals` (converted to the kernel's
// parameter types) to graph g after `dep`.
template<typename... KArgs, typename... Vals>
cudaGraphNode_t
add_kernel(cudaGraph_t g, cudaGraphNode_t dep, void (*fn)(KArgs...), unsigned grid, unsigned block, Vals... vals)
{
  static_assert(sizeof...(KArgs) == sizeof...(Vals), "argument count");
  std::tuple<std::decay_t<KArgs>...> held(static_cast<std::decay_t<KArgs>>(vals)...);
  void*                              params[sizeof...(KArgs) ? sizeof...(KArgs) : 1];
  std::apply(
    [&](auto&... a) {
      int i = 0;
      ((params[i++] = static_cast<void*>(&a)), ...);
    },
    held);
  cudaKernelNodeParams p = {};
  p.func                 = reinterpret_cast<void*>(fn);
  p.gridDim              = dim3(grid);
  p.blockDim             = dim3(block);
  p.sharedMemBytes       = 0;
  p.kernelParams         = params;
  cudaGraphNode_t node   = nullptr;
  KSPN_CUDA(cudaGraphAddKernelNode(&node, g, dep ? &dep : nullptr, dep ? 1 : 0, &p));
  return node;
}

struct search_io
{
  uint64_t const* td_head;
  uint32_t const* td_adj;
  uint64_t const* bu_head;
  uint32_t const* bu_adj;
  uint32_t*       avail;
  uint32_t*       mark;
};

// The kernels of one level, in order: into graph g (a while-body) when g is
// given, else launched on the stream with the expansion kernels bracketed
// by the profiling events.
template<bool BW>
void
level_body(kspn_context* ctx, cudaGraph_t g, dgraph const& gr, search_io const& io, reach_state* st, cudaGraphConditionalHandle h)
{
  auto&     ws = ctx->ws;
  fio const f{ ws.q0, ws.q1, &st->qn[0], &st->qn[1], &st->cur };
  if (g) {
    cudaGraphNode_t dep = nullptr;
    gate const      sg{ &st->scan, 1 };
    dep                 = add_kernel(g, dep, &k_r_prescan, 1, 1, st);
    dep                 = add_kernel(g, dep, &k_fs_reduce, FS_BLOCKS, FS_THREADS, io.td_head, f, ws.blocks, sg);
    dep                 = add_kernel(g, dep, &k_fs_partials, 1, 1024, ws.blocks, ws.prefix, f, &st->ntiles, static_cast<unsigned long long*>(nullptr), &st->m_f, sg);
    dep                 = add_kernel(g, dep, &k_fs_down, FS_BLOCKS, FS_THREADS, io.td_head, f, ws.blocks, ws.prefix, ws.tile_start, sg);
    dep                 = add_kernel(g, dep, &k_r_decide, 1, 1, st);
    dep = add_kernel(g, dep, &k_expand<take_op>, EX_BLOCKS, EX_THREADS, io.td_head, io.td_adj, f, ws.prefix, ws.tile_start, &st->ntiles, gate{ &st->mode, 0 }, take_op{ io.avail, io.mark });
    dep = add_kernel(g, dep, &k_bottom_up, bu_grid(gr.n), R_THREADS, gr.n, io.bu_head, io.bu_adj, io.avail, io.mark, f, gate{ &st->mode, 1 }, st);
    add_kernel(g, dep, &k_r_advance<BW>, 1, 1, st, h, 1);
    return;
  }
  cudaStream_t const s = ctx->stream;
  gate const         sg{ &st->scan, 1 };
  k_r_prescan<<<1, 1, 0, s>>>(st);
  k_fs_reduce<<<FS_BLOCKS, FS_THREADS, 0, s>>>(io.td_head, f, ws.blocks, sg);
  k_fs_partials<<<1, 1024, 0, s>>>(ws.blocks, ws.prefix, f, &st->ntiles, nullptr, &st->m_f, sg);
  k_fs_down<<<FS_BLOCKS, FS_THREADS, 0, s>>>(io.td_head, f, ws.blocks, ws.prefix, ws.tile_start, sg);
  k_r_decide<<<1, 1, 0, s>>>(st);
  prof_start(ctx, 0);
  k_expand<take_op><<<EX_BLOCKS, EX_THREADS, 0, s>>>(io.td_head, io.td_adj, f, ws.prefix, ws.tile_start, &st->ntiles, gate{ &st->mode, 0 }, take_op{ io.avail, io.mark });
  prof_stop(ctx, 0);
  prof_start(ctx, 1);
  k_bottom_up<<<bu_grid(gr.n), R_THREADS, 0, s>>>(gr.n, io.bu_head, io.bu_adj, io.avail, io.mark, f, gate{ &st->mode, 1 }, st);
  prof_stop(ctx, 1);
  k_r_advance<BW><<<1, 1, 0, s>>>(st, h, 0);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 8;
}

search_io
fw_io(kspn_context* ctx, dgraph const& g)
{
  return { g.fh, g.fc, g.bh, g.bc, ctx->ws.mark, ctx->ws.vis_a };
}
search_io
bw_io(kspn_context* ctx, dgraph const& g)
{
  return { g.bh, g.bc, g.fh, g.fc, ctx->ws.vis_a, ctx->ws.vis_b };
}

// Builds the one-launch FW-BW graph for (graph, und, scc_id).
void
build_fwbw_graph(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id)
{
  auto&          ws    = ctx->ws;
  auto*          st    = reinterpret_cast<reach_state*>(ws.rstate);
  uint32_t const words = (g.n + 31) / 32;
  cudaGraph_t    graph = nullptr;
  KSPN_CUDA(cudaGraphCreate(&graph, 0));
  try {
    cudaGraphNode_t dep = nullptr;
    dep = add_kernel(graph, dep, &k_r_init, r_grid(words), R_THREADS, words, und, ws.mark, ws.vis_a, ws.vis_b, st);
    dep = add_kernel(graph, dep, &k_und_degrees, r_grid(g.n), R_THREADS, g.n, und, g.fh, g.bh, st);
    for (int bw = 0; bw < 2; ++bw) {
      search_io const io = bw ? bw_io(ctx, g) : fw_io(ctx, g);
      dep = bw ? add_kernel(graph, dep, &k_r_seed<true>, 1, 1, io.avail, io.mark, ws.q0, st) : add_kernel(graph, dep, &k_r_seed<false>, 1, 1, io.avail, io.mark, ws.q0, st);
      cudaGraphConditionalHandle h;
      KSPN_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp = {};
      cp.type                = cudaGraphNodeTypeConditional;
      cp.conditional.handle  = h;
      cp.conditional.type    = cudaGraphCondTypeWhile;
      cp.conditional.size    = 1;
      cudaGraphNode_t loop   = nullptr;
      KSPN_CUDA(cudaGraphAddNode(&loop, graph, &dep, 1, &cp));
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      if (bw) level_body<true>(ctx, body, g, io, st, h);
      else level_body<false>(ctx, body, g, io, st, h);
      dep = loop;
    }
    dep = add_kernel(graph, dep, &k_r_setid, 1, 1, st);
    dep = add_kernel(graph, dep, &k_bitmap_min, r_grid(words), R_THREADS, g.n, ws.vis_b, st);
    add_kernel(graph, dep, &k_fwbw_finalize, r_grid(words), R_THREADS, g.n, ws.vis_b, und, scc_id, st);
    cudaGraphExec_t exec = nullptr;
    KSPN_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    ctx->fwbw.graph = graph;
    ctx->fwbw.exec  = exec;
  } catch (...) {
    cudaGraphDestroy(graph);
    throw;
  }
}

} // namespace

size_t
reach_state_bytes()
{
  return sizeof(reach_state);
}

void
release_graphs(kspn_context* ctx)
{
  if (ctx->fwbw.exec) cudaGraphExecDestroy(ctx->fwbw.exec);
  if (ctx->fwbw.graph) cudaGraphDestroy(ctx->fwbw.graph);
  ctx->fwbw = {};
}

uint32_t
fw_bw(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t pivot, kspn_options const& opt, kspn_stats* st, bool min_ids)
{
  auto& ws = ctx->ws;
  if (pivot >= g.n) throw error{ KSPN_ERR_INVALID_ARGUMENT, "forward_backward_search: pivot >= n" };
  auto* rs = reinterpret_cast<reach_state*>(ws.rstate);
  auto* hs = reinterpret_cast<reach_state*>(ctx->h_state);
  // parameters of this search
  std::memset(hs, 0, sizeof(reach_state));
  hs->pivot   = pivot;
  hs->cap     = opt.max_levels ? opt.max_levels : g.n + 2;
  hs->alpha   = opt.bu_enter_div ? opt.bu_enter_div : 1;
  hs->beta    = opt.bu_leave_div ? opt.bu_leave_div : 1;
  hs->min_ids = min_ids ? 1u : 0u;
  KSPN_CUDA(cudaMemcpyAsync(rs, hs, sizeof(reach_state), cudaMemcpyHostToDevice, ctx->stream));

  if (!ctx->prof) {
    graph_key const key{ g.fh, g.fc, g.bh, g.bc, und, scc_id, ws.base, g.n, g.m };
    if (!ctx->fwbw.exec || !(ctx->fwbw.key == key)) {
      release_graphs(ctx);
      build_fwbw_graph(ctx, g, und, scc_id);
      ctx->fwbw.key = key;
    }
    KSPN_CUDA(cudaGraphLaunch(ctx->fwbw.exec, ctx->stream));
  } else {
    // host-driven loop over the same kernels, expansion kernels bracketed
    // by CUDA events (kspn_options.profile)
    bool const     trace_done = st && st->levels_fw != 0; // trace the first FW-BW only
    uint32_t const words      = (g.n + 31) / 32;
    k_r_init<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(words, und, ws.mark, ws.vis_a, ws.vis_b, rs);
    k_und_degrees<<<r_grid(g.n), R_THREADS, 0, ctx->stream>>>(g.n, und, g.fh, g.bh, rs);
    ctx->launches += 2;
    for (int bw = 0; bw < 2; ++bw) {
      search_io const io = bw ? bw_io(ctx, g) : fw_io(ctx, g);
      if (bw) k_r_seed<true><<<1, 1, 0, ctx->stream>>>(io.avail, io.mark, ws.q0, rs);
      else k_r_seed<false><<<1, 1, 0, ctx->stream>>>(io.avail, io.mark, ws.q0, rs);
      ctx->launches += 1;
      for (;;) {
        KSPN_CUDA(cudaMemcpyAsync(hs, rs, sizeof(reach_state), cudaMemcpyDeviceToHost, ctx->stream));
        KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
        uint32_t const           qn0 = hs->qn[hs->cur & 1u];
        unsigned long long const e0 = hs->edges_bu, c0 = hs->cands_bu;
        if (qn0 == 0 || hs->err) break;
        if (hs->level >= hs->cap) {
          hs->err = 1;
          break;
        }
        if (bw) level_body<true>(ctx, nullptr, g, io, rs, cudaGraphConditionalHandle{});
        else level_body<false>(ctx, nullptr, g, io, rs, cudaGraphConditionalHandle{});
        KSPN_CUDA(cudaMemcpyAsync(hs, rs, sizeof(reach_state), cudaMemcpyDeviceToHost, ctx->stream));
        KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
        uint32_t const qn1 = hs->qn[hs->cur & 1u];
        float          ms  = 0;
        if (hs->mode == 0) ms = prof_add(ctx, 0, KSPN_KERNEL_EXPAND, expand_bytes(qn0, hs->m_f, qn1, 4));
        // bottom-up: candidate sweep reads the avail bitmap (n/8 B), then per
        // candidate its offset pair, per edge id + probe, per join queue
        // entry + two bit writes
        else ms = prof_add(ctx, 1, KSPN_KERNEL_BOTTOM_UP, static_cast<uint64_t>(g.n) / 8 + 16 * (hs->cands_bu - c0) + 8 * (hs->edges_bu - e0) + 8ull * qn1);
        if (st && st->trace_levels < 32 && !trace_done) {
          auto& t          = st->trace[st->trace_levels++];
          t.backward       = static_cast<uint32_t>(bw);
          t.bottom_up      = hs->mode;
          t.frontier       = qn0;
          t.discovered     = qn1;
          t.frontier_edges = hs->m_f;
          t.scanned        = hs->mode ? hs->edges_bu - e0 : hs->m_f;
          t.candidates     = hs->mode ? hs->cands_bu - c0 : 0;
          t.ms             = ms;
        }
      }
      if (hs->err) break;
    }
    if (hs->err) throw error{ KSPN_ERR_TIMEOUT, "reachability: level cap exceeded" };
    k_r_setid<<<1, 1, 0, ctx->stream>>>(rs);
    k_bitmap_min<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(g.n, ws.vis_b, rs);
    k_fwbw_finalize<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(g.n, ws.vis_b, und, scc_id, rs);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 3;
  }
  KSPN_CUDA(cudaMemcpyAsync(hs, rs, sizeof(reach_state), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  if (hs->err) throw error{ KSPN_ERR_TIMEOUT, "reachability: level cap exceeded" };
  // kernels the graph ran: init, degrees, 2 seeds, 8 per level, 3 to finish
  if (!ctx->prof) ctx->launches += 7 + 8ull * (hs->levels_fw + hs->levels_bw);
  ctx->td_edges += hs->edges_td + hs->edges_bu;
  if (st && st->levels_fw == 0 && st->levels_bw == 0) {
    st->levels_fw        = hs->levels_fw;
    st->levels_bw        = hs->levels_bw;
    st->levels_bottom_up = hs->bu_fw + hs->bu_bw;
  }
  return hs->decided;
}

} // namespace kspn
