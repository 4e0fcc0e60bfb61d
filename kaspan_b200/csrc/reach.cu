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
// Level control lives on the device (reach_state).  Each search is ONE
// persistent cooperative launch (k_search) whose blocks run every level:
// frontier scan, direction choice, top-down tiles or bottom-up chunks, and
// the queue flip, separated by a bounded grid barrier.  With profiling on,
// the same phase bodies run as separate launches from a host loop
// (decide / expand / bottom-up / advance kernels) with CUDA events around
// the expansion kernels.
#include "expand.cuh"

#include <algorithm>
#include <cstring>
#include <tuple>

namespace kspn {

namespace {

constexpr int R_THREADS = 256;
constexpr int BU_BUF    = 2048;
constexpr int BU_ILP    = 4;

unsigned
r_grid(uint64_t items)
{
  uint64_t const b = (items + R_THREADS - 1) / R_THREADS;
  return static_cast<unsigned>(b < 148ull * 8 ? (b ? b : 1) : 148ull * 8);
}

// bottom-up: one block per (8 warps x 32 bitmap words), capped at the
// resident-block count
unsigned
bu_grid(uint32_t n)
{
  uint64_t const chunks = ((static_cast<uint64_t>(n) + 31) / 32 + 32 * (R_THREADS / 32) - 1) / (32 * (R_THREADS / 32));
  return static_cast<unsigned>(chunks < 148ull * 5 ? (chunks ? chunks : 1) : 148ull * 5);
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
  uint32_t           mat;      // 1: build the frontier queue from `fresh` first (bottom-up -> top-down)
  uint32_t           mat_n;    // slots handed out while building it
  uint32_t           levels_fw, bu_fw, levels_bw, bu_bw;
  unsigned long long m_u, m_out, m_in, m_f, alpha, beta;
  unsigned long long edges_td, edges_bu, cands_bu;
  uint32_t           bar_count, bar_gen, bar_err; // grid barrier of the persistent search
  uint32_t           marks;                       // phase stamps taken (kspn_options.trace)
};

// phase stamps live after the state: uint32 phase[128], uint64 ns[128]
constexpr int MARKS = 128;
static_assert(sizeof(reach_state) <= 512, "reach_state must fit its workspace slot");

// Per search pair: cand = und, vis_a = vis_b = 0, n_und = |und| (one
// atomic per warp), and the unexplored-edge bound m_out = m_in = m (Beamer's
// m_u only has to be of the right size: it gates the switch to bottom-up).
__global__ void __launch_bounds__(R_THREADS)
k_r_init(uint32_t words, uint64_t m, uint32_t const* __restrict__ und, uint32_t* __restrict__ cand, uint32_t* __restrict__ vis_a, uint32_t* __restrict__ vis_b, reach_state* st)
{
  uint32_t c = 0;
  for (uint32_t w = blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) {
    uint32_t const u = und[w];
    cand[w]          = u;
    vis_a[w]         = 0;
    vis_b[w]         = 0;
    c += __popc(u);
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, sh);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(&st->n_und, c);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->m_out = st->m_in = m;
    st->edges_td = st->edges_bu = st->cands_bu = 0;
    st->err                                    = 0;
    st->decided                                = 0;
    st->levels_fw = st->bu_fw = st->levels_bw = st->bu_bw = 0;
    st->bar_count = st->bar_gen = st->bar_err = 0;
    st->marks                                 = 0;
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
  st->scan  = 1;
  st->mat   = 0;
  st->m_f   = 0;
}

// Before the frontier scan: a bottom-up search whose frontier is still
// large stays bottom-up and needs no scan (scan = 0); otherwise scan = 1 and
// the direction is settled after the scan by k_r_decide.
__global__ void
k_r_decide(reach_state* st)
{
  if (!st->scan) return; // stays bottom-up
  unsigned long long const mf = st->m_f;
  if (st->mode == 0 && mf * st->alpha > st->m_u) st->mode = 1;
  else if (st->mode == 1) st->mode = 0; // frontier fell below n_und / beta
  if (st->mode == 0) st->edges_td += mf;
}

// End of a level: explored edges, level count, queue flip, cap, and the
// next level's pre-scan step.  Returns the loop condition.
// (state read through L2: counters were updated by other blocks)
template<bool BW>
__device__ __forceinline__ unsigned
advance_body(reach_state* st)
{
  unsigned long long const mf   = __ldcg(&st->m_f);
  unsigned long long const mu   = __ldcg(&st->m_u);
  uint32_t const           mode = __ldcg(&st->mode);
  uint32_t const           lvl  = __ldcg(&st->level) + 1;
  uint32_t const           bu   = __ldcg(&st->bu) + mode;
  uint32_t const           cur  = (__ldcg(&st->cur) ^ 1u) & 1u;
  uint32_t const           qn   = __ldcg(&st->qn[cur]);
  st->m_u                       = mu > mf ? mu - mf : 0;
  st->level                     = lvl;
  st->bu                        = bu;
  st->cur                       = cur;
  unsigned cond                 = qn > 0;
  if (cond && lvl >= __ldcg(&st->cap)) {
    st->err = 1;
    cond    = 0;
  }
  if (!cond) {
    if (BW) st->levels_bw = lvl, st->bu_bw = bu;
    else st->levels_fw = lvl, st->bu_fw = bu;
  } else {
    // the next level's pre-scan step; a bottom-up search about to return
    // top-down first builds its frontier queue from `fresh`
    uint32_t const scan = !(mode == 1 && static_cast<unsigned long long>(qn) * __ldcg(&st->beta) >= __ldcg(&st->n_und));
    st->scan            = scan;
    st->mat             = (mode == 1 && scan) ? 1u : 0u;
    st->mat_n           = 0;
    st->m_f             = 0;
    st->qn[cur ^ 1u]    = 0;
  }
  return cond;
}

template<bool BW>
__global__ void
k_r_advance(reach_state* st)
{
  advance_body<BW>(st);
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
constexpr int BU_WARPS = R_THREADS / 32;
constexpr int BU_STEPS = 32; // neighbours a candidate checks itself before its warp helps

// Per-warp shared memory of the sweep.
struct bu_warp_smem
{
  uint32_t cand[32 * 32]; // the warp's chunk (32 words = 1024 vertices), packed
  uint32_t found[32];     // found bits per word of the chunk
};

// Bottom-up sweep over the chunks of 32 bitmap words given to this warp
// (chunk c = words [32c, 32c + 32), c = first, first + step, ...).
// Candidates are the set bits of `avail`; one joins when a neighbour in its
// head/adj row is in `mark`.  Warps work independently (no block barrier):
// the warp packs its chunk's candidates (popcount scan over its 32 words),
// each lane walks BU_ILP candidates interleaved -- all neighbour loads of a
// step, then all probes -- and rows still open after BU_STEPS neighbours
// are finished by the whole warp with early exit.  Lane i then owns word i
// of the chunk: it clears the found bits from avail, sets them in mark and
// writes the word of `fresh` (the sweep's discoveries).  No queue is
// written; the count goes to *found_count.  `avail` and `mark` are read
// through L2 (other blocks of a persistent launch change them).
__device__ __forceinline__ void
bu_sweep_warp(uint32_t first,
              uint32_t step,
              uint32_t n,
              uint64_t const* __restrict__ head,
              uint32_t const* __restrict__ adj,
              uint32_t* avail,
              uint32_t* mark,
              uint32_t* fresh,
              bu_warp_smem& sm,
              uint32_t& nfound,
              uint64_t& nedge,
              uint64_t& ncand)
{
  unsigned const lane   = threadIdx.x & 31u;
  uint32_t const words  = (n + 31) / 32;
  uint32_t const chunks = (words + 31) / 32;
  for (uint32_t c = first; c < chunks; c += step) {
    uint32_t const w    = c * 32 + lane;
    uint32_t       word = w < words ? __ldcg(avail + w) : 0u;
    if (w == words - 1 && (n & 31)) word &= (1u << (n & 31)) - 1u;
    uint32_t const cnt = __popc(word);
    uint32_t       pos = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, pos, d);
      if (lane >= static_cast<unsigned>(d)) pos += y;
    }
    uint32_t const total = __shfl_sync(0xFFFFFFFFu, pos, 31);
    pos -= cnt;
    while (word) {
      uint32_t const bb = __ffs(word) - 1;
      word &= word - 1;
      sm.cand[pos++] = w * 32 + bb;
    }
    sm.found[lane] = 0;
    __syncwarp();
    ncand += lane == 0 ? total : 0;
    for (uint32_t r = 0; r < total; r += 32 * BU_ILP) {
      uint32_t v[BU_ILP];
      uint64_t b[BU_ILP], e[BU_ILP];
      bool     live[BU_ILP], found[BU_ILP];
#pragma unroll
      for (int k = 0; k < BU_ILP; ++k) {
        uint32_t const i = r + k * 32 + lane;
        live[k]          = i < total;
        v[k]             = live[k] ? sm.cand[i] : 0u;
        b[k] = e[k] = 0;
        if (live[k]) b[k] = head[v[k]], e[k] = head[v[k] + 1];
        found[k] = false;
      }
      for (int s_i = 0; s_i < BU_STEPS; ++s_i) {
        bool     act[BU_ILP];
        uint32_t x[BU_ILP], wd[BU_ILP];
        bool     any = false;
#pragma unroll
        for (int k = 0; k < BU_ILP; ++k) {
          act[k] = live[k] && b[k] < e[k];
          x[k]   = act[k] ? adj[b[k]] : 0u;
          any |= act[k];
        }
        if (!__any_sync(0xFFFFFFFFu, any)) break;
#pragma unroll
        for (int k = 0; k < BU_ILP; ++k) wd[k] = act[k] ? __ldcg(mark + (x[k] >> 5)) : 0u;
#pragma unroll
        for (int k = 0; k < BU_ILP; ++k) {
          if (!act[k]) {
            live[k] = false;
            continue;
          }
          ++b[k];
          ++nedge;
          if ((wd[k] >> (x[k] & 31)) & 1u) found[k] = true, live[k] = false;
        }
      }
      // rows still open: the whole warp, one at a time, with early exit
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
            bool const     in = x + lane < e0;
            uint32_t const y  = in ? adj[x + lane] : 0u;
            bool const     h  = in && ((__ldcg(mark + (y >> 5)) >> (y & 31)) & 1u);
            nedge += in;
            if (__any_sync(0xFFFFFFFFu, h)) {
              hit = true;
              break;
            }
          }
          if (lane == l) found[k] = hit;
        }
      }
#pragma unroll
      for (int k = 0; k < BU_ILP; ++k)
        if (found[k]) atomicOr(&sm.found[(v[k] >> 5) - c * 32], 1u << (v[k] & 31));
    }
    __syncwarp();
    uint32_t const fnd = sm.found[lane];
    if (w < words) {
      if (fnd) {
        atomicAnd(avail + w, ~fnd);
        atomicOr(mark + w, fnd);
      }
      fresh[w] = fnd;
    }
    nfound += __popc(fnd);
    __syncwarp();
  }
}

// Frontier queue from `fresh` (when a search returns to top-down after
// bottom-up sweeps): one bitmap word per thread, block scan, one global
// atomic per block.  All threads of the block call it.
__device__ __forceinline__ void
materialize_block(uint32_t blk, uint32_t nblk, uint32_t n, uint32_t const* fresh, uint32_t* q, uint32_t* qn, uint32_t* s_base)
{
  uint32_t const words = (n + 31) / 32;
  for (uint32_t wbase = blk * R_THREADS; wbase < words; wbase += nblk * R_THREADS) {
    uint32_t const w    = wbase + threadIdx.x;
    uint32_t       word = w < words ? __ldcg(fresh + w) : 0u;
    uint32_t       total;
    uint32_t       off = block_exclusive_scan<uint32_t, R_THREADS>(static_cast<uint32_t>(__popc(word)), &total);
    if (threadIdx.x == 0) *s_base = total ? atomicAdd(qn, total) : 0u;
    __syncthreads();
    uint32_t j = *s_base + off;
    while (word) {
      uint32_t const bb = __ffs(word) - 1;
      word &= word - 1;
      q[j++] = w * 32 + bb;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(R_THREADS)
k_materialize(uint32_t n, uint32_t const* __restrict__ fresh, fio f, reach_state* st)
{
  if (!st->mat) return;
  __shared__ uint32_t s_base;
  // the queue being built is the next level's input; its length is
  // already known (the sweep's count), slots come from mat_n
  materialize_block(blockIdx.x, gridDim.x, n, fresh, const_cast<uint32_t*>(f.in()), &st->mat_n, &s_base);
}

// Bottom-up sweep as its own launch (profiled levels): every chunk once,
// the discovery count into the output counter.
__global__ void __launch_bounds__(R_THREADS)
k_bottom_up(uint32_t n,
            uint64_t const* __restrict__ head,
            uint32_t const* __restrict__ adj,
            uint32_t* __restrict__ avail,
            uint32_t* __restrict__ mark,
            uint32_t* __restrict__ fresh,
            fio f,
            gate g,
            reach_state* st)
{
  if (g.closed()) return;
  __shared__ bu_warp_smem sm[BU_WARPS];
  uint32_t                nfound = 0;
  uint64_t                nedge = 0, ncand = 0;
  unsigned const          wid = threadIdx.x >> 5;
  bu_sweep_warp(blockIdx.x * BU_WARPS + wid, gridDim.x * BU_WARPS, n, head, adj, avail, mark, fresh, sm[wid], nfound, nedge, ncand);
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    nedge += __shfl_down_sync(0xFFFFFFFFu, nedge, s);
    nfound += __shfl_down_sync(0xFFFFFFFFu, nfound, s);
  }
  if ((threadIdx.x & 31) == 0) {
    if (nedge) atomicAdd(&st->edges_bu, static_cast<unsigned long long>(nedge));
    if (nfound) atomicAdd(f.out_n(), nfound);
    if (ncand) atomicAdd(&st->cands_bu, static_cast<unsigned long long>(ncand));
  }
}

// ---------------------------------------------------------------- persistent search
// One whole reachability search (every level) in ONE cooperative launch.
// Blocks meet at a grid barrier between the phases of a level; the barrier
// waits at most GRID_SYNC_SPINS polls, after which it sets bar_err and every
// block leaves (the host reports KSPN_ERR_TIMEOUT) -- a launch whose blocks
// were not all resident could therefore never hang.
constexpr unsigned GRID_SYNC_SPINS = 1u << 22;

__device__ __forceinline__ bool
grid_sync(reach_state* st)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t const g0 = ld_acquire(&st->bar_gen);
    __threadfence();
    if (atomicAdd(&st->bar_count, 1u) == gridDim.x - 1) {
      atomicExch(&st->bar_count, 0u);
      __threadfence();
      atomicAdd(&st->bar_gen, 1u);
    } else {
      unsigned spins = 0;
      while (ld_acquire(&st->bar_gen) == g0) {
        if (++spins > GRID_SYNC_SPINS) {
          atomicExch(&st->bar_err, 1u);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ld_acquire(&st->bar_err) == 0;
}

struct search_args
{
  uint32_t        n;
  uint32_t        trace;  // stamp phases into stamp_phase / stamp_ns
  uint32_t*       stamp_phase;
  uint64_t*       stamp_ns;
  uint64_t const* td_head;
  uint32_t const* td_adj;
  uint64_t const* bu_head;
  uint32_t const* bu_adj;
  uint32_t*       avail;
  uint32_t*       mark;
  uint32_t*       fresh;
  uint32_t*       q0;
  uint32_t*       q1;
  uint64_t*       prefix;
  uint32_t*       tile_start;
  uint64_t*       partial;
  reach_state*    st;
};

__device__ __forceinline__ void
chunk_of(uint32_t qn, uint32_t& beg, uint32_t& end)
{
  uint32_t const chunk = (qn + gridDim.x - 1) / gridDim.x;
  uint64_t const b     = static_cast<uint64_t>(blockIdx.x) * chunk;
  beg                  = static_cast<uint32_t>(b < qn ? b : qn);
  end                  = static_cast<uint32_t>(b + chunk < qn ? b + chunk : qn);
}

__device__ __forceinline__ uint64_t
globaltimer()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// block 0, thread 0: record that `phase` ended now
__device__ __forceinline__ void
stamp(search_args const& a, uint32_t phase)
{
  if (!a.trace || blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t const i = a.st->marks;
  if (i < MARKS) {
    a.stamp_phase[i] = phase;
    a.stamp_ns[i]    = globaltimer();
    a.st->marks      = i + 1;
  }
}

template<bool BW>
__global__ void __launch_bounds__(R_THREADS)
k_search(search_args a)
{
  __shared__ bu_warp_smem sm[BU_WARPS]; // bottom-up warp chunks; sm[0..] also holds a top-down tile's rows
  __shared__ uint32_t     s_buf[BU_BUF];
  __shared__ uint32_t     s_i[2], s_n, s_base;
  static_assert(sizeof(sm) >= EX_TILE * sizeof(uint32_t), "tile rows must fit the warp buffers");
  uint32_t* const tile_rows = reinterpret_cast<uint32_t*>(sm);
  reach_state* const  st = a.st;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  block_queue    bq{ s_buf, &s_n };
  uint64_t       nedge = 0, ncand = 0;
  uint32_t       nfound = 0;
  for (;;) {
    // control values, written by block 0 before the last barrier
    uint32_t const cur = __ldcg(&st->cur) & 1u;
    uint32_t const qn  = __ldcg(&st->qn[cur]);
    if (qn == 0 || __ldcg(&st->err)) break;
    if (__ldcg(&st->mat)) {
      // back to top-down: the frontier queue from the last sweep's bits
      materialize_block(blockIdx.x, gridDim.x, a.n, a.fresh, cur ? a.q1 : a.q0, &st->mat_n, &s_base);
      if (!grid_sync(st)) break;
      stamp(a, 7);
    }
    uint32_t const* qin    = cur ? a.q1 : a.q0;
    uint32_t* const qout   = cur ? a.q0 : a.q1;
    uint32_t* const qout_n = &st->qn[cur ^ 1u];
    if (__ldcg(&st->scan)) {
      // degrees of the frontier (top-down direction): block partial sums
      uint32_t beg, end;
      chunk_of(qn, beg, end);
      uint64_t sum = 0;
      for (uint32_t i = beg + threadIdx.x; i < end; i += R_THREADS) {
        uint32_t const v = __ldcg(qin + i);
        sum += a.td_head[v + 1] - a.td_head[v];
      }
      uint64_t total;
      block_exclusive_scan<uint64_t, R_THREADS>(sum, &total);
      if (threadIdx.x == 0) a.partial[blockIdx.x] = total;
      if (!grid_sync(st)) break;
      stamp(a, 1);
      // block 0: scan of the partial sums, totals, direction
      if (blockIdx.x == 0) {
        uint32_t const nb  = gridDim.x;
        uint32_t const per = (nb + R_THREADS - 1) / R_THREADS;
        uint32_t const b0  = threadIdx.x * per;
        uint64_t       loc = 0;
        for (uint32_t i = b0; i < b0 + per && i < nb; ++i) loc += __ldcg(a.partial + i);
        uint64_t all;
        uint64_t run = block_exclusive_scan<uint64_t, R_THREADS>(loc, &all);
        for (uint32_t i = b0; i < b0 + per && i < nb; ++i) {
          uint64_t const x = __ldcg(a.partial + i);
          a.partial[i]     = run;
          run += x;
        }
        if (threadIdx.x == 0) {
          a.prefix[qn]    = all;
          st->ntiles      = static_cast<uint32_t>((all + EX_TILE - 1) / EX_TILE);
          st->m_f         = all;
          uint32_t mode   = __ldcg(&st->mode);
          if (mode == 0 && all * __ldcg(&st->alpha) > __ldcg(&st->m_u)) mode = 1;
          else if (mode == 1) mode = 0; // the frontier fell below n_und / beta
          st->mode = mode;
          if (mode == 0) st->edges_td = __ldcg(&st->edges_td) + all;
        }
      }
      if (!grid_sync(st)) break;
      stamp(a, 2);
      if (__ldcg(&st->mode) == 0) {
        // frontier prefix and tile starts
        uint64_t run = __ldcg(a.partial + blockIdx.x);
        for (uint32_t base = beg; base < end; base += R_THREADS) {
          uint32_t const i   = base + threadIdx.x;
          uint64_t       deg = 0;
          if (i < end) {
            uint32_t const v = __ldcg(qin + i);
            deg              = a.td_head[v + 1] - a.td_head[v];
          }
          uint64_t       tot;
          uint64_t const p = run + block_exclusive_scan<uint64_t, R_THREADS>(deg, &tot);
          if (i < end) {
            a.prefix[i] = p;
            if (deg) {
              uint64_t const t0 = (p + EX_TILE - 1) / EX_TILE;
              uint64_t const t1 = (p + deg - 1) / EX_TILE;
              for (uint64_t t = t0; t <= t1; ++t) a.tile_start[t] = i;
            }
          }
          run += tot;
        }
        if (!grid_sync(st)) break;
        stamp(a, 3);
      }
    }
    uint32_t const phase = __ldcg(&st->mode) == 0 ? 4u : 5u;
    if (__ldcg(&st->mode) == 0) {
      uint32_t const ntiles = __ldcg(&st->ntiles);
      uint64_t const total  = __ldcg(a.prefix + qn);
      take_op const  op{ a.avail, a.mark };
      for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        expand_tile(tile, ntiles, qin, qn, total, a.prefix, a.tile_start, a.td_head, a.td_adj, tile_rows, s_i, bq, op);
        bq.flush(qout, qout_n, &s_base);
      }
    } else {
      unsigned const wid = threadIdx.x >> 5;
      nfound             = 0;
      bu_sweep_warp(blockIdx.x * BU_WARPS + wid, gridDim.x * BU_WARPS, a.n, a.bu_head, a.bu_adj, a.avail, a.mark, a.fresh, sm[wid], nfound, nedge, ncand);
#pragma unroll
      for (int sh = 16; sh; sh >>= 1) nfound += __shfl_down_sync(0xFFFFFFFFu, nfound, sh);
      if ((threadIdx.x & 31) == 0 && nfound) atomicAdd(qout_n, nfound);
    }
    if (!grid_sync(st)) break;
    stamp(a, phase);
    if (blockIdx.x == 0 && threadIdx.x == 0) advance_body<BW>(st);
    if (!grid_sync(st)) break;
    stamp(a, 6);
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) nedge += __shfl_down_sync(0xFFFFFFFFu, nedge, sh);
  if ((threadIdx.x & 31) == 0 && nedge) atomicAdd(&st->edges_bu, static_cast<unsigned long long>(nedge));
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

struct search_io
{
  uint64_t const* td_head;
  uint32_t const* td_adj;
  uint64_t const* bu_head;
  uint32_t const* bu_adj;
  uint32_t*       avail;
  uint32_t*       mark;
  uint32_t*       fresh;
};

// One level as separate launches (profiled searches): the same phase
// bodies as k_search, with CUDA events around the two expansion kernels.
template<bool BW>
void
level_body(kspn_context* ctx, dgraph const& gr, search_io const& io, reach_state* st)
{
  auto&              ws = ctx->ws;
  fio const          f{ ws.q0, ws.q1, &st->qn[0], &st->qn[1], &st->cur };
  cudaStream_t const s = ctx->stream;
  gate const         sg{ &st->scan, 1 };
  k_materialize<<<r_grid((gr.n + 31) / 32), R_THREADS, 0, s>>>(gr.n, io.fresh, f, st);
  k_fs_reduce<<<FS_BLOCKS, FS_THREADS, 0, s>>>(io.td_head, f, ws.blocks, sg);
  k_fs_partials<<<1, 1024, 0, s>>>(ws.blocks, ws.prefix, f, &st->ntiles, nullptr, &st->m_f, sg);
  k_fs_down<<<FS_BLOCKS, FS_THREADS, 0, s>>>(io.td_head, f, ws.blocks, ws.prefix, ws.tile_start, sg);
  k_r_decide<<<1, 1, 0, s>>>(st);
  prof_start(ctx, 0);
  k_expand<take_op><<<EX_BLOCKS, EX_THREADS, 0, s>>>(io.td_head, io.td_adj, f, ws.prefix, ws.tile_start, &st->ntiles, gate{ &st->mode, 0 }, take_op{ io.avail, io.mark });
  prof_stop(ctx, 0);
  prof_start(ctx, 1);
  k_bottom_up<<<bu_grid(gr.n), R_THREADS, 0, s>>>(gr.n, io.bu_head, io.bu_adj, io.avail, io.mark, io.fresh, f, gate{ &st->mode, 1 }, st);
  prof_stop(ctx, 1);
  k_r_advance<BW><<<1, 1, 0, s>>>(st);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 8;
}

search_io
fw_io(kspn_context* ctx, dgraph const& g)
{
  return { g.fh, g.fc, g.bh, g.bc, ctx->ws.mark, ctx->ws.vis_a, ctx->ws.fresh };
}
search_io
bw_io(kspn_context* ctx, dgraph const& g)
{
  return { g.bh, g.bc, g.fh, g.fc, ctx->ws.vis_a, ctx->ws.vis_b, ctx->ws.fresh };
}

// Cooperative launch of one persistent search: as many blocks as fit on
// the device at once (all co-resident, which the grid barrier needs).
template<bool BW>
void
launch_search(kspn_context* ctx, search_args const& a)
{
  static int bps = 0, sms = 0;
  if (!bps) {
    KSPN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_search<BW>, R_THREADS, 0));
    KSPN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (bps < 1) throw error{ KSPN_ERR_CUDA, "persistent search kernel does not fit on an SM" };
  }
  unsigned const grid = static_cast<unsigned>(std::min(bps * sms, 4000));
  search_args    arg  = a;
  void*          args[] = { &arg };
  KSPN_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void const*>(&k_search<BW>), dim3(grid), dim3(R_THREADS), args, 0, ctx->stream));
  ctx->launches += 1;
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
  for (cached_graph* c : { &ctx->fwbw, &ctx->trim }) {
    if (c->exec) cudaGraphExecDestroy(c->exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    *c = {};
  }
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

  uint32_t const words = (g.n + 31) / 32;
  if (!ctx->prof) {
    // whole searches on the device: one cooperative launch per direction
    k_r_init<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(words, g.m, und, ws.mark, ws.vis_a, ws.vis_b, rs);
    ctx->launches += 1;
    for (int bw = 0; bw < 2; ++bw) {
      search_io const io = bw ? bw_io(ctx, g) : fw_io(ctx, g);
      auto* stamp_phase = reinterpret_cast<uint32_t*>(static_cast<char*>(ws.rstate) + 2048);
      auto* stamp_ns    = reinterpret_cast<uint64_t*>(static_cast<char*>(ws.rstate) + 2048 + 4 * MARKS);
      bool const tr     = opt.trace && st && st->search_marks == 0;
      search_args const a{ g.n, tr ? 1u : 0u, stamp_phase, stamp_ns, io.td_head, io.td_adj, io.bu_head, io.bu_adj, io.avail, io.mark, io.fresh, ws.q0, ws.q1, ws.prefix, ws.tile_start, ws.blocks, rs };
      if (bw) {
        k_r_seed<true><<<1, 1, 0, ctx->stream>>>(io.avail, io.mark, ws.q0, rs);
        launch_search<true>(ctx, a);
      } else {
        k_r_seed<false><<<1, 1, 0, ctx->stream>>>(io.avail, io.mark, ws.q0, rs);
        launch_search<false>(ctx, a);
      }
      ctx->launches += 1;
    }
    k_r_setid<<<1, 1, 0, ctx->stream>>>(rs);
    k_bitmap_min<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(g.n, ws.vis_b, rs);
    k_fwbw_finalize<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(g.n, ws.vis_b, und, scc_id, rs);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 3;
  } else {
    // host-driven loop over the same kernels, expansion kernels bracketed
    // by CUDA events (kspn_options.profile)
    bool const trace_done = st && st->levels_fw != 0; // trace the first FW-BW only
    k_r_init<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(words, g.m, und, ws.mark, ws.vis_a, ws.vis_b, rs);
    ctx->launches += 1;
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
        if (bw) level_body<true>(ctx, g, io, rs);
        else level_body<false>(ctx, g, io, rs);
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
  if (hs->bar_err) throw error{ KSPN_ERR_TIMEOUT, "reachability: grid barrier wait limit reached" };
  if (opt.trace && st && st->search_marks == 0 && hs->marks) {
    uint32_t const k = std::min<uint32_t>(hs->marks, MARKS);
    KSPN_CUDA(cudaMemcpyAsync(st->search_phase, static_cast<char*>(ws.rstate) + 2048, 4 * k, cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaMemcpyAsync(st->search_ns, static_cast<char*>(ws.rstate) + 2048 + 4 * MARKS, 8 * k, cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    st->search_marks = k;
  }
  ctx->td_edges += hs->edges_td + hs->edges_bu;
  if (st && st->levels_fw == 0 && st->levels_bw == 0) {
    st->levels_fw        = hs->levels_fw;
    st->levels_bw        = hs->levels_bw;
    st->levels_bottom_up = hs->bu_fw + hs->bu_bw;
  }
  return hs->decided;
}

} // namespace kspn
