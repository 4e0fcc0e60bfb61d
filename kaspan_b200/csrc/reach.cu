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
// Production runs the whole FW-BW as ONE persistent cooperative launch
// (k_fwbw, below) with one grid barrier per level.  With profiling on (or a
// graph too large for the packed level counters) the same phase bodies run
// as separate launches from a host loop (decide / expand / bottom-up /
// advance kernels, control in reach_state) with CUDA events around the
// expansion kernels.
#include "expand.cuh"
#include "mlp.cuh"

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
  uint32_t           bar_err; // 1: the persistent launch's grid barrier gave up
  uint32_t           marks;   // phase stamps taken (kspn_options.trace)
  unsigned long long lq[3];   // persistent launch: packed level counters (edges << qbits | vertices), FW search
  unsigned long long mat_q;   // persistent launch: counter of a frontier built from `fresh`, FW search
  unsigned long long lq_bw[3]; // the same for the BW search (FW and BW run side by side)
  unsigned long long mat_q_bw;
  // resident pipeline (FW-BW launch with the trim fixpoint as its tail)
  uint32_t           pivot_used;   // pivot the launch searched from (n: none)
  uint32_t           trim_decided; // vertices the trim tail decided
  uint32_t           trim_levels;  // its push levels
  uint32_t           und_left;     // undecided vertices when the launch ended
  unsigned long long trim_edges;   // adjacency entries the trim tail read
  unsigned long long list_n;       // undecided vertices listed for the trim tail
  uint32_t           bu_bitmap;    // bottom-up levels that swept the bitmap
  uint32_t           async_phases; // searches finished on the worklist
  unsigned long long rows_td;      // rows the top-down levels expanded
  unsigned long long pushed_td;    // vertices they queued (offsets read once more)
  uint32_t           mats;         // frontiers built from `fresh`
  unsigned long long t_ns[3];      // %globaltimer: launch start, FW-BW end, trim end
  uint32_t           cut_n[2];     // bottom-up rows cut short (FW, BW search; host-driven levels use [0])
  uint32_t           fixups;       // fix-up steps run (both searches)
  uint32_t           hseed_n;      // trim tail: listed vertices with a heavy row
  uint32_t           joint;        // the BW search ran inside the FW search's worklist phase
  uint32_t           hq_n[6];      // trim tail: heavy out-/in-rows listed per push level (pairs rotating like lq)
  uint32_t           heavy_err;    // a heavy or cut list would have overflowed
  uint32_t           trim_async;   // the trim tail finished on the worklist
  uint32_t           restricts;    // passes that cut one search's candidates down to the other's set
  uint32_t           pivot_rejected; // the pivot model rejected the launch's pivot: the launch ended after its first level
  uint32_t           handoff;        // the launch ended where its worklist phase starts; a resume launch continues
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
    st->bar_err                               = 0;
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
  st->cut_n[0]                  = 0; // (host-driven levels: the level's cut rows were walked)
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
// (`word` = avail's word of v, probed ahead through L2)
struct take_op
{
  uint32_t* avail; // FW: cand; BW: vis_a
  uint32_t* mark;  // FW: vis_a; BW: vis_b
  __device__ __forceinline__ uint32_t probe(uint32_t v) const { return __ldcg(avail + (v >> 5)); }
  __device__ __forceinline__ bool     operator()(uint32_t, uint32_t v, bool valid, uint32_t word) const
  {
    if (!valid || !((word >> (v & 31)) & 1u) || !bit_take(avail, v)) return false;
    bit_claim(mark, v);
    return true;
  }
};

// Bottom-up levels: a candidate (a set bit of avail) joins -- taken from
// avail, set in mark -- when a neighbour in its opposite-direction row is
// already in mark.
constexpr int BU_WARPS = R_THREADS / 32;

// Sparse sweeps hand a warp up to BU_GROUP consecutive chunks at once, so
// that their few candidates share the dependent head -> neighbour -> probe
// chains instead of paying one chain per chunk; a group is sized for about
// BU_GROUP_CANDS candidates.
constexpr int      BU_GROUP       = 8;
constexpr uint32_t BU_GROUP_CANDS = 256;

// Per-warp shared memory of the sweep.
struct bu_warp_smem
{
  uint16_t cand[32 * 32];       // the warp's chunk (32 words = 1024 vertices) or group packed, as offsets from its first vertex
  uint32_t found[32 * BU_GROUP]; // found bits per word of the chunk or group
};

// Rows cut short in bottom-up sweeps: a row the warp has walked HEAVY_ROW
// entries of without a hit is left open (the vertex stays a candidate) and
// its vertex listed once (map) for a fix-up step that walks the listed
// rows in slices over the whole grid.
struct bu_cut
{
  uint32_t* map;  // bitmap of listed vertices
  uint32_t* list; // listed vertices
  uint32_t* n;    // list length
  uint32_t  cap;  // list capacity (never reached: a listed row has HEAVY_ROW+ entries)
  uint32_t* err;  // set if it were
};

// The sweeps' cut descriptors (FW search, BW search): block-shared, set by
// thread 0 before the first sweep (a barrier between) and read only on the
// rare path, so the sweep's hot loop holds no register for them.
__shared__ bu_cut s_bu_cut[2];

// Row walks of up to BU_ILP candidates per lane (v[k], live[k]): all
// neighbour loads of a step, then all probes of `mark`; rows still open
// after BU_STEPS neighbours are finished by the whole warp with early exit,
// a row longer than HEAVY_ROW cut short and listed (bu_cut).  found[k]: a
// neighbour of v[k] is in mark.  All lanes call it.
constexpr int BU_STEPS = 32; // neighbours a candidate checks itself before its warp helps

__device__ __forceinline__ void
bu_rows(uint32_t const (&v)[BU_ILP], bool (&live)[BU_ILP], bool (&found)[BU_ILP], uint64_t const* __restrict__ head, uint32_t const* __restrict__ adj, uint32_t const* mark,
        bu_cut const& cut, uint64_t& nedge)
{
  unsigned const lane = threadIdx.x & 31u;
  uint64_t       b[BU_ILP], e[BU_ILP];
#pragma unroll
  for (int k = 0; k < BU_ILP; ++k) {
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
      uint64_t const e1 = e0 - b0 > HEAVY_ROW ? b0 + HEAVY_ROW : e0;
      bool           hit = false;
      for (uint64_t x = b0; x < e1; x += 32) {
        bool const     in = x + lane < e1;
        uint32_t const y  = in ? adj[x + lane] : 0u;
        bool const     h  = in && ((__ldcg(mark + (y >> 5)) >> (y & 31)) & 1u);
        nedge += in;
        if (__any_sync(0xFFFFFFFFu, h)) {
          hit = true;
          break;
        }
      }
      if (lane == l) {
        found[k] = hit;
        if (!hit && e1 < e0 && bit_claim(cut.map, v[k])) {
          uint32_t const i = atomicAdd(cut.n, 1u);
          if (i < cut.cap) cut.list[i] = v[k];
          else atomicExch(cut.err, 1u);
        }
      }
    }
  }
}

// Bottom-up sweep of chunk c (bitmap words [32c, 32c + 32)) by one warp.
// Candidates are the set bits of `avail`; one joins when a neighbour in its
// head/adj row is in `mark`.  Warps work independently (no block barrier):
// the warp packs its chunk's candidates (popcount scan over its 32 words)
// as 16-bit offsets in shared memory, each lane walks BU_ILP candidates'
// rows interleaved (bu_rows).  Lane i then owns word i of the chunk: it
// clears the found bits from avail, sets them in mark and writes the word
// of `fresh` (the sweep's discoveries).  No queue is written; the discovery
// count goes to nfound.  `avail` and `mark` are read through L2 (other
// blocks of a persistent launch change them).
__device__ __forceinline__ void
bu_sweep_chunk(uint32_t c,
               uint32_t n,
               uint64_t const* __restrict__ head,
               uint32_t const* __restrict__ adj,
               uint32_t* avail,
               uint32_t* mark,
               uint32_t* fresh,
               bu_cut const& cut,
               bu_warp_smem& sm,
               uint32_t& nfound,
               uint64_t& nedge,
               uint64_t& ncand)
{
  unsigned const lane  = threadIdx.x & 31u;
  uint32_t const words = (n + 31) / 32;
  uint32_t const w     = c * 32 + lane;
  uint32_t       word  = w < words ? __ldcg(avail + w) : 0u;
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
    sm.cand[pos++] = static_cast<uint16_t>(lane * 32 + bb);
  }
  sm.found[lane] = 0;
  __syncwarp();
  ncand += lane == 0 ? total : 0;
  for (uint32_t r = 0; r < total; r += 32 * BU_ILP) {
    uint32_t v[BU_ILP];
    bool     live[BU_ILP], found[BU_ILP];
#pragma unroll
    for (int k = 0; k < BU_ILP; ++k) {
      uint32_t const i = r + k * 32 + lane;
      live[k]          = i < total;
      v[k]             = live[k] ? c * 1024 + sm.cand[i] : 0u;
    }
    bu_rows(v, live, found, head, adj, mark, cut, nedge);
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

// Bottom-up sweep of the cnt <= BU_GROUP consecutive chunks [c0, c0 + cnt)
// by one warp (cnt = 1 on dense levels): lane i loads word i of every chunk
// (independent loads); the chunks are then taken in segments of at most
// 32 x 32 candidates (the pack buffer), each packed once and walked in
// batches of 32 x BU_ILP as bu_rows does, after which lane i writes back
// word i of each chunk of the segment.  On a sparse level one segment holds
// the whole group, so its few candidates share one dependent head ->
// neighbour -> probe chain instead of one chain per chunk.
__device__ __forceinline__ void
bu_sweep_group(uint32_t c0,
               uint32_t cnt,
               uint32_t n,
               uint64_t const* __restrict__ head,
               uint32_t const* __restrict__ adj,
               uint32_t* avail,
               uint32_t* mark,
               uint32_t* fresh,
               bu_cut const& cut,
               bu_warp_smem& sm,
               uint32_t& nfound,
               uint64_t& nedge,
               uint64_t& ncand)
{
  unsigned const lane  = threadIdx.x & 31u;
  uint32_t const words = (n + 31) / 32;
  // the chunks' words wait in the lane's own slots of `found` until their
  // segment is packed (no register array across the scans)
#pragma unroll
  for (int g = 0; g < BU_GROUP; ++g) {
    uint32_t const w = (c0 + g) * 32 + lane;
    uint32_t       x = static_cast<uint32_t>(g) < cnt && w < words ? __ldcg(avail + w) : 0u;
    if (w == words - 1 && (n & 31)) x &= (1u << (n & 31)) - 1u;
    sm.found[g * 32 + lane] = x;
  }
  for (uint32_t s0 = 0; s0 < cnt;) {
    // the segment [s0, s1): whole chunks while the pack buffer holds them
    // (warp-uniform; a chunk alone always fits)
    uint32_t s1 = s0, total = 0;
    while (s1 < cnt) {
      uint32_t const t = __reduce_add_sync(0xFFFFFFFFu, static_cast<uint32_t>(__popc(sm.found[s1 * 32 + lane])));
      if (s1 > s0 && total + t > 32 * 32) break;
      total += t;
      ++s1;
    }
    uint32_t cl = 0;
    for (uint32_t g = s0; g < s1; ++g) cl += __popc(sm.found[g * 32 + lane]);
    uint32_t pos = cl;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, pos, d);
      if (lane >= static_cast<unsigned>(d)) pos += y;
    }
    pos -= cl;
    for (uint32_t g = s0; g < s1; ++g) {
      uint32_t word = sm.found[g * 32 + lane];
      while (word) {
        uint32_t const bb = __ffs(word) - 1;
        word &= word - 1;
        sm.cand[pos++] = static_cast<uint16_t>((g - s0) * 1024 + lane * 32 + bb);
      }
      sm.found[g * 32 + lane] = 0;
    }
    __syncwarp();
    ncand += lane == 0 ? total : 0;
    uint32_t const vbase = (c0 + s0) * 1024;
    for (uint32_t r = 0; r < total; r += 32 * BU_ILP) {
      uint32_t v[BU_ILP];
      bool     live[BU_ILP], found[BU_ILP];
#pragma unroll
      for (int k = 0; k < BU_ILP; ++k) {
        uint32_t const i = r + k * 32 + lane;
        live[k]          = i < total;
        v[k]             = live[k] ? vbase + sm.cand[i] : 0u;
      }
      bu_rows(v, live, found, head, adj, mark, cut, nedge);
#pragma unroll
      for (int k = 0; k < BU_ILP; ++k)
        if (found[k]) atomicOr(&sm.found[(v[k] >> 5) - c0 * 32], 1u << (v[k] & 31));
    }
    __syncwarp();
    for (uint32_t g = s0; g < s1; ++g) {
      uint32_t const w   = (c0 + g) * 32 + lane;
      uint32_t const fnd = sm.found[g * 32 + lane];
      if (w < words) {
        if (fnd) {
          atomicAnd(avail + w, ~fnd);
          atomicOr(mark + w, fnd);
        }
        fresh[w] = fnd;
      }
      nfound += __popc(fnd);
    }
    __syncwarp();
    s0 = s1;
  }
}

// Chunks per sweep group for a bottom-up level over `cand` candidates of n
// vertices (1: dense, chunk by chunk): the largest power of two up to
// BU_GROUP whose expected candidates stay within BU_GROUP_CANDS.
__device__ __forceinline__ uint32_t
bu_group_size(uint64_t cand, uint32_t n)
{
  uint64_t const per_chunk = n ? cand * 1024 / n : 0;
  uint32_t       g         = 1;
  while (g < BU_GROUP && per_chunk * 2 * g <= BU_GROUP_CANDS) g *= 2;
  return g;
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
            reach_state* st,
            bu_cut cut)
{
  if (g.closed()) return;
  __shared__ bu_warp_smem sm[BU_WARPS];
  if (threadIdx.x == 0) s_bu_cut[0] = cut;
  __syncthreads();
  uint32_t       nfound = 0;
  uint64_t       nedge = 0, ncand = 0;
  unsigned const wid    = threadIdx.x >> 5;
  uint32_t const chunks = ((n + 31) / 32 + 31) / 32;
  for (uint32_t c = blockIdx.x * BU_WARPS + wid; c < chunks; c += gridDim.x * BU_WARPS)
    bu_sweep_chunk(c, n, head, adj, avail, mark, fresh, s_bu_cut[0], sm[wid], nfound, nedge, ncand);
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

// The rows k_bottom_up cut short, walked to the end in slices over the
// grid: a listed candidate with a neighbour in mark joins (avail, mark and
// fresh updated, counted into the level's output count).
__global__ void __launch_bounds__(R_THREADS)
k_bu_cut_rows(uint64_t const* __restrict__ head, uint32_t const* __restrict__ adj, uint32_t* avail, uint32_t* mark, uint32_t* fresh, fio f, gate g, bu_cut cut)
{
  if (g.closed()) return;
  unsigned const lane   = threadIdx.x & 31u;
  uint32_t const nc     = *cut.n < cut.cap ? *cut.n : cut.cap;
  uint32_t       nfound = 0;
  heavy_slices(cut.list, nc, head, [&](uint32_t, uint32_t v, uint64_t b, uint64_t e) {
    if (!((__shfl_sync(0xFFFFFFFFu, __ldcg(avail + (v >> 5)), 0) >> (v & 31)) & 1u)) return;
    bool hit = false;
    for (uint64_t x = b; x < e; x += 32) {
      bool const     in = x + lane < e;
      uint32_t const y  = in ? adj[x + lane] : 0u;
      if (__any_sync(0xFFFFFFFFu, in && ((__ldcg(mark + (y >> 5)) >> (y & 31)) & 1u))) {
        hit = true;
        break;
      }
    }
    if (hit && lane == 0 && bit_take(avail, v)) {
      atomicOr(mark + (v >> 5), 1u << (v & 31));
      atomicOr(fresh + (v >> 5), 1u << (v & 31));
      ++nfound;
    }
  });
  if (nfound) atomicAdd(f.out_n(), nfound);
}

// Clears the listed rows' cutmap bits (the count is reset by k_r_advance).
__global__ void __launch_bounds__(R_THREADS)
k_bu_cut_clear(gate g, bu_cut cut)
{
  if (g.closed()) return;
  uint32_t const nc = *cut.n < cut.cap ? *cut.n : cut.cap;
  for (uint32_t i = blockIdx.x * R_THREADS + threadIdx.x; i < nc; i += gridDim.x * R_THREADS) {
    uint32_t const v = cut.list[i];
    atomicAnd(cut.map + (v >> 5), ~(1u << (v & 31)));
  }
}

// ---------------------------------------------------------------- persistent FW-BW
// The whole FW-BW -- both searches, the SCC's id and its write-back -- is
// ONE cooperative launch whose blocks stay resident and meet at a grid
// barrier once per level:
//   init      cand = und minus the pivot, vis_a = vis_b = {pivot}, |und| per
//             block; the pivot alone is the first level's frontier.
//   FW, BW    a top-down level writes the next level's frontier already
//             scanned: each block flush reserves its queue slots AND its
//             range of the frontier's edge prefix with ONE 64-bit atomic on
//             a packed (edges << qbits | vertices) counter, then writes the
//             queue entries, their prefix and the tile starts.  Right after
//             the barrier every block knows the next frontier's size and
//             edge count and can expand it (or choose bottom-up) at once.
//             A bottom-up level only counts its discoveries (the `fresh`
//             bitmap holds them); a level that returns to top-down first
//             builds its frontier from that bitmap the same way (one extra
//             barrier).
//   finalize  smallest member (one barrier, min-id mode), then und and the
//             ids are written a bitmap word at a time.
// Every block derives the level's control (direction, tile count, edge
// budget) from the same counter values read after the barrier, so nothing
// is broadcast.  Level counters rotate over three slots: level L reads slot
// L%3, adds to (L+1)%3 and clears (L+2)%3, which no block touches again
// until after the next barrier.
constexpr unsigned GRID_SYNC_SPINS = 1u << 22; // default wait limit (kspn_options.wait_limit = 0)

// Grid barrier with a monotonically growing counter: every block adds 1
// with a release reduction (no return value, so arrivals never wait on one
// another) and waits, with acquire loads, until the counter reaches
// epoch * blocks.  The counter is never reset inside a launch; `epoch`
// carries the count to the next launch of the same grid.  The host clears
// the whole struct when a wait gave up.
struct grid_barrier
{
  unsigned long long root;
  unsigned long long pad0[15];
  unsigned long long epoch; // barriers completed by every block
  uint32_t           err;   // 1: a wait reached the wait limit
  uint32_t           pad1[29];
};
static_assert(sizeof(grid_barrier) <= 4096, "grid barrier must fit its workspace slot");

__device__ __forceinline__ unsigned long long
ld_acquire64(unsigned long long const* p)
{
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Barrier count of the running launch at its start (thread 0 of each block
// sets it before the block's first barrier).
__shared__ unsigned long long s_epoch0;

// All threads of every block call it.  False when a wait gave up (then every
// block returns false here or at its next barrier, and the launch ends).
// `limit` bounds the polls; with drop != 0 the grid's last block leaves the
// drop-th barrier of the launch without arriving (the test hook of
// kspn_options.drop_barrier), so the others' waits run out.
__device__ __forceinline__ bool
grid_sync(grid_barrier* b, unsigned long long& epoch, unsigned limit, unsigned drop)
{
  __shared__ uint32_t s_ok;
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    if (drop && blockIdx.x == gridDim.x - 1 && epoch - s_epoch0 == drop) ok = 0;
    else {
      asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(&b->root), "l"(1ull) : "memory");
      unsigned long long const target = epoch * gridDim.x;
      for (unsigned spins = 0; ld_acquire64(&b->root) < target; ++spins) {
        if (spins > limit || ((spins & 63u) == 63u && ld_acquire(&b->err))) {
          atomicExch(&b->err, 1u);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// A scanned frontier: queue, exclusive prefix of the queued vertices'
// degrees, and per tile of EX_TILE edges the queue index holding its first
// edge.
struct frontier_buf
{
  uint32_t* q;
  uint64_t* prefix;
  uint32_t* tile_start;
};

struct fwbw_args
{
  uint32_t           n;
  uint32_t           pivot;
  uint64_t           m;
  uint32_t           cap; // level cap per search
  uint32_t           min_ids;
  uint32_t           qbits; // vertex bits of the packed level counters
  uint32_t           trace;
  unsigned long long alpha, beta;
  uint64_t const*    fh;
  uint32_t const*    fc;
  uint64_t const*    bh;
  uint32_t const*    bc;
  uint32_t*          und;
  uint32_t*          scc_id;
  uint32_t*          cand;
  uint32_t*          vis_a;
  uint32_t*          vis_b;
  uint32_t*          fresh;
  uint32_t*          fresh_bw; // the BW search's sweep discoveries
  uint32_t*          cand_bw;  // BW candidates (und minus the pivot, then what BW has not reached)
  frontier_buf       fb[2];
  frontier_buf       fb_bw[2]; // the BW search's frontier pair
  frontier_buf       seed;    // q[0] = pivot, prefix[0] = 0, tile starts all 0
  uint64_t*          partial; // one per block
  // resident pipeline: pivot == PIVOT_FROM_DEVICE takes trim_1_first's
  // (pv_prod, pv_id); trim != 0 runs the trim-1 fixpoint after the FW-BW
  uint64_t const*    pv_prod;
  uint32_t const*    pv_id;
  uint32_t           trim;
  uint32_t           ids_at_end; // resident launch: write every vertex's id at the end
  unsigned long long* aw;        // asynchronous tail: worklist (aw_cap tagged entries, 0 when unused)
  uint64_t           aw_cap;
  unsigned long long* aq;        // its counters: head at [0], tail at [16], done at [32] (own lines)
  uint32_t*          indeg;
  uint32_t*          outdeg;
  // heavy rows: four lists of heavy_cap entries -- [0] trim seed (and the
  // BW search's cut rows), [1] [2] trim push levels by parity, [3] the FW
  // search's cut rows -- and the bitmap of cut rows (zero between searches)
  uint32_t*          heavy;
  uint32_t           heavy_cap;
  uint32_t*          cutmap;    // FW search's cut rows; the BW search's follow at cutmap + cut_words
  uint32_t           cut_words;
  grid_barrier*      bar;
  reach_state*       st;
  uint32_t*          stamp_phase;
  uint64_t*          stamp_ns;
  uint32_t           wait_limit;   // polls before a wait gives up
  uint32_t           drop_barrier; // test hook: the last block leaves this barrier of the launch (0 = off)
  uint64_t           aw_exact;     // worklist items after which warps take their finds exactly
  float const*       model;        // pivot MLP parameters: the launch scores its pivot first (null: no check)
  void*              jsave;        // the level loop's saved control (handoff, resume)
  uint32_t           resume;       // 1: continue a launch that handed off, at its worklist phase
};

__device__ __forceinline__ bool
gsync(fwbw_args const& a, unsigned long long& epoch)
{
  return grid_sync(a.bar, epoch, a.wait_limit, a.drop_barrier);
}

// Block-shared scratch of the persistent kernel.
struct fwbw_smem
{
  // bottom-up and trim per-warp buffers; during a top-down level the same
  // bytes hold the tile's row map (tile_rows) and the block queue (buf)
  bu_warp_smem warp[BU_WARPS];
  uint32_t              tile_i[2];
  uint32_t              buf_n;
  uint32_t              cnt;
  unsigned long long    old;
  unsigned long long    edges_bu, cands_bu; // bottom-up statistics of the launch
  __device__ __forceinline__ uint32_t* tile_rows() { return reinterpret_cast<uint32_t*>(warp); }
  __device__ __forceinline__ uint32_t* buf() { return reinterpret_cast<uint32_t*>(warp) + EX_TILE; }
};
static_assert(sizeof(bu_warp_smem) * BU_WARPS >= (EX_TILE + BU_BUF + 512 * 3) * sizeof(uint32_t), "tile rows and block queue must fit the warp buffers");
static_assert(BU_BUF == EX_TILE && BU_BUF % R_THREADS == 0, "flush: whole runs per thread");

__device__ __forceinline__ uint64_t
globaltimer()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// block 0, thread 0: record that `phase` ended now
__device__ __forceinline__ void
stamp(fwbw_args const& a, uint32_t phase)
{
  if (!a.trace || blockIdx.x != 0 || threadIdx.x != 0) return;
  uint32_t const i = a.st->marks;
  if (i < MARKS) {
    a.stamp_phase[i] = phase;
    a.stamp_ns[i]    = globaltimer();
    a.st->marks      = i + 1;
  }
}

// Tiles whose first edge lies in [p, p + d) start at queue index i; tiles
// past the graph's m edges are never written (tile_start holds
// m / EX_TILE + 4 entries).
__device__ __forceinline__ void
put_tile_starts(uint32_t* tile_start, uint64_t p, uint64_t d, uint32_t i, uint64_t m)
{
  if (!d) return;
  uint64_t const end = p + d < m ? p + d : m;
  for (uint64_t t = (p + EX_TILE - 1) / EX_TILE; t * EX_TILE < end; ++t) tile_start[t] = i;
}

// Appends the block queue (sm.buf()[0, sm.buf_n)) to a scanned frontier.
// Thread t owns entries [8t, 8t + 8); one block scan of the degree sums
// and one packed atomic give every entry its queue slot and edge prefix.
// Degrees are read twice (the second time from cache) rather than held in
// registers.  All threads call it; leaves sm.buf_n == 0.
__device__ __forceinline__ void
flush_scanned(fwbw_smem& sm, frontier_buf const& out, unsigned long long* ctr, uint32_t qbits, uint64_t const* __restrict__ head, uint32_t qcap, uint64_t ecap)
{
  constexpr int K = BU_BUF / R_THREADS;
  __syncthreads();
  uint32_t const cnt = sm.buf_n;
  if (cnt) {
    uint32_t const i0  = threadIdx.x * K;
    uint32_t const k1  = cnt > i0 ? (cnt - i0 < K ? cnt - i0 : K) : 0u; // entries of this thread
    uint64_t       sum = 0;
#pragma unroll
    for (int k = 0; k < K; ++k)
      if (k < k1) {
        uint32_t const v = sm.buf()[i0 + k];
        sum += head[v + 1] - head[v];
      }
    uint64_t       tot;
    uint64_t const off = block_exclusive_scan<uint64_t, R_THREADS>(sum, &tot);
    if (threadIdx.x == 0) sm.old = atomicAdd(ctr, (static_cast<unsigned long long>(tot) << qbits) | cnt);
    __syncthreads();
    unsigned long long const old = sm.old;
    uint64_t const           pos0 = (old & ((1ull << qbits) - 1)) + i0;
    uint32_t                 pos  = static_cast<uint32_t>(pos0);
    uint64_t                 p    = (old >> qbits) + off;
    for (uint32_t k = 0; k < k1 && pos0 + k < qcap && p < ecap; ++k, ++pos) {
      uint32_t const v = sm.buf()[i0 + k];
      uint64_t const d = head[v + 1] - head[v];
      out.q[pos]       = v;
      out.prefix[pos]  = p;
      put_tile_starts(out.tile_start, p, d, pos, ecap);
      p += d;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) sm.buf_n = 0;
  __syncthreads();
}

// Frontier from the `fresh` bitmap (a search returning to top-down after
// bottom-up sweeps), scanned like flush_scanned: a thread owns MAT_WORDS
// consecutive words, a block pass packs (edges << 16 | vertices) per
// thread (at most 256 * 32 * MAT_WORDS < 2^16 vertices a pass).
constexpr int MAT_WORDS = 4;

__device__ __forceinline__ void
materialize_scanned(uint32_t n, uint32_t const* fresh, frontier_buf const& out, unsigned long long* ctr, uint32_t qbits, uint64_t const* __restrict__ head, uint64_t ecap, fwbw_smem& sm)
{
  uint32_t const words = (n + 31) / 32;
  uint64_t const qcap  = n; // queue slots
  for (uint32_t wbase = blockIdx.x * R_THREADS * MAT_WORDS; wbase < words; wbase += gridDim.x * R_THREADS * MAT_WORDS) {
    uint32_t const w0 = wbase + threadIdx.x * MAT_WORDS;
    uint32_t       word[MAT_WORDS];
    uint32_t       c   = 0;
    uint64_t       deg = 0;
#pragma unroll
    for (int k = 0; k < MAT_WORDS; ++k) {
      word[k] = w0 + k < words ? __ldcg(fresh + w0 + k) : 0u;
      c += __popc(word[k]);
    }
#pragma unroll
    for (int k = 0; k < MAT_WORDS; ++k)
      for (uint32_t x = word[k]; x; x &= x - 1) {
        uint32_t const v = (w0 + k) * 32 + __ffs(x) - 1;
        deg += head[v + 1] - head[v];
      }
    uint64_t       tot;
    uint64_t const off = block_exclusive_scan<uint64_t, R_THREADS>((deg << 16) | c, &tot);
    if (tot == 0) continue; // block-uniform
    if (threadIdx.x == 0) sm.old = atomicAdd(ctr, ((tot >> 16) << qbits) | (tot & 0xFFFFu));
    __syncthreads();
    unsigned long long const old = sm.old;
    uint64_t                 pos = (old & ((1ull << qbits) - 1)) + (off & 0xFFFFu);
    uint64_t                 p   = (old >> qbits) + (off >> 16);
#pragma unroll
    for (int k = 0; k < MAT_WORDS; ++k)
      for (uint32_t x = word[k]; x && pos < qcap && p < ecap; x &= x - 1) {
        uint32_t const v = (w0 + k) * 32 + __ffs(x) - 1;
        uint64_t const d = head[v + 1] - head[v];
        out.q[pos]       = v;
        out.prefix[pos]  = p;
        put_tile_starts(out.tile_start, p, d, static_cast<uint32_t>(pos), ecap);
        p += d;
        ++pos;
      }
    __syncthreads(); // sm.old
  }
}

// Warp-aggregated append to a queue whose length is a 64-bit counter: all
// lanes of the warp call it (warp_push64) or only the active ones
// (warp_push_active64).  Slots at or past `cap` are not written.
__device__ __forceinline__ void
warp_push64(bool pred, uint32_t v, uint32_t* q, unsigned long long* count, uint64_t cap)
{
  unsigned const ballot = __ballot_sync(0xFFFFFFFFu, pred);
  if (!ballot) return;
  unsigned const     lane = threadIdx.x & 31u, leader = __ffs(ballot) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, static_cast<unsigned long long>(__popc(ballot)));
  base                = __shfl_sync(0xFFFFFFFFu, base, leader);
  uint64_t const slot = base + __popc(ballot & ((1u << lane) - 1u));
  if (pred && slot < cap) q[slot] = v;
}
__device__ __forceinline__ void
warp_push_active64(uint32_t v, uint32_t* q, unsigned long long* count, uint64_t cap)
{
  unsigned const     mask = __activemask();
  unsigned const     lane = threadIdx.x & 31u, leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(count, static_cast<unsigned long long>(__popc(mask)));
  base                = __shfl_sync(mask, base, leader);
  uint64_t const slot = base + __popc(mask & ((1u << lane) - 1u));
  if (slot < cap) q[slot] = v;
}

// Outcome of a search phase: done, level cap reached, or the grid barrier
// (or a worklist wait) gave up.
enum : int
{
  SEARCH_DONE     = 0,
  SEARCH_CAPPED   = 1,
  SEARCH_FAILED   = 2,
  SEARCH_REJECTED = 3, // the pivot model rejected the pivot: the launch ended after its first level
  SEARCH_HANDOFF  = 4  // the launch ended where the worklist phase starts; a resume launch runs it
};

// ---------------------------------------------------------------- asynchronous tail
// A search whose frontier stays small level after level (a high-diameter
// graph, e.g. RGG) pays a grid barrier and a chain of dependent loads per
// level for little work.  The reached SET does not depend on level order,
// so such a search finishes on a global worklist instead: entries are
// (AW_TAG | vertex), written once per slot; a warp claims 32 slots at a
// time, waits for each to be written, expands the vertex (take from avail,
// set in mark, as a top-down level) and appends its finds; a warp adds its
// finished items to the processed count when it next runs out of ready
// slots.  The phase ends when the processed count equals the appended count
// (nothing in flight can append any more); the used slots are then cleared to 0, so the worklist
// is all zeros outside a phase.  Every wait is bounded.
constexpr uint32_t           ASYNC_AFTER    = 16;        // top-down levels before a search may switch
constexpr uint32_t           ASYNC_FRONTIER = 1u << 16;  // largest frontier that switches
constexpr unsigned long long AW_TAG         = 1ull << 32; // marks a written slot
constexpr int                AW_BATCH       = 8;         // neighbours a lane loads at once
constexpr int                AW_WARPS       = 8;         // warps per block that take worklist items (the others wait at the phase's end)

// Finds a warp keeps on its own stack (in its shared buffer) and expands in
// its next round instead of appending them: a hop then costs the chain of
// loads of one expansion, not a trip through the worklist to whichever warp
// claimed the slot.  Finds past AW_LOCAL_KEEP go to the worklist, where idle
// warps pick them up.  Stack entries are items (below) with slice 0.
constexpr uint32_t           AW_LOCAL_KEEP = 16;
constexpr unsigned long long AW_BW         = 1ull << 63; // item of the BW search of a joint phase
constexpr unsigned long long AW_TAKEN      = 1ull << 62; // the vertex was taken when it was pushed (else its consumer takes it)
static_assert(sizeof(bu_warp_smem) >= AW_LOCAL_KEEP * sizeof(unsigned long long), "local stack must fit the warp buffer");
static_assert(R_THREADS / 32 == 8 && AW_BATCH == 8, "AW_STALE counts 8 warps per block and 8 finds per lane per pass");

// One search's arrays in the worklist phase: rows to walk, the candidates a
// find is taken from, the set it joins.
struct aw_dir
{
  uint64_t const* head;
  uint32_t const* adj;
  uint32_t*       avail;
  uint32_t*       mark;
};

// Appends the finds of one pass: lane has c finds, at positions [q, q + c)
// of the warp's tot (exclusive scan); the first min(tot, room) go to the
// stack, the others to the worklist.  Warp-uniform; returns the stack's new
// size.
struct aw_sink
{
  unsigned long long* stk;
  unsigned long long* aw;
  unsigned long long* tail;
  uint64_t            cap;
  __device__ __forceinline__ uint32_t reserve(uint32_t ls_n, uint32_t tot, unsigned long long& gbase, uint32_t& nloc) const
  {
    uint32_t const room = ls_n < AW_LOCAL_KEEP ? AW_LOCAL_KEEP - ls_n : 0u;
    nloc                = tot < room ? tot : room;
    unsigned long long b = 0;
    if ((threadIdx.x & 31u) == 0 && tot > nloc) b = atomicAdd(tail, static_cast<unsigned long long>(tot - nloc));
    gbase = __shfl_sync(0xFFFFFFFFu, b, 0);
    return ls_n + nloc;
  }
  __device__ __forceinline__ void put(uint32_t ls_n, uint32_t nloc, unsigned long long gbase, uint32_t q, unsigned long long item) const
  {
    if (q < nloc) stk[ls_n + q] = item;
    else if (gbase + (q - nloc) < cap) __stcg(aw + gbase + (q - nloc), item);
  }
};

// Runs the rest of the search from frontier fq0[0, qn0) (direction d0).
// With d1 (a joint phase) the other search runs in the same phase from its
// frontier fq1[0, qn1): its items carry AW_BW.  All threads of every block
// call it.
// An item is AW_TAG | dir << 63 | slice << 33 | v: slice 0 of a row longer
// than HEAVY_ROW appends the row's other HEAVY_SLICE-entry slices as items
// of their own (so idle warps share the row) and walks the first; a vertex
// whose row is shorter is one item.  Each round a warp polls its claimed
// slots and fills its other lanes from its own stack; the done count only
// grows while the stack is empty, so done == appended still means that
// nothing is left anywhere.
__device__ __forceinline__ int
run_async(fwbw_args const& a, uint32_t const* fq0, uint32_t qn0, aw_dir const d0, uint32_t const* fq1, uint32_t qn1, aw_dir const* d1, unsigned long long& epoch,
          uint64_t& edges, fwbw_smem& sm)
{
  unsigned long long* const aw   = a.aw;
  unsigned long long* const head = a.aq;
  unsigned long long* const tail = a.aq + 16;
  unsigned long long* const done = a.aq + 32;
  uint64_t const            cap  = a.aw_cap;
  unsigned const            lane = threadIdx.x & 31u;
  unsigned const            lt   = (1u << lane) - 1u;
  bool const                joint = d1 != nullptr;
  aw_dir const              e1    = joint ? *d1 : d0;
  uint32_t const            qb    = joint ? qn1 : 0u;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; i < qn0 + qb; i += static_cast<uint64_t>(gridDim.x) * R_THREADS)
    __stcg(aw + i, i < qn0 ? AW_TAG | AW_TAKEN | __ldcg(fq0 + i) : AW_TAG | AW_TAKEN | AW_BW | __ldcg(fq1 + (i - qn0)));
  if (blockIdx.x == 0 && threadIdx.x == 0) *head = 0, *tail = qn0 + qb, *done = 0;
  if (!gsync(a, epoch)) return SEARCH_FAILED;
  aw_sink const sink{ reinterpret_cast<unsigned long long*>(&sm.warp[threadIdx.x >> 5]), aw, tail, cap };
  bool          failed      = false;
  uint32_t      unpublished = 0; // worklist items this warp finished, not yet added to done
  uint32_t      ls_n        = 0; // items on this warp's stack (warp-uniform)
  // A find whose probe shows it available is pushed without taking it:
  // its consumer takes it (the atomic issued beside the row-offset loads,
  // so the hop waits for one of them, not both) and drops the item if
  // another push of the same vertex won.  Duplicate items use worklist
  // slots, so once this warp's last reservation passed half of them it
  // takes its finds itself (exactly, AW_TAKEN); the worklist holds
  // 4n + 2 AW_STALE + 4m / HEAVY_SLICE items: half, the passes of every
  // warp around the switch, one winning item per vertex and direction, and
  // the slices (only a winner appends them).
  bool          exact       = false; // warp-uniform
  bool          batch       = false;
  bool          pending     = false;
  uint64_t      slot        = 0;
  unsigned      spins       = 0;
  for (bool alive = (threadIdx.x >> 5) < AW_WARPS; alive;) {
    if (!batch && ls_n == 0) {
      // only a warp without its own work claims slots: items appended to
      // the worklist then land with warps that are polling, not behind a
      // busy warp's round
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(head, 32ull);
      slot    = __shfl_sync(0xFFFFFFFFu, base, 0) + lane;
      pending = true;
      batch   = true;
    }
    bool               got  = false;
    unsigned long long item = 0;
    // an idle warp (spins > 0, stack empty) first looks at its lowest
    // pending slot only: slots are reserved in order and written right
    // after, so the others are rarely ready before it; thousands of idle
    // warps polling 32 slots each would crowd the busy ones out of L2
    bool look = pending && slot < cap;
    if (spins && ls_n == 0) {
      unsigned const pm    = __ballot_sync(0xFFFFFFFFu, look);
      bool           ready = false;
      if (pm && lane == static_cast<unsigned>(__ffs(pm) - 1)) ready = (ld_acquire64(aw + slot) & AW_TAG) != 0;
      if (!__any_sync(0xFFFFFFFFu, ready)) look = false;
    }
    if (look) {
      unsigned long long const e = ld_acquire64(aw + slot);
      if (e & AW_TAG) item = e, got = true, pending = false;
    }
    unsigned const gm = __ballot_sync(0xFFFFFFFFu, got); // worklist items this round
    if (ls_n) {
      // the lanes left free take the top of the stack
      unsigned const freem = ~gm;
      uint32_t const nfree = __popc(freem);
      uint32_t const k     = ls_n < nfree ? ls_n : nfree;
      uint32_t const r     = __popc(freem & lt);
      if (!got && r < k) item = sink.stk[ls_n - k + r], got = true;
      ls_n -= k;
      __syncwarp(); // the slots just read are reused by this round's finds
    }
    batch                = __any_sync(0xFFFFFFFFu, pending);
    unsigned const gmask = __ballot_sync(0xFFFFFFFFu, got);
    if (gmask) {
      uint32_t const           v   = static_cast<uint32_t>(item);
      uint32_t const           sl  = static_cast<uint32_t>(item >> 33) & 0x1FFFFFFFu;
      unsigned long long const dir = item & AW_BW;
      aw_dir const             d   = dir ? e1 : d0;
      uint64_t                 b = 0, e = 0;
      bool                     won = got;
      if (got) {
        // an untaken item: take it now (the atomic and the offset loads in
        // flight together); a lost take means a duplicate, which is dropped
        if (!(item & AW_TAKEN) && sl == 0) won = bit_take(d.avail, v);
        b = d.head[v], e = d.head[v + 1];
        if (!(item & AW_TAKEN) && sl == 0 && won) bit_set_async(d.mark, v);
        if (!won) e = b;
      }
      if (got && e - b > HEAVY_ROW) {
        if (sl == 0) {
          // the row's other slices become items (by the winner only)
          uint64_t const           ns = (e - b + HEAVY_SLICE - 1) / HEAVY_SLICE;
          unsigned long long const at = atomicAdd(tail, static_cast<unsigned long long>(ns - 1));
          for (uint64_t j = 1; j < ns; ++j)
            if (at + j - 1 < cap) __stcg(aw + at + j - 1, AW_TAG | AW_TAKEN | dir | (static_cast<unsigned long long>(j) << 33) | v);
        }
        b += static_cast<uint64_t>(sl) * HEAVY_SLICE;
        e = b + HEAVY_SLICE < e ? b + HEAVY_SLICE : e;
      }
      bool const big = got && e - b > 32;
      if (got) edges += e - b;
      // small rows, AW_BATCH neighbours per pass: all ids, then all probes,
      // then the takes; the warp's finds placed with at most one atomic per pass
      uint64_t x = got && !big ? b : e;
      while (__any_sync(0xFFFFFFFFu, x < e)) {
        unsigned long long const tk = exact ? AW_TAKEN : 0ull; // the pass's finds were taken here
        uint32_t w[AW_BATCH], found = 0;
#pragma unroll
        for (int k = 0; k < AW_BATCH; ++k) w[k] = x + k < e ? d.adj[x + k] : 0u;
        uint32_t wd[AW_BATCH];
#pragma unroll
        for (int k = 0; k < AW_BATCH; ++k) wd[k] = x + k < e ? __ldcg(d.avail + (w[k] >> 5)) : 0u;
#pragma unroll
        for (int k = 0; k < AW_BATCH; ++k)
          if (x + k < e && ((wd[k] >> (w[k] & 31)) & 1u)) {
            if (!exact) found |= 1u << k;
            else if (bit_take(d.avail, w[k])) bit_set_async(d.mark, w[k]), found |= 1u << k;
          }
        uint32_t const c = __popc(found);
        uint32_t       p = c;
#pragma unroll
        for (int dd = 1; dd < 32; dd <<= 1) {
          uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, p, dd);
          if (lane >= static_cast<unsigned>(dd)) p += y;
        }
        uint32_t const tot = __shfl_sync(0xFFFFFFFFu, p, 31);
        if (tot) {
          unsigned long long gbase;
          uint32_t           nloc;
          uint32_t const     next = sink.reserve(ls_n, tot, gbase, nloc);
          exact                   = exact || gbase > a.aw_exact;
          uint32_t           q    = p - c;
#pragma unroll
          for (int k = 0; k < AW_BATCH; ++k)
            if ((found >> k) & 1u) sink.put(ls_n, nloc, gbase, q++, AW_TAG | tk | dir | w[k]);
          ls_n = next;
        }
        x = x + AW_BATCH < e ? x + AW_BATCH : e;
      }
      for (unsigned todo = __ballot_sync(0xFFFFFFFFu, big); todo; todo &= todo - 1) {
        unsigned const           l   = __ffs(todo) - 1;
        uint64_t const           b0  = __shfl_sync(0xFFFFFFFFu, b, l), e0 = __shfl_sync(0xFFFFFFFFu, e, l);
        unsigned long long const dl  = __shfl_sync(0xFFFFFFFFu, dir, l);
        aw_dir const             dd_ = dl ? e1 : d0;
        for (uint64_t xb = b0; xb < e0; xb += 32) {
          uint64_t const x1 = xb + lane;
          uint32_t       w  = 0;
          bool           f  = false;
          if (x1 < e0) {
            w = dd_.adj[x1];
            f = ((__ldcg(dd_.avail + (w >> 5)) >> (w & 31)) & 1u) != 0;
            if (f && exact) {
              f = bit_take(dd_.avail, w);
              if (f) bit_set_async(dd_.mark, w);
            }
          }
          unsigned const fm = __ballot_sync(0xFFFFFFFFu, f);
          if (fm) {
            unsigned long long gbase;
            uint32_t           nloc;
            uint32_t const     next = sink.reserve(ls_n, __popc(fm), gbase, nloc);
            unsigned long long const tk = exact ? AW_TAKEN : 0ull; // before this chunk's switch
            exact                       = exact || gbase > a.aw_exact;
            if (f) sink.put(ls_n, nloc, gbase, __popc(fm & lt), AW_TAG | tk | dl | w);
            ls_n = next;
          }
        }
      }
      __syncwarp(); // this round's stack writes before the next round's reads
      // worklist items are counted as done when this warp next goes idle
      // (its stack empty, so their finds are expanded or appended)
      unpublished += __popc(gm);
      spins = 0;
    } else {
      // nothing arrived and the stack is empty: publish this warp's finished
      // items, then finished when every appended item is done
      if (unpublished) {
        __threadfence();
        if (lane == 0) atomicAdd(done, static_cast<unsigned long long>(unpublished));
        unpublished = 0;
      }
      uint32_t stop = 0;
      ++spins; // every lane: the count steers warp-wide choices above
      if (lane == 0) {
        unsigned long long const dn = ld_acquire64(done);
        unsigned long long const t  = ld_acquire64(tail);
        stop                        = dn == t ? 1u : 0u;
        if (!stop && (spins > a.wait_limit || ((spins & 63u) == 63u && ld_acquire(&a.bar->err)))) {
          atomicExch(&a.bar->err, 1u);
          stop = 2;
        }
      }
      stop = __shfl_sync(0xFFFFFFFFu, stop, 0);
      if (stop) {
        alive  = false;
        failed = stop == 2;
      } else __nanosleep(spins < 32 ? 64u : (spins < 256 ? 256u : 1024u)); // longer idle, longer sleep
    }
  }
  if (!gsync(a, epoch) || failed) return SEARCH_FAILED;
  // leave the worklist all zeros
  uint64_t t = __ldcg(tail);
  t          = t < cap ? t : cap;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; i < t; i += static_cast<uint64_t>(gridDim.x) * R_THREADS) __stcg(aw + i, 0ull);
  return SEARCH_DONE;
}

// ---------------------------------------------------------------- joint level loop
// The FW and BW searches from the pivot run side by side, one grid barrier
// per level for both: FW over out-edges (candidates cand, reached vis_a),
// BW over in-edges (candidates cand_bw, reached vis_b), each from the pivot
// over every undecided vertex, and the SCC is FW(p) & BW(p).  Each search
// keeps its own direction (top-down or bottom-up, Beamer's rule), frontier
// pair, level counters, sweep bitmap and cut list; a level runs both
// searches' steps over the whole grid (top-down tiles of both in one unit
// range, bottom-up chunks of both in one chunk range), so the latency-bound
// thin levels of the two searches overlap instead of adding up.  When one
// search ends, the other's candidates are cut down to the finished search's
// set (an SCC member reaches or is reached by the pivot inside the SCC, so
// nothing of the SCC is lost) -- after that it costs what the restricted
// search of the reference would.  When every running search is top-down
// and thin after ASYNC_AFTER levels, both finish on the worklist together.

// One search's arrays.
struct jdir
{
  uint64_t const*     td_head;
  uint32_t const*     td_adj;
  uint64_t const*     bu_head;
  uint32_t const*     bu_adj;
  uint32_t*           avail;
  uint32_t*           mark;
  uint32_t*           fresh;
  frontier_buf        fb0, fb1; // the pair, by level parity
  unsigned long long* lq;       // 3 rotating level counters
  unsigned long long* mat_q;
  uint32_t*           cut_list;
  uint32_t*           cut_n;
};

__device__ __forceinline__ jdir
joint_dir(fwbw_args const& a, int d)
{
  reach_state* const st = a.st;
  if (d == 0) return jdir{ a.fh, a.fc, a.bh, a.bc, a.cand, a.vis_a, a.fresh, a.fb[0], a.fb[1], st->lq, &st->mat_q, a.heavy + 3u * a.heavy_cap, &st->cut_n[0] };
  return jdir{ a.bh, a.bc, a.fh, a.fc, a.cand_bw, a.vis_b, a.fresh_bw, a.fb_bw[0], a.fb_bw[1], st->lq_bw, &st->mat_q_bw, a.heavy, &st->cut_n[1] };
}

__device__ __forceinline__ frontier_buf const&
jbuf(jdir const& D, uint32_t parity)
{
  return parity & 1u ? D.fb1 : D.fb0;
}

// Block-shared control of the loop: thread 0 of every block computes it from
// the same counters (so every block takes the same branches; nothing is
// broadcast), the other threads read it after a block barrier.
enum : uint32_t
{
  JK_NONE  = 0,
  JK_TD    = 1, // top-down expansion
  JK_BU    = 2, // bottom-up sweep
  JK_FIXUP = 3  // cut rows walked in slices
};
struct jctl
{
  unsigned long long c[2];        // the level's frontier: edges << qbits | vertices
  unsigned long long m_u[2];      // Beamer's unexplored-edge budget
  unsigned long long edges_td[2]; // top-down edges expanded
  unsigned long long seen[2];     // vertices this search has reached (the pivot included)
  uint32_t           grp[2];      // chunks per bottom-up sweep group this level
  uint32_t           lvl[2], bu[2], mode[2], mat[2], fixed[2], live[2], kind[2];
  uint32_t           restrict_to[2]; // 1: cut this search's candidates down to the other's set first
  uint32_t           capped, async, any_td, any_bu;
  uint32_t           cnt[2];
};
__shared__ jctl s_j;

// The level loop's control where a launch handed off its worklist phase
// (written by block 0, read by every block of the resume launch).
struct joint_save
{
  jctl               j;
  uint32_t           glvl, n_und;
  unsigned long long barriers; // grid barriers the handing-off launch completed (the drop_barrier test hook counts on)
};

template<int MINB>
__device__ __forceinline__ int
run_joint(fwbw_args const& a, fwbw_smem& sm, uint32_t pivot, uint32_t n_und, uint32_t& glvl, unsigned long long& epoch, bool resume)
{
  reach_state* const       st    = a.st;
  unsigned long long const qmask = (1ull << a.qbits) - 1;
  bool const               tally = blockIdx.x == 0 && threadIdx.x == 0; // keeps the byte-model counts in st
  unsigned const           lane  = threadIdx.x & 31u;
  unsigned const           wid   = threadIdx.x >> 5;
  uint32_t const           words = (a.n + 31) / 32;
  if (threadIdx.x == 0) {
    s_bu_cut[0] = bu_cut{ a.cutmap, a.heavy + 3u * a.heavy_cap, &st->cut_n[0], a.heavy_cap, &st->heavy_err };
    s_bu_cut[1] = bu_cut{ a.cutmap + a.cut_words, a.heavy, &st->cut_n[1], a.heavy_cap, &st->heavy_err };
    if (resume) s_j = static_cast<joint_save const*>(a.jsave)->j;
    for (int d = 0; d < 2 && !resume; ++d) {
      uint64_t const* h = d ? a.bh : a.fh;
      s_j.c[d]          = (static_cast<unsigned long long>(h[pivot + 1] - h[pivot]) << a.qbits) | 1u; // the pivot alone
      s_j.m_u[d]        = a.m;
      s_j.edges_td[d]   = 0;
      s_j.seen[d]       = 1;
      s_j.lvl[d] = s_j.bu[d] = s_j.mode[d] = s_j.mat[d] = s_j.fixed[d] = 0;
      s_j.live[d]                                                      = 1;
      s_j.restrict_to[d]                                               = 0;
    }
    if (!resume) s_j.capped = 0;
  }
  int  rc         = SEARCH_DONE;
  bool resume_now = resume; // the first iteration of a resume launch starts at its worklist phase
  for (;; ++glvl) {
    __syncthreads();
    uint32_t const s_out = (glvl + 1) % 3, s_clr = (glvl + 2) % 3;
    if (!resume_now) {
      // frontiers that return to top-down are built from the sweeps' finds first
      if (s_j.mat[0] || s_j.mat[1]) {
#pragma unroll 1
        for (int d = 0; d < 2; ++d)
          if (s_j.mat[d]) {
            jdir const D = joint_dir(a, d);
            materialize_scanned(a.n, D.fresh, jbuf(D, glvl), D.mat_q, a.qbits, D.td_head, a.m, sm);
          }
        if (!gsync(a, epoch)) return SEARCH_FAILED;
        stamp(a, 7);
        if (threadIdx.x == 0)
          for (int d = 0; d < 2; ++d)
            if (s_j.mat[d]) s_j.c[d] = __ldcg(joint_dir(a, d).mat_q);
        if (tally) st->mats += (s_j.mat[0] ? 1u : 0u) + (s_j.mat[1] ? 1u : 0u);
      }
      if (threadIdx.x == 0) {
        if (blockIdx.x == 0)
          for (int d = 0; d < 2; ++d) {
            jdir const D = joint_dir(a, d);
            D.lq[s_clr]  = 0;
            if (!s_j.mat[d]) *D.mat_q = 0;
          }
        bool async = a.aw != nullptr, live = false;
        s_j.restrict_to[0] = s_j.restrict_to[1] = 0; // one pass, in the level the partner ended
        for (int d = 0; d < 2; ++d) {
          s_j.kind[d] = JK_NONE;
          if (!s_j.live[d]) continue;
          unsigned long long const c  = s_j.c[d];
          uint64_t const           qn = c & qmask, mf = c >> a.qbits;
          if (qn == 0) {
            // the search ran dry: rows the sweeps cut short are walked to the
            // end in slices; it ends when a fix-up step finds nothing
            if (__ldcg(joint_dir(a, d).cut_n) == 0 || s_j.fixed[d]) {
              s_j.live[d] = 0;
              if (s_j.live[d ^ 1]) s_j.restrict_to[d ^ 1] = 1; // the other search keeps only this one's set
              continue;
            }
            s_j.kind[d] = JK_FIXUP;
            async       = false;
            live        = true;
            continue;
          }
          live          = true;
          s_j.fixed[d]  = 0;
          if (s_j.lvl[d] >= a.cap || qn > a.n || mf > a.m) {
            // level cap; or counters beyond the graph, which a correct search
            // never produces (then nothing more is read or written)
            s_j.capped = 1;
            break;
          }
          if (s_j.mat[d]) s_j.mode[d] = 0;
          else if (s_j.mode[d] == 0 && mf * a.alpha > s_j.m_u[d]) s_j.mode[d] = 1;
          s_j.kind[d] = s_j.mode[d] ? JK_BU : JK_TD;
          s_j.grp[d]  = s_j.mode[d] ? bu_group_size(n_und > s_j.seen[d] ? n_und - s_j.seen[d] : 0, a.n) : 1u;
          if (!(s_j.mode[d] == 0 && s_j.lvl[d] >= ASYNC_AFTER && qn <= ASYNC_FRONTIER)) async = false;
        }
        s_j.async  = async && live && !s_j.capped;
        s_j.any_td = s_j.kind[0] == JK_TD || s_j.kind[1] == JK_TD;
        s_j.any_bu = s_j.kind[0] == JK_BU || s_j.kind[1] == JK_BU;
        if (!live) s_j.capped |= 2; // both searches are done
        s_j.cnt[0] = s_j.cnt[1] = 0;
      }
      __syncthreads();
      if (s_j.capped) break;
      // a search that lost its partner: keep only candidates in the partner's set
#pragma unroll 1
      for (int d = 0; d < 2; ++d)
        if (s_j.restrict_to[d] && s_j.live[d]) {
          if (tally) st->restricts += 1;
          uint32_t* const       av = joint_dir(a, d).avail;
          uint32_t const* const ot = joint_dir(a, d ^ 1).mark;
          for (uint32_t w = blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) {
            uint32_t const keep = __ldcg(ot + w), cur = __ldcg(av + w);
            if (cur & ~keep) atomicAnd(av + w, keep);
          }
        }
    }
    resume_now = false;
    if (MINB != 2 && s_j.async) {
      // the worklist phase runs in a launch with more registers per thread
      // (its hop chains stay in flight without spills): save the control
      // and end this launch; the resume launch starts at this point
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        auto* const js = static_cast<joint_save*>(a.jsave);
        js->j          = s_j;
        js->glvl       = glvl;
        js->n_und      = n_und;
        js->barriers   = epoch - s_epoch0;
        st->handoff    = 1;
      }
      return SEARCH_HANDOFF;
    }
    if constexpr (MINB == 2) {
      if (s_j.async) {
        // long and thin: both searches finish on the worklist
        uint64_t   ea = 0;
        int const  d0 = s_j.live[0] ? 0 : 1;
        bool const two = s_j.live[0] && s_j.live[1];
        jdir const D0 = joint_dir(a, d0), D1 = joint_dir(a, 1);
        aw_dir const w0{ D0.td_head, D0.td_adj, D0.avail, D0.mark };
        aw_dir const w1{ D1.td_head, D1.td_adj, D1.avail, D1.mark };
        frontier_buf const f0 = s_j.lvl[d0] == 0 ? a.seed : jbuf(D0, glvl);
        frontier_buf const f1 = s_j.lvl[1] == 0 ? a.seed : jbuf(D1, glvl);
        int const r = run_async(a, f0.q, static_cast<uint32_t>(s_j.c[d0] & qmask), w0, f1.q, static_cast<uint32_t>(s_j.c[1] & qmask), two ? &w1 : nullptr, epoch, ea, sm);
        if (r != SEARCH_DONE) return r;
        stamp(a, 13);
        if (threadIdx.x == 0) {
          s_j.edges_td[d0] += ea;
          for (int d = 0; d < 2; ++d)
            if (s_j.live[d]) s_j.c[d] = 0, s_j.mode[d] = 0, s_j.mat[d] = 0, s_j.lvl[d] += 1; // nothing queued: next it runs dry (or fixes up cut rows)
        }
        if (tally) st->async_phases += 1;
        continue;
      }
    }
    if (glvl == 0 && a.model && blockIdx.x == gridDim.x - 1 && threadIdx.x < 32) {
      // the pivot model scores the pivot during the first level, in the
      // grid's last block (which expands nothing there unless the pivot's
      // rows span the grid): the learned rule keeps the plain pivot when
      // the model accepts it; a rejection ends the launch at this level's
      // barrier and the host scores every candidate
      float f[MLP_IN], h1, h2;
      mlp_features(pivot, a.fh, a.fc, a.bh, a.bc, f);
      float const z = mlp_forward_w(mlp_weights_global{ a.model }, f, h1, h2);
      if (threadIdx.x == 0 && !(z >= 0.f)) st->pivot_rejected = 1;
    }
    // ---- the level's steps
    if (s_j.any_td || s_j.kind[0] == JK_FIXUP || s_j.kind[1] == JK_FIXUP) {
      uint32_t ntl[2] = { 0, 0 }, parts[2] = { 1, 1 }, units[2] = { 0, 0 };
      uint32_t const share = s_j.kind[0] == JK_TD && s_j.kind[1] == JK_TD ? 4u : 2u; // the grid is split between two expansions
#pragma unroll
      for (int d = 0; d < 2; ++d)
        if (s_j.kind[d] == JK_TD) {
          uint64_t const mf = s_j.c[d] >> a.qbits;
          ntl[d]            = static_cast<uint32_t>((mf + EX_TILE - 1) / EX_TILE);
          // few tiles: split each into `parts` slot ranges on separate blocks,
          // so a small frontier still spreads over the grid
          while (parts[d] < EX_ITEMS && static_cast<uint64_t>(ntl[d]) * parts[d] * share <= gridDim.x) parts[d] *= 2;
          units[d] = ntl[d] * parts[d];
        }
      block_queue bq{ sm.buf(), &sm.buf_n };
      for (uint32_t unit = blockIdx.x; unit < units[0] + units[1]; unit += gridDim.x) {
        int const          d    = unit < units[0] ? 0 : 1;
        uint32_t const     u    = d ? unit - units[0] : unit;
        uint32_t const     pd   = d ? parts[1] : parts[0];
        jdir const         D    = joint_dir(a, d);
        frontier_buf const fin  = s_j.lvl[d] == 0 ? a.seed : jbuf(D, glvl);
        int const          per  = EX_ITEMS / static_cast<int>(pd);
        int const          part = static_cast<int>(u % pd);
        take_op const      op{ D.avail, D.mark };
        expand_tile(u / pd, d ? ntl[1] : ntl[0], fin.q, static_cast<uint32_t>(s_j.c[d] & qmask), s_j.c[d] >> a.qbits, fin.prefix, fin.tile_start, D.td_head, D.td_adj, sm.tile_rows(), sm.tile_i, bq, op,
                    part * per, part * per + per, reinterpret_cast<uint32_t*>(sm.warp) + EX_TILE + BU_BUF,
                    reinterpret_cast<uint64_t*>(reinterpret_cast<uint32_t*>(sm.warp) + EX_TILE + BU_BUF + 512));
        flush_scanned(sm, jbuf(D, glvl + 1), &D.lq[s_out], a.qbits, D.td_head, a.n, a.m);
      }
#pragma unroll 1
      for (int d = 0; d < 2; ++d)
        if (s_j.kind[d] == JK_FIXUP) {
          jdir const     D   = joint_dir(a, d);
          uint32_t const nc  = __ldcg(D.cut_n);
          uint32_t const lim = nc < a.heavy_cap ? nc : a.heavy_cap;
          for (uint32_t off = 0; off < lim; off += BU_BUF / 2) {
            uint32_t const k = lim - off < BU_BUF / 2 ? lim - off : BU_BUF / 2; // at most k joins: the block queue holds them
            heavy_slices(D.cut_list + off, k, D.bu_head, [&](uint32_t, uint32_t v, uint64_t b, uint64_t e) {
              if (!((__shfl_sync(0xFFFFFFFFu, __ldcg(D.avail + (v >> 5)), 0) >> (v & 31)) & 1u)) return; // joined meanwhile
              bool hit = false;
              for (uint64_t x = b; x < e; x += 32) {
                bool const     in = x + lane < e;
                uint32_t const y  = in ? D.bu_adj[x + lane] : 0u;
                bool const     h  = in && ((__ldcg(D.mark + (y >> 5)) >> (y & 31)) & 1u);
                if (__any_sync(0xFFFFFFFFu, h)) {
                  hit = true;
                  break;
                }
              }
              bool const took = hit && lane == 0 && bit_take(D.avail, v);
              if (took) bit_claim(D.mark, v);
              bq.push(took, v);
            });
            flush_scanned(sm, jbuf(D, glvl + 1), &D.lq[s_out], a.qbits, D.td_head, a.n, a.m);
          }
          if (tally) st->fixups += 1;
        }
    }
    if (s_j.any_bu) {
      // both searches' chunks (or sparse groups of chunks) in one range,
      // spread over every warp of the grid
      uint32_t const chunks = (words + 31) / 32;
      uint32_t const g0     = s_j.grp[0], g1 = s_j.grp[1];
      uint32_t const c0     = s_j.kind[0] == JK_BU ? (chunks + g0 - 1) / g0 : 0u;
      uint32_t const c1     = s_j.kind[1] == JK_BU ? (chunks + g1 - 1) / g1 : 0u;
      uint32_t       nf0 = 0, nf1 = 0;
      uint64_t       ne = 0, ncd = 0;
      for (uint32_t cc = blockIdx.x * BU_WARPS + wid; cc < c0 + c1; cc += gridDim.x * BU_WARPS) {
        int const      d  = cc < c0 ? 0 : 1;
        jdir const     D  = joint_dir(a, d);
        uint32_t const gs = d ? g1 : g0;
        uint32_t const ch = (d ? cc - c0 : cc) * gs;
        uint32_t       f  = 0;
        bu_sweep_group(ch, chunks - ch < gs ? chunks - ch : gs, a.n, D.bu_head, D.bu_adj, D.avail, D.mark, D.fresh, s_bu_cut[d], sm.warp[wid], f, ne, ncd);
        if (d) nf1 += f;
        else nf0 += f;
      }
#pragma unroll
      for (int sh = 16; sh; sh >>= 1) {
        nf0 += __shfl_down_sync(0xFFFFFFFFu, nf0, sh);
        nf1 += __shfl_down_sync(0xFFFFFFFFu, nf1, sh);
        ne += __shfl_down_sync(0xFFFFFFFFu, ne, sh);
      }
      if (lane == 0) {
        if (nf0) atomicAdd(&s_j.cnt[0], nf0);
        if (nf1) atomicAdd(&s_j.cnt[1], nf1);
        if (ne) atomicAdd(&sm.edges_bu, static_cast<unsigned long long>(ne));
        if (ncd) atomicAdd(&sm.cands_bu, static_cast<unsigned long long>(ncd)); // counted by lane 0
      }
      __syncthreads();
      if (threadIdx.x == 0)
        for (int d = 0; d < 2; ++d)
          if (s_j.cnt[d]) atomicAdd(&joint_dir(a, d).lq[s_out], static_cast<unsigned long long>(s_j.cnt[d])); // vertices only
      if (tally) st->bu_bitmap += (c0 ? 1u : 0u) + (c1 ? 1u : 0u);
    }
    if (!gsync(a, epoch)) return SEARCH_FAILED;
    if (glvl == 0 && a.model && __ldcg(&st->pivot_rejected)) return SEARCH_REJECTED;
    stamp(a, s_j.any_td ? 4u : (s_j.any_bu ? 5u : 14u));
    if (threadIdx.x == 0) {
      for (int d = 0; d < 2; ++d) {
        uint32_t const k = s_j.kind[d];
        if (k == JK_NONE) continue;
        jdir const               D    = joint_dir(a, d);
        unsigned long long const next = __ldcg(&D.lq[s_out]);
        uint64_t const           mf   = s_j.c[d] >> a.qbits;
        s_j.lvl[d] += 1;
        s_j.mat[d] = 0;
        if (k == JK_FIXUP) {
          s_j.fixed[d] = 1;
          s_j.mode[d]  = 0;
        } else {
          s_j.m_u[d] = s_j.m_u[d] > mf ? s_j.m_u[d] - mf : 0;
          if (k == JK_BU) {
            s_j.bu[d] += 1;
            // stay bottom-up while the sweep found at least n_und / beta vertices
            uint64_t const nx = next & qmask;
            s_j.mat[d]        = nx != 0 && nx * a.beta < n_und;
          } else {
            s_j.edges_td[d] += mf;
            if (tally) st->rows_td += s_j.c[d] & qmask, st->pushed_td += next & qmask;
          }
        }
        s_j.c[d] = next;
        s_j.seen[d] += next & qmask;
      }
    }
  }
  if (s_j.capped & 1) rc = SEARCH_CAPPED;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->levels_fw = s_j.lvl[0], st->bu_fw = s_j.bu[0];
    st->levels_bw = s_j.lvl[1], st->bu_bw = s_j.bu[1];
    st->edges_td += s_j.edges_td[0] + s_j.edges_td[1];
    st->joint = 1;
  }
  // the cut rows' bits leave the cut maps before the next search can cut
  // (its first sweep comes after at least one more barrier)
#pragma unroll 1
  for (int d = 0; d < 2; ++d) {
    jdir const     D  = joint_dir(a, d);
    uint32_t const nc = __ldcg(D.cut_n);
    for (uint32_t i = blockIdx.x * R_THREADS + threadIdx.x; i < nc && i < a.heavy_cap; i += gridDim.x * R_THREADS) {
      uint32_t const v = __ldcg(D.cut_list + i);
      atomicAnd(s_bu_cut[d].map + (v >> 5), ~(1u << (v & 31)));
    }
  }
  // the SCC is FW(p) & BW(p): the min-id search and the finalize pass read
  // both bitmaps, and the finalize pass leaves the intersection in vis_b
  return rc;
}

// ---------------------------------------------------------------- trim tail
// The trim-1 fixpoint on what the FW-BW left undecided, in the same launch.
// Live degrees are counted against `snap` (und as the trim starts, written
// by the finalize pass), so the vertices this first pass decides do not
// disturb the counts; afterwards every decided vertex decrements each
// still-undecided neighbour's count once per edge, and a count reaching 0
// decides that neighbour (one push level per barrier).
constexpr int PIVOT_FROM_DEVICE = -1; // fwbw_args.pivot: take trim_1_first's pivot

__device__ __forceinline__ uint32_t
snap_bit(uint32_t const* snap, uint32_t v)
{
  return (__ldcg(snap + (v >> 5)) >> (v & 31)) & 1u;
}

constexpr uint64_t TRIM_SMALL = 32; // row entries (both directions) a lane counts alone

// Neighbours in adj[b, e) set in snap; four ids, then their four snap
// words, in flight at once.
__device__ __forceinline__ uint32_t
count_live(uint32_t const* snap, uint32_t const* __restrict__ adj, uint64_t b, uint64_t e)
{
  uint32_t c = 0;
  for (; b + 4 <= e; b += 4) {
    uint32_t const x0 = adj[b], x1 = adj[b + 1], x2 = adj[b + 2], x3 = adj[b + 3];
    c += snap_bit(snap, x0) + snap_bit(snap, x1) + snap_bit(snap, x2) + snap_bit(snap, x3);
  }
  for (; b < e; ++b) c += snap_bit(snap, adj[b]);
  return c;
}

// First trim pass: live degrees of every listed undecided vertex; the dead
// ones (no live in- or out-neighbour) are decided and queued.  A lane
// counts one vertex; rows longer than TRIM_SMALL are counted by the whole
// warp; a vertex with a row longer than HEAVY_ROW is listed (heavy list 0,
// st->hseed_n) with both counts zeroed, for run_trim's slice pass.
__device__ __forceinline__ void
trim_seed(fwbw_args const& a, uint32_t const* list, uint64_t list_n, uint32_t* qout, unsigned long long* octr, uint32_t& dec, uint64_t& edges)
{
  unsigned const  lane = threadIdx.x & 31u;
  uint32_t const* snap = a.cand;
  uint64_t const  span = (list_n + 31) & ~31ull;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * R_THREADS) {
    bool const     have = t < list_n;
    uint32_t const x    = have ? __ldcg(list + t) : 0u;
    uint64_t       ob = 0, oe = 0, ib = 0, ie = 0;
    if (have) ob = a.fh[x], oe = a.fh[x + 1], ib = a.bh[x], ie = a.bh[x + 1];
    bool const small = have && (oe - ob) + (ie - ib) <= TRIM_SMALL;
    bool       hv    = false;
    uint32_t   co = 0, ci = 0;
    if (small) {
      co = count_live(snap, a.fc, ob, oe);
      ci = count_live(snap, a.bc, ib, ie);
    }
    for (unsigned todo = __ballot_sync(0xFFFFFFFFu, have && !small); todo; todo &= todo - 1) {
      unsigned const l  = __ffs(todo) - 1;
      uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, ob, l), e0 = __shfl_sync(0xFFFFFFFFu, oe, l);
      uint64_t const b1 = __shfl_sync(0xFFFFFFFFu, ib, l), e1 = __shfl_sync(0xFFFFFFFFu, ie, l);
      if (e0 - b0 > HEAVY_ROW || e1 - b1 > HEAVY_ROW) {
        // listed for the slice pass, counts zeroed for it
        if (lane == l) {
          hv = true;
          a.outdeg[x] = a.indeg[x] = 0;
          uint32_t const i = atomicAdd(&a.st->hseed_n, 1u);
          if (i < a.heavy_cap) a.heavy[i] = x;
          else atomicExch(&a.st->heavy_err, 1u);
        }
        continue;
      }
      uint32_t       xo = 0, xi = 0;
      for (uint64_t e = b0 + lane; e < e0; e += 32) xo += snap_bit(snap, a.fc[e]);
      for (uint64_t e = b1 + lane; e < e1; e += 32) xi += snap_bit(snap, a.bc[e]);
#pragma unroll
      for (int sh = 16; sh; sh >>= 1) xo += __shfl_xor_sync(0xFFFFFFFFu, xo, sh), xi += __shfl_xor_sync(0xFFFFFFFFu, xi, sh);
      if (lane == l) co = xo, ci = xi;
    }
    bool const dead = have && !hv && (co == 0 || ci == 0);
    if (dead) {
      atomicAnd(a.und + (x >> 5), ~(1u << (x & 31)));
      if (!a.ids_at_end) a.scc_id[x] = x;
      ++dec;
    } else if (have && !hv) {
      a.outdeg[x] = co;
      a.indeg[x]  = ci;
    }
    if (have) edges += (oe - ob) + (ie - ib);
    warp_push64(dead, x, qout, octr, a.n);
  }
}

// One trim push level: every queued vertex decrements its undecided
// neighbours' live counts (out-neighbours' in-degree, in-neighbours'
// out-degree); a neighbour whose count reaches 0 is decided and queued.
// Heavy rows of the push levels: a queued vertex's row longer than
// HEAVY_ROW is skipped by its lane and listed instead, in heavy list
// 1 + ((glvl + 1) & 1) -- out-rows from the front, in-rows from the back,
// counted in hq_n[2 * ((glvl + 1) % 3)] and the entry after it -- and the
// next level walks the listed rows in slices over the whole grid (a push
// one level late: the fixpoint does not depend on the order).
struct trim_hq
{
  uint32_t* list; // heavy list of this parity
  uint32_t* n;    // [0] out-rows (front), [1] in-rows (back)
};

__device__ __forceinline__ trim_hq
trim_heavy_at(fwbw_args const& a, uint32_t glvl)
{
  return { a.heavy + (1 + (glvl & 1)) * a.heavy_cap, &a.st->hq_n[2 * (glvl % 3)] };
}

__device__ __forceinline__ void
trim_push(fwbw_args const& a, uint32_t const* qin, uint32_t qn, uint32_t* qout, unsigned long long* octr, uint32_t& dec, uint64_t& edges, uint32_t glvl)
{
  unsigned const lane = threadIdx.x & 31u;
  trim_hq const  hin = trim_heavy_at(a, glvl), hout = trim_heavy_at(a, glvl + 1);
  uint32_t const hn0 = __ldcg(hin.n), hn1 = __ldcg(hin.n + 1); // issued early
  uint64_t const span = (static_cast<uint64_t>(qn) + 31) & ~31ull;
  // w's und word already probed: decrement, decide and queue at 0
  auto const hit = [&](uint32_t w, uint32_t word, uint32_t* deg) {
    if (((word >> (w & 31)) & 1u) && atomicSub(deg + w, 1u) == 1u && bit_take(a.und, w)) {
      if (!a.ids_at_end) a.scc_id[w] = w;
      ++dec;
      warp_push_active64(w, qout, octr, a.n);
    }
  };
  // a lane's own row: four neighbour ids, then their four und words, in
  // flight at once
  auto const row = [&](uint32_t const* adj, uint64_t b, uint64_t e, uint32_t* deg) {
    for (; b + 4 <= e; b += 4) {
      uint32_t w[4], u[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) w[k] = adj[b + k];
#pragma unroll
      for (int k = 0; k < 4; ++k) u[k] = __ldcg(a.und + (w[k] >> 5));
#pragma unroll
      for (int k = 0; k < 4; ++k) hit(w[k], u[k], deg);
    }
    for (; b < e; ++b) {
      uint32_t const w = adj[b];
      hit(w, __ldcg(a.und + (w >> 5)), deg);
    }
  };
#pragma unroll 1
  for (int dir = 0; dir < 2; ++dir) {
    uint64_t const* head = dir ? a.bh : a.fh;
    uint32_t const* adj  = dir ? a.bc : a.fc;
    uint32_t*       deg  = dir ? a.outdeg : a.indeg;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * R_THREADS) {
      bool const     have = t < qn;
      uint32_t const u    = have ? __ldcg(qin + t) : 0u;
      uint64_t       b = 0, e = 0;
      if (have) b = head[u], e = head[u + 1];
      bool const big = have && e - b >= TRIM_SMALL;
      edges += e - b;
      if (have && !big) row(adj, b, e, deg);
      for (unsigned todo = __ballot_sync(0xFFFFFFFFu, big); todo; todo &= todo - 1) {
        unsigned const l  = __ffs(todo) - 1;
        uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, b, l), e0 = __shfl_sync(0xFFFFFFFFu, e, l);
        if (e0 - b0 > HEAVY_ROW) {
          // listed for the next level's slices (front: out-rows, back:
          // in-rows; they never meet, heavy_capacity covers both)
          if (lane == l) {
            uint32_t const i = atomicAdd(hout.n + dir, 1u);
            if (i < a.heavy_cap / 2) hout.list[dir ? a.heavy_cap - 1 - i : i] = u;
            else atomicExch(&a.st->heavy_err, 1u);
          }
          continue;
        }
        for (uint64_t x = b0 + lane; x < e0; x += 32) {
          uint32_t const w = adj[x];
          hit(w, __ldcg(a.und + (w >> 5)), deg);
        }
      }
    }
    uint32_t const hn = dir ? hn1 : hn0;
    heavy_slices(dir ? hin.list + a.heavy_cap - hn : hin.list, hn, head, [&](uint32_t, uint32_t, uint64_t b0, uint64_t e0) {
      for (uint64_t x = b0 + lane; x < e0; x += 32) {
        uint32_t const w = adj[x];
        hit(w, __ldcg(a.und + (w >> 5)), deg);
      }
    });
  }
}

// Live degrees of the hs listed heavy vertices (heavy list 0), counted in
// slices against snap.
__device__ __forceinline__ void
trim_count_heavy(fwbw_args const& a, uint32_t hs)
{
  unsigned const lane = threadIdx.x & 31u;
#pragma unroll 1
  for (int dir = 0; dir < 2; ++dir) {
    uint32_t const* adj = dir ? a.bc : a.fc;
    uint32_t* const deg = dir ? a.indeg : a.outdeg;
    heavy_slices(a.heavy, hs, dir ? a.bh : a.fh, [&](uint32_t, uint32_t x, uint64_t b, uint64_t e) {
      uint32_t c = 0;
      for (uint64_t y = b + lane; y < e; y += 32) c += snap_bit(a.cand, adj[y]);
#pragma unroll
      for (int sh = 16; sh; sh >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, sh);
      if (lane == 0 && c) atomicAdd(deg + x, c);
    });
  }
}

// First push level: the listed heavy vertices with a live degree of 0 are
// decided and queued (their rows are listed by the next level's walk);
// returns how many this thread decided.
__device__ __forceinline__ uint32_t
trim_dead_heavy(fwbw_args const& a, uint32_t hs, uint32_t glvl)
{
  uint32_t dec = 0;
  for (uint32_t i = blockIdx.x * R_THREADS + threadIdx.x; i < hs; i += gridDim.x * R_THREADS) {
    uint32_t const x = __ldcg(a.heavy + i);
    if ((__ldcg(a.outdeg + x) == 0 || __ldcg(a.indeg + x) == 0) && bit_take(a.und, x)) {
      if (!a.ids_at_end) a.scc_id[x] = x;
      ++dec;
      warp_push_active64(x, a.fb[(glvl + 1) & 1].q, &a.st->lq[(glvl + 1) % 3], a.n);
    }
  }
  return dec;
}

// ---------------------------------------------------------------- trim worklist tail
// A long, thin trim (peeling chains: thousands of levels of a few vertices
// each) finishes on the same worklist as the search tail instead of one
// grid barrier per level.  Items: AW_TAG | v (a decided vertex: push both
// rows), or AW_TAG | AW_SLICE | dir << 63 | slice << 33 | v (slice `slice`
// of v's out- (dir 0) or in-row (dir 1), for rows longer than HEAVY_ROW).
// A warp takes 32 items; per direction its lanes split the edges of the
// items' rows (warp scan of the lengths), and a neighbour whose live count
// reaches 0 is decided and appended.  Ends when every appended item is
// done; every wait is bounded.
constexpr unsigned long long AW_SLICE = 1ull << 62;

__device__ __forceinline__ void
aw_push_item(unsigned long long item, bool pred, unsigned long long* aw, unsigned long long* tail, uint64_t cap)
{
  unsigned const mask = __ballot_sync(0xFFFFFFFFu, pred);
  if (!mask) return;
  unsigned const     lane = threadIdx.x & 31u, leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane == leader) base = atomicAdd(tail, static_cast<unsigned long long>(__popc(mask)));
  base                = __shfl_sync(0xFFFFFFFFu, base, leader);
  uint64_t const slot = base + __popc(mask & ((1u << lane) - 1u));
  if (pred && slot < cap) __stcg(aw + slot, item);
}

__device__ __forceinline__ int
run_trim_async(fwbw_args const& a, uint32_t const* fq, uint32_t qn, unsigned long long& epoch, uint32_t& dec, uint64_t& edges)
{
  unsigned long long* const aw   = a.aw;
  unsigned long long* const head = a.aq;
  unsigned long long* const tail = a.aq + 16;
  unsigned long long* const done = a.aq + 32;
  uint64_t const            cap  = a.aw_cap;
  unsigned const            lane = threadIdx.x & 31u;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; i < qn; i += static_cast<uint64_t>(gridDim.x) * R_THREADS) __stcg(aw + i, AW_TAG | __ldcg(fq + i));
  if (blockIdx.x == 0 && threadIdx.x == 0) *head = 0, *tail = qn, *done = 0;
  if (!gsync(a, epoch)) return SEARCH_FAILED;
  bool     failed      = false;
  uint32_t unpublished = 0;
  for (bool alive = true; alive;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(head, 32ull);
    base                = __shfl_sync(0xFFFFFFFFu, base, 0);
    uint64_t const slot = base + lane;
    bool           pending = true;
    unsigned       spins   = 0;
    while (__any_sync(0xFFFFFFFFu, pending)) {
      bool               got  = false;
      unsigned long long item = 0;
      if (pending && slot < cap) {
        item = ld_acquire64(aw + slot);
        if (item & AW_TAG) got = true, pending = false;
      }
      unsigned const gmask = __ballot_sync(0xFFFFFFFFu, got);
      if (gmask) {
        uint32_t const v = static_cast<uint32_t>(item);
#pragma unroll 1
        for (int dir = 0; dir < 2; ++dir) {
          uint64_t const* hd  = dir ? a.bh : a.fh;
          uint32_t const* adj = dir ? a.bc : a.fc;
          uint32_t* const deg = dir ? a.outdeg : a.indeg;
          uint64_t        b = 0, e = 0;
          if (got) {
            bool const is_slice = (item & AW_SLICE) != 0;
            if (!is_slice || static_cast<int>(item >> 63) == dir) {
              b = hd[v], e = hd[v + 1];
              if (is_slice) {
                b += static_cast<uint64_t>((item >> 33) & 0x1FFFFFFFull) * HEAVY_SLICE;
                e = b + HEAVY_SLICE < e ? b + HEAVY_SLICE : e;
              } else if (e - b > HEAVY_ROW) {
                // a heavy row: its slices become items of their own
                uint64_t const           ns = (e - b + HEAVY_SLICE - 1) / HEAVY_SLICE;
                unsigned long long const at = atomicAdd(tail, static_cast<unsigned long long>(ns));
                for (uint64_t j = 0; j < ns; ++j)
                  if (at + j < cap) __stcg(aw + at + j, AW_TAG | AW_SLICE | (static_cast<unsigned long long>(dir) << 63) | (static_cast<unsigned long long>(j) << 33) | v);
                e = b; // nothing walked here
              }
            }
          }
          edges += e - b;
          // the lanes' rows split over the warp (warp scan of the lengths)
          uint32_t const d    = static_cast<uint32_t>(e - b);
          uint32_t       incl = d;
#pragma unroll
          for (int sh = 1; sh < 32; sh <<= 1) {
            uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, incl, sh);
            if (lane >= static_cast<unsigned>(sh)) incl += y;
          }
          uint32_t const total = __shfl_sync(0xFFFFFFFFu, incl, 31);
          uint32_t const excl  = incl - d;
          for (uint32_t kb = 0; kb < total; kb += 32) {
            uint32_t const k = kb + lane;
            uint32_t       j = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1) {
              uint32_t const ex = __shfl_sync(0xFFFFFFFFu, excl, j + step);
              if (ex <= k) j += step;
            }
            uint64_t const bj   = __shfl_sync(0xFFFFFFFFu, b, j);
            uint32_t const xj   = __shfl_sync(0xFFFFFFFFu, excl, j);
            bool           take = false;
            uint32_t       w    = 0;
            if (k < total) {
              w    = adj[bj + (k - xj)];
              take = ((__ldcg(a.und + (w >> 5)) >> (w & 31)) & 1u) && atomicSub(deg + w, 1u) == 1u && bit_take(a.und, w);
              if (take) {
                if (!a.ids_at_end) a.scc_id[w] = w;
                ++dec;
              }
            }
            aw_push_item(AW_TAG | w, take, aw, tail, cap);
          }
        }
        unpublished += __popc(gmask);
        spins = 0;
      } else {
        if (unpublished) {
          __threadfence();
          if (lane == 0) atomicAdd(done, static_cast<unsigned long long>(unpublished));
          unpublished = 0;
        }
        uint32_t stop = 0;
        if (lane == 0) {
          unsigned long long const dn = ld_acquire64(done);
          unsigned long long const t  = ld_acquire64(tail);
          stop                        = dn == t ? 1u : 0u;
          if (!stop && (++spins > a.wait_limit || ((spins & 63u) == 63u && ld_acquire(&a.bar->err)))) {
            atomicExch(&a.bar->err, 1u);
            stop = 2;
          }
        }
        stop = __shfl_sync(0xFFFFFFFFu, stop, 0);
        if (stop) {
          pending = false;
          alive   = false;
          failed  = stop == 2;
        } else __nanosleep(64);
      }
    }
  }
  if (!gsync(a, epoch) || failed) return SEARCH_FAILED;
  uint64_t t = __ldcg(tail);
  t          = t < cap ? t : cap;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * R_THREADS + threadIdx.x; i < t; i += static_cast<uint64_t>(gridDim.x) * R_THREADS) __stcg(aw + i, 0ull);
  return SEARCH_DONE;
}

// The trim fixpoint; levels continue the launch's numbering (glvl).
__device__ __forceinline__ int
run_trim(fwbw_args const& a, uint32_t& glvl, unsigned long long& epoch)
{
  reach_state* const       st    = a.st;
  unsigned long long const qmask = (1ull << a.qbits) - 1;
  uint32_t                 dec   = 0;
  uint64_t                 edges = 0;
  uint32_t                 lvl   = 0;
  int                      rc    = SEARCH_DONE;
  if (blockIdx.x == 0 && threadIdx.x == 0) st->lq[(glvl + 2) % 3] = 0;
  // the finalize pass listed the undecided vertices in fb[glvl & 1].q
  trim_seed(a, a.fb[glvl & 1].q, __ldcg(&st->list_n), a.fb[(glvl + 1) & 1].q, &st->lq[(glvl + 1) % 3], dec, edges);
  if (!gsync(a, epoch)) rc = SEARCH_FAILED;
  stamp(a, 11);
  ++glvl;
  uint32_t const hs = rc == SEARCH_DONE ? __ldcg(&st->hseed_n) : 0u;
  if (hs) {
    // the listed heavy vertices' live degrees, counted in slices
    trim_count_heavy(a, hs);
    if (!gsync(a, epoch)) rc = SEARCH_FAILED;
    stamp(a, 15);
  }
  while (rc == SEARCH_DONE) {
    uint64_t const qn    = __ldcg(&st->lq[glvl % 3]) & qmask;
    bool const     first = lvl == 0 && hs; // also decides the dead heavy vertices
    if (qn == 0 && !first && __ldcg(&st->hq_n[2 * (glvl % 3)]) == 0 && __ldcg(&st->hq_n[2 * (glvl % 3) + 1]) == 0) break;
    if (lvl >= a.cap || qn > a.n) {
      rc = SEARCH_CAPPED;
      break;
    }
    if (lvl >= ASYNC_AFTER && qn <= ASYNC_FRONTIER && a.aw && !first && __ldcg(&st->hq_n[2 * (glvl % 3)]) == 0 && __ldcg(&st->hq_n[2 * (glvl % 3) + 1]) == 0) {
      // long and thin: the rest of the fixpoint on the worklist (no heavy
      // rows are pending from the level before)
      rc = run_trim_async(a, a.fb[glvl & 1].q, static_cast<uint32_t>(qn), epoch, dec, edges);
      stamp(a, 16);
      if (blockIdx.x == 0 && threadIdx.x == 0) st->trim_async = 1;
      ++lvl;
      break;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->lq[(glvl + 2) % 3] = 0, st->hq_n[2 * ((glvl + 2) % 3)] = st->hq_n[2 * ((glvl + 2) % 3) + 1] = 0;
    if (first) dec += trim_dead_heavy(a, hs, glvl);
    trim_push(a, a.fb[glvl & 1].q, static_cast<uint32_t>(qn), a.fb[(glvl + 1) & 1].q, &st->lq[(glvl + 1) % 3], dec, edges, glvl);
    if (!gsync(a, epoch)) rc = SEARCH_FAILED;
    stamp(a, 12);
    ++lvl;
    ++glvl;
  }
  // one atomic per block for each tally
  uint64_t d_all, e_all;
  block_exclusive_scan<uint64_t, R_THREADS>(dec, &d_all);
  block_exclusive_scan<uint64_t, R_THREADS>(edges, &e_all);
  if (threadIdx.x == 0 && d_all) atomicAdd(&st->trim_decided, static_cast<uint32_t>(d_all)), atomicSub(&st->und_left, static_cast<uint32_t>(d_all));
  if (threadIdx.x == 0 && e_all) atomicAdd(&st->trim_edges, static_cast<unsigned long long>(e_all));
  if (blockIdx.x == 0 && threadIdx.x == 0) st->trim_levels = lvl;
  return rc;
}

// All ids from the bitmaps: a warp covers 32 words (1024 vertices), lane l
// writing vertices 128j + 4l .. +3 of them (512 contiguous bytes per store
// instruction; 16-byte stores when the output is 16-byte aligned).
__device__ __forceinline__ void
write_ids(fwbw_args const& a, uint32_t words, bool search, uint32_t scc)
{
  unsigned const lane = threadIdx.x & 31u;
  bool const     vec  = (reinterpret_cast<uintptr_t>(a.scc_id) & 15u) == 0;
  for (uint32_t wb = (blockIdx.x * R_THREADS + threadIdx.x) & ~31u; wb < words; wb += gridDim.x * R_THREADS) {
    uint32_t const w   = wb + lane;
    uint32_t const und = w < words ? __ldcg(a.und + w) : 0u;
    uint32_t const mem = search && w < words ? __ldcg(a.vis_b + w) : 0u;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      unsigned const src = j * 4 + (lane >> 3);
      uint32_t const uw  = __shfl_sync(0xFFFFFFFFu, und, src);
      uint32_t const mw  = __shfl_sync(0xFFFFFFFFu, mem, src);
      unsigned const b0  = (lane & 7u) * 4;
      uint64_t const v0  = (static_cast<uint64_t>(wb) + src) * 32 + b0;
      uint32_t       o[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) o[i] = ((mw >> (b0 + i)) & 1u) ? scc : (((uw >> (b0 + i)) & 1u) ? UNDECIDED : static_cast<uint32_t>(v0 + i));
      if (vec && v0 + 4 <= a.n) *reinterpret_cast<uint4*>(a.scc_id + v0) = make_uint4(o[0], o[1], o[2], o[3]);
      else
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (v0 + i < a.n) a.scc_id[v0 + i] = o[i];
    }
  }
}

// MINB: blocks per SM the launch is compiled for.  The level loop runs
// with 4 (64 registers per thread); a search that moves to the worklist
// phase hands off to a resume launch with 2 (128 registers), whose hop
// chains keep their loads in flight without spills.
template<int MINB>
__global__ void __launch_bounds__(R_THREADS, MINB)
k_fwbw(fwbw_args a)
{
  __shared__ fwbw_smem sm;
  reach_state* const   st    = a.st;
  unsigned long long   epoch = __ldcg(&a.bar->epoch);
  uint32_t const       words = (a.n + 31) / 32;
  uint32_t             p     = a.pivot;
  if (p == static_cast<uint32_t>(PIVOT_FROM_DEVICE)) {
    // trim_1_first's choice: largest in*out among its survivors; none
    // (product 0) when it decided every vertex
    uint64_t const prod = __ldcg(a.pv_prod);
    uint32_t const id   = __ldcg(a.pv_id);
    p                   = prod == 0 || id >= a.n ? a.n : id;
  }
  bool const search = p < a.n; // block-uniform
  // a resume launch numbers its barriers on from the launch it continues
  if (threadIdx.x == 0) sm.buf_n = 0, sm.edges_bu = sm.cands_bu = 0, s_epoch0 = a.resume ? epoch - static_cast<joint_save const*>(a.jsave)->barriers : epoch;
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.resume) st->handoff = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0 && !a.resume) {
    st->t_ns[0] = globaltimer();
    st->marks   = 0;
    stamp(a, 0);
    st->lq[0] = st->lq[1] = st->lq[2] = 0;
    st->lq_bw[0] = st->lq_bw[1] = st->lq_bw[2] = 0;
    st->mat_q = st->mat_q_bw = 0;
    st->id                            = UNDECIDED;
    st->decided                       = 0;
    st->edges_bu = st->cands_bu = st->edges_td = 0;
    st->levels_fw = st->bu_fw = st->levels_bw = st->bu_bw = 0;
    st->pivot_used                                        = p;
    st->trim_decided = st->trim_levels = st->und_left = 0;
    st->trim_edges = st->list_n                       = 0;
    st->rows_td = st->pushed_td = 0;
    st->mats = st->bu_bitmap    = 0;
    st->async_phases            = 0;
    st->cut_n[0] = st->cut_n[1] = st->fixups = 0;
    st->hseed_n = st->heavy_err = st->trim_async = st->joint = st->restricts = 0;
    st->pivot_rejected = st->handoff = 0;
    for (int i = 0; i < 6; ++i) st->hq_n[i] = 0;
    if (search) a.seed.q[0] = p, a.seed.prefix[0] = 0;
  }
  int      rc   = SEARCH_DONE;
  uint32_t glvl = 0;
  uint32_t id   = p;
  uint32_t n_und = 0;
  if (search && a.resume) {
    auto const* js = static_cast<joint_save const*>(a.jsave);
    glvl           = js->glvl;
    n_und          = js->n_und;
  } else if (search) {
    // init: cand = und \ {p}, vis_a = vis_b = {p}; |und| per block
    uint32_t c = 0;
    for (uint32_t w = blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) {
      uint32_t const u   = __ldcg(a.und + w);
      uint32_t const pin = w == (p >> 5) ? 1u << (p & 31) : 0u;
      a.cand[w]          = u & ~pin;
      a.vis_a[w]         = pin;
      a.vis_b[w]         = pin;
      a.cand_bw[w]       = u & ~pin;
      c += __popc(u);
    }
    uint64_t tot;
    block_exclusive_scan<uint64_t, R_THREADS>(c, &tot);
    if (threadIdx.x == 0) a.partial[blockIdx.x] = tot;
    rc = gsync(a, epoch) ? SEARCH_DONE : SEARCH_FAILED;
    if (rc == SEARCH_DONE) {
      stamp(a, 8);
      uint64_t s = 0;
      for (uint32_t i = threadIdx.x; i < gridDim.x; i += R_THREADS) s += __ldcg(a.partial + i);
      block_exclusive_scan<uint64_t, R_THREADS>(s, &tot);
      n_und = static_cast<uint32_t>(tot);
    }
  }
  if (search) {
    if (rc == SEARCH_DONE) rc = run_joint<MINB>(a, sm, p, n_und, glvl, epoch, a.resume != 0);
    if (rc == SEARCH_DONE && a.min_ids) {
      // smallest member = first set bit of vis_a & vis_b.  Every block first looks
      // at the same leading MIN_WORDS words (the SCC is usually dense
      // there); only when they are all empty does the grid search the rest
      // and meet at a barrier.  Every block reads the same words, so all
      // take the same branch.
      constexpr uint32_t MIN_WORDS = 4 * R_THREADS;
      uint32_t           best      = UNDECIDED;
      for (uint32_t w = threadIdx.x; w < MIN_WORDS && w < words; w += R_THREADS) {
        uint32_t const s = __ldcg(a.vis_b + w) & __ldcg(a.vis_a + w);
        if (s) {
          best = w * 32 + (__ffs(s) - 1);
          break;
        }
      }
      best = __reduce_min_sync(0xFFFFFFFFu, best);
      if ((threadIdx.x & 31) == 0) sm.cnt = UNDECIDED;
      __syncthreads();
      if ((threadIdx.x & 31) == 0 && best != UNDECIDED) atomicMin(&sm.cnt, best);
      __syncthreads();
      id = sm.cnt;
      if (id == UNDECIDED) {
        for (uint32_t w = MIN_WORDS + blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) {
          uint32_t const s = __ldcg(a.vis_b + w) & __ldcg(a.vis_a + w);
          if (s) {
            best = w * 32 + (__ffs(s) - 1);
            break; // later words of this thread only hold larger ids
          }
        }
        best = __reduce_min_sync(0xFFFFFFFFu, best);
        if ((threadIdx.x & 31) == 0 && best != UNDECIDED && best < __ldcg(&st->id)) atomicMin(&st->id, best);
        if (!gsync(a, epoch)) rc = SEARCH_FAILED;
        id = __ldcg(&st->id);
      }
    }
    if (rc == SEARCH_DONE) {
      // the SCC (vis_b) leaves und with its id; a warp loads 32 words at
      // once, then for each non-empty one lane l writes vertex 32w + l (one
      // coalesced 128-byte store per word).  With the trim tail every word
      // of und is also copied to snap (cand).
      unsigned const  lane = threadIdx.x & 31u;
      uint32_t        cnt = 0, left = 0;
      uint32_t* const list = a.fb[glvl & 1].q; // trim: the undecided vertices
      for (uint32_t wb = (blockIdx.x * R_THREADS + threadIdx.x) & ~31u; wb < words; wb += gridDim.x * R_THREADS) {
        uint32_t const w    = wb + lane;
        uint32_t const vb   = w < words ? __ldcg(a.vis_b + w) : 0u;
        uint32_t const mine = vb & (w < words ? __ldcg(a.vis_a + w) : 0u); // the SCC: FW & BW
        uint32_t       u    = 0;
        if (mine != vb) a.vis_b[w] = mine; // the ids pass reads the SCC from vis_b
        if (w < words && (mine || a.trim)) {
          u = __ldcg(a.und + w) & ~mine;
          if (mine) a.und[w] = u;
          if (a.trim) a.cand[w] = u, left += __popc(u);
          cnt += __popc(mine);
        }
        if (a.trim) {
          // append the word's undecided vertices to the list (one atomic per warp)
          uint32_t const c = __popc(u);
          uint32_t       p = c;
#pragma unroll
          for (int d = 1; d < 32; d <<= 1) {
            uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, p, d);
            if (lane >= static_cast<unsigned>(d)) p += y;
          }
          uint32_t const     tot  = __shfl_sync(0xFFFFFFFFu, p, 31);
          unsigned long long base = 0;
          if (lane == 31 && tot) base = atomicAdd(&st->list_n, static_cast<unsigned long long>(tot));
          base = __shfl_sync(0xFFFFFFFFu, base, 31) + p - c;
          for (; u; u &= u - 1, ++base)
            if (base < a.n) list[base] = w * 32 + __ffs(u) - 1;
        }
        if (!a.ids_at_end)
          for (unsigned todo = __ballot_sync(0xFFFFFFFFu, mine != 0); todo; todo &= todo - 1) {
            unsigned const j = __ffs(todo) - 1;
            uint32_t const s = __shfl_sync(0xFFFFFFFFu, mine, j);
            if ((s >> lane) & 1u) a.scc_id[(wb + j) * 32 + lane] = id;
          }
      }
#pragma unroll
      for (int sh = 16; sh; sh >>= 1) cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, sh), left += __shfl_down_sync(0xFFFFFFFFu, left, sh);
      if (lane == 0 && cnt) atomicAdd(&st->decided, cnt);
      if (lane == 0 && left) atomicAdd(&st->und_left, left); // the trim subtracts its decisions
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) st->t_ns[1] = globaltimer();
    stamp(a, 10);
    if (rc == SEARCH_DONE && a.trim) {
      rc = gsync(a, epoch) ? SEARCH_DONE : SEARCH_FAILED; // snap and und complete
      if (rc == SEARCH_DONE) rc = run_trim(a, glvl, epoch);
    }
  }
  if (a.ids_at_end && rc == SEARCH_DONE) {
    // every vertex's id in one coalesced pass (und is final: after the
    // trim's last barrier, or untouched by this launch without a pivot):
    // SCC members the SCC's id, other decided vertices themselves (trim_1_first
    // and the trim decide singletons), undecided ones UNDECIDED
    write_ids(a, words, search, id);
  }
  if (!search && a.trim) {
    // no pivot: und is untouched, count it (with a pivot, und_left is the
    // finalize pass's count minus the trim's decisions)
    uint32_t c = 0;
    for (uint32_t w = blockIdx.x * R_THREADS + threadIdx.x; w < words; w += gridDim.x * R_THREADS) c += __popc(__ldcg(a.und + w));
#pragma unroll
    for (int sh = 16; sh; sh >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, sh);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&st->und_left, c);
  }
  // statistics
  __syncthreads();
  if (threadIdx.x == 0 && sm.edges_bu) atomicAdd(&st->edges_bu, sm.edges_bu);
  if (threadIdx.x == 0 && sm.cands_bu) atomicAdd(&st->cands_bu, sm.cands_bu);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->id      = id;
    st->err     = rc == SEARCH_CAPPED ? 1u : 0u;
    st->bar_err = rc == SEARCH_FAILED ? 1u : 0u;
    if (rc != SEARCH_FAILED) a.bar->epoch = epoch; // every block completed the same barriers
    if (!search) st->t_ns[1] = st->t_ns[0];
    st->t_ns[2] = globaltimer();
    stamp(a, 9);
  }
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
  bu_cut const cut{ ws.cutmap, ws.heavy + 3 * ws.heavy_cap, &st->cut_n[0], static_cast<uint32_t>(ws.heavy_cap), &st->heavy_err };
  k_bottom_up<<<bu_grid(gr.n), R_THREADS, 0, s>>>(gr.n, io.bu_head, io.bu_adj, io.avail, io.mark, io.fresh, f, gate{ &st->mode, 1 }, st, cut);
  k_bu_cut_rows<<<148 * 8, R_THREADS, 0, s>>>(io.bu_head, io.bu_adj, io.avail, io.mark, io.fresh, f, gate{ &st->mode, 1 }, cut);
  k_bu_cut_clear<<<148, R_THREADS, 0, s>>>(gate{ &st->mode, 1 }, cut);
  prof_stop(ctx, 1);
  k_r_advance<BW><<<1, 1, 0, s>>>(st);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 10;
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

unsigned
bit_width64(uint64_t x)
{
  return x ? 64u - static_cast<unsigned>(__builtin_clzll(x)) : 0u;
}

// The packed level counters hold a frontier's vertices in the low qbits and
// its edges above them; the frontier built from `fresh` packs (edges << 16 |
// vertices) per block pass.
bool
packed_counters_fit(uint32_t n, uint64_t m)
{
  return bit_width64(n) + bit_width64(m) <= 64 && m < (1ull << 48);
}

// Grid of the persistent FW-BW: every block resident at once (which the
// grid barrier needs), fixed per context (the barrier's epoch count assumes
// the same grid at every launch).
unsigned
fwbw_grid(kspn_context* ctx)
{
  if (!ctx->search_grid) {
    int bps = 0, sms = 0;
    KSPN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_fwbw<4>, R_THREADS, 0));
    KSPN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (bps < 1) throw error{ KSPN_ERR_CUDA, "persistent FW-BW kernel does not fit on an SM" };
    // at most AW_GRID_MAX blocks: the worklist's spare slots (AW_STALE)
    // are sized for that many warps
    ctx->search_grid = static_cast<unsigned>(std::min<int>(bps * sms, AW_GRID_MAX));
  }
  return ctx->search_grid;
}

// The grid barrier's arrival counter advances by the grid size per
// barrier (a wait's target is epoch x grid), so it restarts from zero when a
// launch's grid differs from the last one's on this barrier.
void
barrier_for_grid(kspn_context* ctx, unsigned grid)
{
  if (ctx->bar_grid == grid) return;
  KSPN_CUDA(cudaMemsetAsync(ctx->ws.gbar, 0, offsetof(grid_barrier, err), ctx->stream));
  ctx->bar_grid = grid;
}

unsigned
resume_grid(kspn_context* ctx)
{
  if (!ctx->resume_grid) {
    int bps = 0, sms = 0;
    KSPN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_fwbw<2>, R_THREADS, 0));
    KSPN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    if (bps < 1) throw error{ KSPN_ERR_CUDA, "persistent FW-BW resume kernel does not fit on an SM" };
    ctx->resume_grid = static_cast<unsigned>(std::min<int>(bps * sms, AW_GRID_MAX));
  }
  return ctx->resume_grid;
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
  for (cached_graph* c : { &ctx->trim }) {
    if (c->exec) cudaGraphExecDestroy(c->exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    *c = {};
  }
}

namespace {

// Launches k_fwbw (pivot, or PIVOT_FROM_DEVICE; trim tail on or off) and
// queues the copies of its results into the pinned state mirror; the
// caller synchronises, then calls check_persistent.
void
launch_persistent(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t pivot, bool trim, kspn_options const& opt, kspn_stats* st, bool min_ids,
                  cudaEvent_t after_kernel = nullptr, bool ids_at_end = true, float const* model = nullptr)
{
  auto&       ws   = ctx->ws;
  auto* const rs   = reinterpret_cast<reach_state*>(ws.rstate);
  auto* const hs   = reinterpret_cast<reach_state*>(ctx->h_state);
  auto* const gbar = static_cast<grid_barrier*>(ws.gbar);
  bool const  tr   = opt.trace && st && st->search_marks == 0;
  fwbw_args   a{};
  a.n           = g.n;
  a.pivot       = pivot;
  a.m           = g.m;
  a.cap         = opt.max_levels ? opt.max_levels : g.n + 2;
  a.min_ids     = min_ids ? 1u : 0u;
  a.qbits       = bit_width64(g.n);
  a.trace       = tr ? 1u : 0u;
  a.alpha       = opt.bu_enter_div ? opt.bu_enter_div : 1;
  a.beta        = opt.bu_leave_div ? opt.bu_leave_div : 1;
  a.fh          = g.fh;
  a.fc          = g.fc;
  a.bh          = g.bh;
  a.bc          = g.bc;
  a.und         = und;
  a.scc_id      = scc_id;
  a.cand        = ws.mark;
  a.vis_a       = ws.vis_a;
  a.vis_b       = ws.vis_b;
  a.fresh       = ws.fresh;
  a.fresh_bw    = ws.fresh_bw;
  a.cand_bw     = ws.cand_bw;
  a.fb[0]       = { ws.q0, ws.prefix, ws.tile_start };
  a.fb[1]       = { ws.q1, ws.prefix2, ws.tile_start2 };
  a.fb_bw[0]    = { ws.q2, ws.prefix3, ws.tile_start3 };
  a.fb_bw[1]    = { ws.q3, ws.prefix4, ws.tile_start4 };
  a.seed        = { ws.seed_q, ws.seed_prefix, ws.tile_zero };
  a.partial     = ws.blocks;
  a.pv_prod     = ws.pivot + PV_FINAL;
  a.pv_id       = reinterpret_cast<uint32_t const*>(ws.pivot + 4096) + PV_FINAL;
  a.trim        = trim ? 1u : 0u;
  a.ids_at_end  = trim && ids_at_end ? 1u : 0u;
  a.aw          = static_cast<unsigned long long*>(ws.aw);
  a.aw_cap      = ws.aw_entries;
  a.aq          = reinterpret_cast<unsigned long long*>(static_cast<char*>(ws.gbar) + 1024);
  a.indeg       = ws.indeg;
  a.outdeg      = ws.outdeg;
  a.heavy       = ws.heavy;
  a.heavy_cap   = static_cast<uint32_t>(ws.heavy_cap);
  a.cutmap      = ws.cutmap;
  a.cut_words   = static_cast<uint32_t>((static_cast<size_t>(ws.n_cap) + 63) / 64 * 2 + 2);
  a.bar         = gbar;
  a.st          = rs;
  a.stamp_phase = reinterpret_cast<uint32_t*>(static_cast<char*>(ws.rstate) + 2048);
  a.stamp_ns    = reinterpret_cast<uint64_t*>(static_cast<char*>(ws.rstate) + 2048 + 4 * MARKS);
  a.wait_limit   = opt.wait_limit ? opt.wait_limit : GRID_SYNC_SPINS;
  a.drop_barrier = opt.drop_barrier;
  // an earlier switch only cuts duplicates; a later one could overrun the worklist's bound
  a.aw_exact     = opt.aw_exact_after && opt.aw_exact_after < ws.aw_entries / 2 ? opt.aw_exact_after : ws.aw_entries / 2;
  a.model        = model;
  a.jsave        = static_cast<char*>(ws.gbar) + 2048;
  a.resume       = 0;
  static_assert(sizeof(fwbw_args) <= sizeof(ctx->fwbw_last), "launch arguments must fit their copy in the context");
  static_assert(sizeof(joint_save) <= 2048, "saved level control must fit its workspace slot");
  std::memcpy(ctx->fwbw_last, &a, sizeof(a));
  ctx->fwbw_after = after_kernel;
  void* args[]    = { &a };
  barrier_for_grid(ctx, fwbw_grid(ctx));
  KSPN_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void const*>(&k_fwbw<4>), dim3(fwbw_grid(ctx)), dim3(R_THREADS), args, 0, ctx->stream));
  ctx->launches += 1;
  if (after_kernel) KSPN_CUDA(cudaEventRecord(after_kernel, ctx->stream));
  // results, and the barrier's error word (read after the launch ended: a
  // block that gave up may set it after block 0 finished)
  auto* const hb = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->h_state) + 1024);
  KSPN_CUDA(cudaMemcpyAsync(hs, rs, sizeof(reach_state), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaMemcpyAsync(hb, &gbar->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
}

// After the stream was synchronised: a launch that handed off its worklist
// phase is continued by the resume launch (same arguments, 128 registers
// per thread; one more host round trip, only on graphs that reach that
// phase); then barrier failures and level caps.  Returns whether a resume
// launch ran.
bool
check_persistent(kspn_context* ctx)
{
  auto* const hs = reinterpret_cast<reach_state*>(ctx->h_state);
  auto* const hb      = reinterpret_cast<uint32_t*>(static_cast<char*>(ctx->h_state) + 1024);
  bool const  resumed = hs->handoff && !*hb && !hs->bar_err;
  if (resumed) {
    fwbw_args a;
    std::memcpy(&a, ctx->fwbw_last, sizeof(a));
    a.resume     = 1;
    void* args[] = { &a };
    barrier_for_grid(ctx, resume_grid(ctx));
    KSPN_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void const*>(&k_fwbw<2>), dim3(resume_grid(ctx)), dim3(R_THREADS), args, 0, ctx->stream));
    ctx->launches += 1;
    if (ctx->fwbw_after) KSPN_CUDA(cudaEventRecord(ctx->fwbw_after, ctx->stream));
    KSPN_CUDA(cudaMemcpyAsync(hs, ctx->ws.rstate, sizeof(reach_state), cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaMemcpyAsync(hb, &static_cast<grid_barrier*>(ctx->ws.gbar)->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  if (*hb || hs->bar_err) {
    // counters of a launch that gave up are not epoch-aligned, and its
    // worklist may hold entries: start over
    KSPN_CUDA(cudaMemsetAsync(ctx->ws.gbar, 0, 4096, ctx->stream));
    KSPN_CUDA(cudaMemsetAsync(ctx->ws.aw, 0, ctx->ws.aw_entries * sizeof(unsigned long long), ctx->stream));
    KSPN_CUDA(cudaMemsetAsync(ctx->ws.cutmap, 0, 2 * ((static_cast<size_t>(ctx->ws.n_cap) + 63) / 64 * 2 + 2) * sizeof(uint32_t), ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    throw error{ KSPN_ERR_TIMEOUT, "reachability: grid barrier wait limit reached" };
  }
  if (hs->heavy_err) throw error{ KSPN_ERR_INTERNAL, "reachability / trim: heavy-row list overflow" };
  if (hs->err) throw error{ KSPN_ERR_TIMEOUT, "reachability / trim: level cap exceeded" };
  return resumed;
}

// Level statistics and phase stamps of the first FW-BW a call ran.
void
record_search_stats(kspn_context* ctx, kspn_options const& opt, kspn_stats* st)
{
  auto& ws = ctx->ws;
  auto* hs = reinterpret_cast<reach_state*>(ctx->h_state);
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
}

} // namespace

bool
resident_fits(dgraph const& g)
{
  return packed_counters_fit(g.n, g.m);
}

void
fw_bw_trim_async(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, kspn_options const& opt, kspn_stats* st, cudaEvent_t after_kernel)
{
  // with the learned rule the launch scores trim_1_first's pivot itself
  float const* model = opt.learned_pivot && ctx->pivot_model ? ctx->pivot_model : nullptr;
  launch_persistent(ctx, g, und, scc_id, static_cast<uint32_t>(PIVOT_FROM_DEVICE), true, opt, st, true, after_kernel, true, model);
}

resident_result
fw_bw_trim_result(kspn_context* ctx, dgraph const& g, kspn_options const& opt, kspn_stats* st)
{
  bool const resumed = check_persistent(ctx);
  auto* hs = reinterpret_cast<reach_state*>(ctx->h_state);
  record_search_stats(ctx, opt, st);
  ctx->h_ctr64[0] += hs->trim_edges;
  if (st) {
    // algorithmic DRAM traffic of the launch (the model kspn_stats
    // states): rows opened by bottom-up candidates, by top-down frontiers,
    // by the vertices pushed into scanned frontiers, and by the trim (both
    // rows of every listed and every queued vertex); neighbour ids read;
    // bitmap passes -- init (und read, three bitmaps written), two per
    // bitmap sweep (avail, fresh), one per frontier built from fresh,
    // a restriction of one search to the other's set (two read), finalize
    // (vis_a and vis_b read, und read + written, snap), ids (und, vis_b) --
    // and the ids written
    uint64_t const rows   = hs->cands_bu + hs->rows_td + hs->pushed_td + 2 * (hs->list_n + hs->trim_decided);
    uint64_t const edges  = hs->edges_td + hs->edges_bu + hs->trim_edges;
    uint32_t const passes = hs->pivot_used < g.n ? 4 + 2 * hs->bu_bitmap + hs->mats + 2 * hs->restricts + 5 + 2 : 1;
    st->resident_rows          = rows;
    st->resident_edges         = edges;
    st->resident_bitmap_passes = passes;
    st->resident_bytes         = 16 * rows + 4 * edges + passes * ((static_cast<uint64_t>(g.n) + 7) / 8) + 4ull * g.n;
    st->heavy_cut_rows         = hs->cut_n[0] + hs->cut_n[1];
    st->heavy_fixups           = hs->fixups;
    st->heavy_trim_seeds       = hs->hseed_n;
    st->trim_worklist          = hs->trim_async;
    st->fwbw_joint             = hs->joint;
    st->search_worklist        = hs->async_phases ? 1u : 0u;
  }
  resident_result r;
  r.resumed           = resumed;
  r.pivot_rejected    = hs->pivot_rejected != 0;
  r.pivot             = hs->pivot_used;
  r.fwbw_decided      = hs->decided;
  r.trim_decided      = hs->trim_decided;
  r.trim_levels       = hs->trim_levels;
  r.und_left          = hs->und_left;
  uint64_t const span = hs->t_ns[2] > hs->t_ns[0] ? hs->t_ns[2] - hs->t_ns[0] : 0;
  r.fwbw_share        = span ? static_cast<double>(hs->t_ns[1] - hs->t_ns[0]) / static_cast<double>(span) : 1.0;
  return r;
}

std::pair<uint32_t, uint32_t>
fw_bw_trim(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t pivot, kspn_options const& opt, kspn_stats* st)
{
  if (pivot >= g.n) throw error{ KSPN_ERR_INVALID_ARGUMENT, "fw_bw_trim: pivot >= n" };
  launch_persistent(ctx, g, und, scc_id, pivot, true, opt, st, true, nullptr, false);
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  check_persistent(ctx);
  auto* hs = reinterpret_cast<reach_state*>(ctx->h_state);
  record_search_stats(ctx, opt, st);
  ctx->h_ctr64[0] += hs->trim_edges;
  return { hs->decided, hs->trim_decided };
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

  uint32_t const words = (g.n + 31) / 32;
  if (!ctx->prof && packed_counters_fit(g.n, g.m)) {
    // the whole FW-BW on the device: one cooperative launch
    launch_persistent(ctx, g, und, scc_id, pivot, false, opt, st, min_ids);
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    check_persistent(ctx);
  } else {
    // host-driven loop over the same kernels, expansion kernels bracketed
    // by CUDA events (kspn_options.profile)
    bool const trace_done = st && st->levels_fw != 0; // trace the first FW-BW only
    KSPN_CUDA(cudaMemcpyAsync(rs, hs, sizeof(reach_state), cudaMemcpyHostToDevice, ctx->stream));
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
    if (hs->heavy_err) throw error{ KSPN_ERR_INTERNAL, "reachability: cut-row list overflow" };
    k_r_setid<<<1, 1, 0, ctx->stream>>>(rs);
    k_bitmap_min<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(g.n, ws.vis_b, rs);
    k_fwbw_finalize<<<r_grid(words), R_THREADS, 0, ctx->stream>>>(g.n, ws.vis_b, und, scc_id, rs);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 3;
    KSPN_CUDA(cudaMemcpyAsync(hs, rs, sizeof(reach_state), cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  }
  if (hs->err) throw error{ KSPN_ERR_TIMEOUT, "reachability: level cap exceeded" };
  record_search_stats(ctx, opt, st);
  return hs->decided;
}

} // namespace kspn
