// Batched path: thousands of independent small graphs of uneven size in one
// captured launch sequence (no reference counterpart: the reference
// decomposes one graph per call; each graph here gets the same partition
// its `scc` would, named by the smallest member).
//
// Layout (kspn_scc_batched): graph g owns vertices [vtx_off[g],
// vtx_off[g+1]) of one concatenated CSR and CSC whose heads hold global edge
// positions (head[vtx_off[g]] = edge_off[g]) and whose rows hold LOCAL ids
// (0 .. n_g - 1); scc_id[vtx_off[g] + v] = the local id of the smallest
// member of v's SCC.
//
// Plan (device, captured): per graph its size class -- a graph of at most
// RS_MAXV vertices and RS_MAXE edges is "small" -- and its bitmap word
// offset (each graph owns whole bitmap words); the large graphs sorted by
// n + m, largest first (a work queue in that order balances the tail).
// Solve (two kernels, independent nodes of the same CUDA graph, so they
// overlap):
//  * k_batch_small: one warp per small graph builds its CSR in shared
//    memory and runs the explicit-stack Tarjan of tarjan_smem.cuh;
//  * k_batch_group: one group per larger graph, claimed from a queue -- a
//    thread-block cluster (up to 8 blocks, distributed shared memory, the
//    cluster barrier) for graphs of n + m >= cluster_min, one block below:
//    init (degrees, in/out = 0 decided), then rounds of {trim-1 push
//    levels, FW-BW from the largest live in*out (SCC named by its smallest
//    member, its members seed the next trim)} until the remainder has at
//    most `rem_tarjan` vertices -- then Tarjan in shared memory -- or the
//    round cap is reached -- then one thread's Tarjan in global memory.
// Every loop is bounded; a round / level cap sets the error word.
#include "kspn_internal.cuh"
#include "prim.cuh"
#include "tarjan_smem.cuh"

#include <cooperative_groups.h>
#include <cstring>

namespace cg = cooperative_groups;

namespace kspn {

namespace {

constexpr int      BT_THREADS = 512;
constexpr int      BS_WARPS   = 4; // warps per block of k_batch_small
constexpr uint32_t BT_NONE    = 0xFFFFFFFFu;

struct bt_args
{
  uint32_t        G;
  uint64_t const* vtx_off;  // G + 1
  uint64_t const* word_off; // G + 1: bitmap words of graph g start at word_off[g]
  uint64_t const* fh;
  uint32_t const* fc;
  uint64_t const* bh;
  uint32_t const* bc;
  uint32_t*       scc_id;
  uint32_t*       und; // bitmaps, word_off-indexed
  uint32_t*       vis_a;
  uint32_t*       vis_b;
  uint32_t*       indeg; // N each, vtx_off-indexed
  uint32_t*       outdeg;
  uint32_t*       q0;
  uint32_t*       q1;
  uint32_t*       q2;
  uint64_t*       pos;   // N: serial Tarjan's edge cursors
  uint32_t const* order; // graphs sorted: large, medium, small; largest first inside a class
  uint32_t*       ctr;   // [0] large claimed, [1] small claimed, [2] n_large, [3] n_small, [4] err,
                         // [5] FW-BW rounds, [6] shared-memory Tarjans, [7] serial Tarjans, [8] trim levels,
                         // [9] n_medium, [10] medium claimed
  uint32_t        max_rounds; // FW-BW rounds per graph before the serial Tarjan
  uint32_t        rem_tarjan; // remainder size that goes to the shared-memory Tarjan (<= RS_MAXV)
  uint32_t        joint;      // FW and BW searches at the same time (bt_reach_joint)
};

__device__ __forceinline__ bool
bt_get(uint32_t const* bm, uint32_t v)
{
  return (__ldcg(bm + (v >> 5)) >> (v & 31)) & 1u;
}

// ---------------------------------------------------------------- plan
// Per graph: its class -- large (n + m >= cluster_min: a cluster), medium
// (a block), small (at most RS_MAXV vertices and RS_MAXE edges: a warp) --
// as the sort key's top bits, ~(n + m) below them (largest first inside a
// class), and its bitmap word count.  Class counts: ctr[2] large, ctr[9]
// medium, ctr[3] small.
__global__ void
k_bt_classify(uint32_t G, uint64_t const* __restrict__ vtx_off, uint64_t const* __restrict__ fh, uint64_t cluster_min, uint32_t* keys, uint32_t* vals, uint32_t* words, uint32_t* ctr)
{
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
    uint64_t const vo = vtx_off[g], n = vtx_off[g + 1] - vo;
    uint64_t const m  = fh[vo + n] - fh[vo];
    uint64_t const size  = n + m;
    uint32_t const cls   = n <= RS_MAXV && m <= RS_MAXE ? 2u : (size >= cluster_min ? 0u : 1u);
    keys[g]  = (cls << 30) | (0x3FFFFFFFu - static_cast<uint32_t>(size < 0x3FFFFFFFull ? size : 0x3FFFFFFFull));
    vals[g]  = g;
    words[g] = static_cast<uint32_t>((n + 31) / 32);
    atomicAdd(ctr + (cls == 0 ? 2 : cls == 1 ? 9 : 3), 1u);
  }
}

struct f_words
{
  uint32_t const* w;
  __device__ __forceinline__ uint64_t operator()(uint64_t i) const { return w[i]; }
};

// ---------------------------------------------------------------- small graphs
__global__ void __launch_bounds__(BS_WARPS * 32)
k_batch_small(bt_args a)
{
  extern __shared__ __align__(16) unsigned char bs_smem[];
  unsigned const lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
  rs_piece&      p    = reinterpret_cast<rs_piece*>(bs_smem)[wid];
  uint32_t const nb   = __ldcg(a.ctr + 2) + __ldcg(a.ctr + 9), ns = __ldcg(a.ctr + 3);
  for (;;) {
    uint32_t i = 0;
    if (lane == 0) i = atomicAdd(a.ctr + 1, 1u);
    i = __shfl_sync(0xFFFFFFFFu, i, 0);
    if (i >= ns) break;
    uint32_t const g  = a.order[nb + i];
    uint64_t const vo = a.vtx_off[g];
    uint32_t const n  = static_cast<uint32_t>(a.vtx_off[g + 1] - vo);
    uint64_t const e0 = a.fh[vo];
    // local CSR straight from the rows (ids are local already)
    for (uint32_t v = lane; v <= n; v += 32) p.off[v] = static_cast<uint16_t>(a.fh[vo + v] - e0);
    uint32_t const m = static_cast<uint32_t>(a.fh[vo + n] - e0);
    for (uint32_t e = lane; e < m; e += 32) p.adj[e] = static_cast<uint16_t>(a.fc[e0 + e]);
    for (uint32_t v = lane; v < n; v += 32) p.vid[v] = v;
    __syncwarp();
    if (lane == 0) rs_tarjan(p, n);
    __syncwarp();
    for (uint32_t v = lane; v < n; v += 32) a.scc_id[vo + v] = p.comp[v];
    __syncwarp();
  }
}

// ---------------------------------------------------------------- larger graphs
// A graph goes to a GROUP: one block (medium graphs) or a thread-block
// cluster of up to 8 blocks on different SMs (large graphs).  The group's
// counters live in the shared memory of its rank-0 block and the others
// reach them as distributed shared memory; group barriers are the
// hardware cluster barrier (release / acquire at cluster scope); data other
// blocks of the group write is read through L2.
struct bt_smem
{
  uint32_t           g, rem, cnt, minid, lo, hi, flag, pad;
  uint32_t           lo2, hi2, cnt2, pad2;
  unsigned long long best;
};

struct bt_group
{
  cg::cluster_group cl;
  bt_smem*          S;   // rank 0's counters (local or distributed shared memory)
  uint32_t          gt;  // thread index in the group
  uint32_t          GT;  // threads in the group
  bool              one; // a single block: block barriers suffice
  __device__ __forceinline__ void sync() const
  {
    if (one) __syncthreads();
    else cl.sync();
  }
  __device__ __forceinline__ bool leader() const { return gt == 0; }
};

// warp-aggregated slot from a group counter (lanes that may be inactive)
__device__ __forceinline__ uint32_t
bt_slot(uint32_t* counter)
{
  unsigned const mask = __activemask();
  unsigned const lane = threadIdx.x & 31u, leader = __ffs(mask) - 1;
  uint32_t       base = 0;
  if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(mask)));
  base = __shfl_sync(mask, base, leader);
  return base + __popc(mask & ((1u << lane) - 1u));
}

// fn(u, e) for every edge e of every row of list[lo, hi): a warp takes 32
// listed vertices at a time and its lanes split their edges evenly (a
// warp-wide scan of the row lengths; each lane finds its row by a binary
// search over the lanes' exclusive prefixes), so 32 independent loads are
// in flight per instruction instead of one dependent row walk per thread.
// All lanes of every warp of the group call it; fn is called by the active
// lanes only.
template<class F>
__device__ __forceinline__ void
bt_warp_edges(bt_group const& g, uint32_t const* list, uint32_t lo, uint32_t hi, uint64_t const* head, F&& fn)
{
  unsigned const lane = threadIdx.x & 31u;
  uint32_t const gw = g.gt >> 5, GW = g.GT >> 5;
  for (uint32_t base = lo + gw * 32; base < hi; base += GW * 32) {
    uint32_t const i  = base + lane;
    bool const     ok = i < hi;
    uint32_t const u  = ok ? __ldcg(list + i) : 0u;
    uint64_t const b  = ok ? head[u] : 0;
    uint32_t const d  = ok ? static_cast<uint32_t>(head[u + 1] - b) : 0u;
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
      uint64_t const bj = __shfl_sync(0xFFFFFFFFu, b, j);
      uint32_t const xj = __shfl_sync(0xFFFFFFFFu, excl, j);
      uint32_t const uj = __shfl_sync(0xFFFFFFFFu, u, j);
      if (k < total) fn(uj, bj + (k - xj));
    }
  }
}

// Group-leader clock of the phases of the larger graphs (init, trim,
// pivot, searches, remainder): %globaltimer deltas summed over all groups
// into the u64 counters after the u32 ones.
__device__ __forceinline__ uint64_t
bt_now()
{
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void
bt_phase(bt_args const& a, bt_group const& g, int k, uint64_t& t)
{
  if (!g.leader()) return;
  uint64_t const now = bt_now();
  atomicAdd(reinterpret_cast<unsigned long long*>(a.ctr + 32) + k, static_cast<unsigned long long>(now - t));
  t = now;
}

// One graph's view for the group.
struct bt_graph
{
  uint64_t        vo;
  uint32_t        n, words;
  uint64_t const* fh; // rows of local v: fc[fh[v] .. fh[v+1])
  uint64_t const* bh;
  uint32_t*       und;
  uint32_t*       va;
  uint32_t*       vb;
  uint32_t*       indeg;
  uint32_t*       outdeg;
  uint32_t*       ids;
  uint32_t*       q0;
  uint32_t*       q1;
  uint32_t*       q2;
};

// Trim-1 push levels from qin[0, qn): every queued (just decided) vertex
// lowers its undecided out-neighbours' live in-degree and in-neighbours'
// live out-degree; a count reaching 0 decides that neighbour (id = itself)
// and queues it.  Queues alternate between the two buffers that are not
// qin; rows are walked warp-cooperatively (bt_warp_edges).  Returns the
// vertices decided.
__device__ uint32_t
bt_trim(bt_args const& a, bt_graph const& G, bt_group const& g, uint32_t* qin, uint32_t qn)
{
  uint32_t  total = 0;
  uint32_t* bufs[2];
  if (qin == G.q0) bufs[0] = G.q1, bufs[1] = G.q2;
  else if (qin == G.q1) bufs[0] = G.q0, bufs[1] = G.q2;
  else bufs[0] = G.q0, bufs[1] = G.q1;
  uint32_t levels = 0;
  for (uint32_t lvl = 0; qn > 0; ++lvl) {
    if (lvl > G.n + 1) {
      if (g.leader()) atomicExch(a.ctr + 4, 1u);
      break;
    }
    uint32_t* const qout = bufs[lvl & 1];
    if (g.leader()) g.S->cnt = 0;
    g.sync();
    auto const hit = [&](uint32_t w, uint32_t* deg) {
      if (bt_get(G.und, w) && atomicSub(deg + w, 1u) == 1u && bit_take(G.und, w)) {
        G.ids[w]                 = w;
        qout[bt_slot(&g.S->cnt)] = w;
      }
    };
#pragma unroll 1
    for (int dir = 0; dir < 2; ++dir) {
      uint32_t const* adj = dir ? a.bc : a.fc;
      uint32_t*       deg = dir ? G.outdeg : G.indeg;
      bt_warp_edges(g, qin, 0, qn, dir ? G.bh : G.fh, [&](uint32_t, uint64_t e) { hit(adj[e], deg); });
    }
    g.sync();
    qn = g.S->cnt;
    total += qn;
    qin = qout;
    ++levels;
    g.sync();
  }
  if (g.leader() && levels) atomicAdd(a.ctr + 8, levels);
  return total;
}

// Level-synchronous reach from `root` over head/adj rows, among vertices
// whose bit is set in `cand` (nullptr: among undecided vertices, n_und of
// them), claiming bits of `mark`; every reached vertex is appended to
// `list`.  Returns how many were reached.
// A level whose frontier holds more than 1/BT_BU_DIV of the undecided
// vertices runs bottom-up: every unreached candidate walks its
// opposite-direction row (bu_head / bu_adj) until a neighbour in `mark`
// (reached so far, this level's finds included: reachability does not
// need BFS levels), and joins.
constexpr int      BT_BU_ILP = 2; // candidates a thread walks side by side in a bottom-up level
constexpr uint32_t BT_BU_DIV = 5; // measured on C5: 1/2 23.1 ms, 1/3 19.2, 1/4 17.7, 1/6 17.7, 1/16 19.6, none 23.3

__device__ uint32_t
bt_reach(bt_args const& a, bt_graph const& G, bt_group const& g, uint64_t const* head, uint32_t const* adj, uint64_t const* bu_head, uint32_t const* bu_adj, uint32_t const* cand,
         uint32_t* mark, uint32_t* list, uint32_t root, uint32_t n_und)
{
  if (g.leader()) {
    list[0] = root;
    atomicOr(mark + (root >> 5), 1u << (root & 31));
    g.S->lo  = 0;
    g.S->hi  = 1;
    g.S->cnt = 1;
  }
  g.sync();
  for (uint32_t lvl = 0;; ++lvl) {
    uint32_t const lo = g.S->lo, hi = g.S->hi;
    if (lo == hi) break;
    if (lvl > G.n + 1) {
      if (g.leader()) atomicExch(a.ctr + 4, 1u);
      break;
    }
    if (static_cast<uint64_t>(hi - lo) * BT_BU_DIV > n_und) {
      // a thread walks up to BT_BU_ILP candidates of its word side by side
      // (their offset loads, then their neighbour loads, then their probes
      // in flight together) instead of one dependent row walk at a time
      for (uint32_t wd = g.gt; wd < G.words; wd += g.GT) {
        uint32_t cw = (cand ? __ldcg(cand + wd) : __ldcg(G.und + wd)) & ~__ldcg(mark + wd);
        while (cw) {
          uint32_t v[BT_BU_ILP];
          uint64_t b[BT_BU_ILP], e[BT_BU_ILP];
#pragma unroll
          for (int k = 0; k < BT_BU_ILP; ++k) {
            v[k] = UNDECIDED;
            b[k] = e[k] = 0;
            if (cw) {
              v[k] = wd * 32 + __ffs(cw) - 1;
              cw &= cw - 1;
            }
          }
#pragma unroll
          for (int k = 0; k < BT_BU_ILP; ++k)
            if (v[k] != UNDECIDED) b[k] = bu_head[v[k]], e[k] = bu_head[v[k] + 1];
          for (bool more = true; more;) {
            uint32_t x[BT_BU_ILP];
#pragma unroll
            for (int k = 0; k < BT_BU_ILP; ++k) x[k] = b[k] < e[k] ? bu_adj[b[k]] : 0u;
            more = false;
#pragma unroll
            for (int k = 0; k < BT_BU_ILP; ++k) {
              if (b[k] >= e[k]) continue;
              if (bt_get(mark, x[k])) {
                if (bit_claim(mark, v[k])) list[bt_slot(&g.S->cnt)] = v[k];
                e[k] = b[k]; // done
              } else if (++b[k] < e[k])
                more = true;
            }
          }
        }
      }
    } else
      bt_warp_edges(g, list, lo, hi, head, [&](uint32_t, uint64_t e) {
        uint32_t const w = adj[e];
        if ((cand ? bt_get(cand, w) : bt_get(G.und, w)) && bit_claim(mark, w)) list[bt_slot(&g.S->cnt)] = w;
      });
    g.sync();
    if (g.leader()) g.S->lo = hi, g.S->hi = g.S->cnt;
    g.sync();
  }
  uint32_t const c = g.S->cnt;
  g.sync();
  return c;
}

// FW and BW reach from `root` at the same time, both among the undecided
// vertices (FW over out-rows claiming vis_a into q1, BW over in-rows
// claiming vis_b into q2), one group barrier per joint level: the SCC is
// their intersection.  Half the levels of FW then BW on a graph's
// critical path, for BW also walking vertices outside the FW set.
// Returns (FW count, BW count).
__device__ uint2
bt_reach_joint(bt_args const& a, bt_graph const& G, bt_group const& g, uint32_t root)
{
  if (g.leader()) {
    G.q1[0] = G.q2[0] = root;
    atomicOr(G.va + (root >> 5), 1u << (root & 31));
    atomicOr(G.vb + (root >> 5), 1u << (root & 31));
    g.S->lo = g.S->lo2 = 0;
    g.S->hi = g.S->hi2 = 1;
    g.S->cnt = g.S->cnt2 = 1;
  }
  g.sync();
  for (uint32_t lvl = 0;; ++lvl) {
    uint32_t const lo = g.S->lo, hi = g.S->hi, lo2 = g.S->lo2, hi2 = g.S->hi2;
    if (lo == hi && lo2 == hi2) break;
    if (lvl > G.n + 1) {
      if (g.leader()) atomicExch(a.ctr + 4, 1u);
      break;
    }
    bt_warp_edges(g, G.q1, lo, hi, G.fh, [&](uint32_t, uint64_t e) {
      uint32_t const w = a.fc[e];
      if (bt_get(G.und, w) && bit_claim(G.va, w)) G.q1[bt_slot(&g.S->cnt)] = w;
    });
    bt_warp_edges(g, G.q2, lo2, hi2, G.bh, [&](uint32_t, uint64_t e) {
      uint32_t const w = a.bc[e];
      if (bt_get(G.und, w) && bit_claim(G.vb, w)) G.q2[bt_slot(&g.S->cnt2)] = w;
    });
    g.sync();
    if (g.leader()) g.S->lo = hi, g.S->hi = g.S->cnt, g.S->lo2 = hi2, g.S->hi2 = g.S->cnt2;
    g.sync();
  }
  uint2 const c = make_uint2(g.S->cnt, g.S->cnt2);
  g.sync();
  return c;
}

// argmax over undecided v of live in * out (lowest id on ties), as
// (saturated prod << 32 | ~id); BT_NONE when nothing is undecided
__device__ uint32_t
bt_pivot(bt_graph const& G, bt_group const& g)
{
  if (g.leader()) g.S->best = 0;
  g.sync();
  unsigned long long best = 0;
  for (uint32_t v = g.gt; v < G.n; v += g.GT) {
    if (!bt_get(G.und, v)) continue;
    uint64_t const           p   = static_cast<uint64_t>(__ldcg(G.indeg + v)) * __ldcg(G.outdeg + v);
    unsigned long long const key = (static_cast<unsigned long long>(p < 0xFFFFFFFFull ? p : 0xFFFFFFFFull) << 32) | (0xFFFFFFFFu - v);
    best                         = key > best ? key : best;
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) {
    unsigned long long const o = __shfl_xor_sync(0xFFFFFFFFu, best, sh);
    best                       = o > best ? o : best;
  }
  if ((threadIdx.x & 31) == 0 && best) atomicMax(&g.S->best, best);
  g.sync();
  unsigned long long const b = g.S->best;
  g.sync();
  return b ? 0xFFFFFFFFu - static_cast<uint32_t>(b & 0xFFFFFFFFu) : BT_NONE;
}

// The remaining (undecided) vertices of a graph in id order into the
// piece (rank 0's warp 0), if there are at most RS_MAXV of them with at
// most RS_MAXE edges among them; then Tarjan and the ids.  Returns false
// (and changes nothing) when they do not fit.
__device__ bool
bt_tarjan_smem(bt_args const& a, bt_graph const& G, bt_group const& g, rs_piece& p)
{
  unsigned const lane = threadIdx.x & 31u;
  if (g.gt < 32) {
    uint32_t k = 0;
    for (uint32_t wb = 0; wb < G.words; wb += 32) {
      uint32_t const w    = wb + lane;
      uint32_t       word = w < G.words ? __ldcg(G.und + w) : 0u;
      uint32_t const c    = __popc(word);
      uint32_t       incl = c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= static_cast<unsigned>(d)) incl += y;
      }
      uint32_t j = k + incl - c;
      for (; word; word &= word - 1, ++j)
        if (j < RS_MAXV) p.vid[j] = w * 32 + __ffs(word) - 1;
      k += __shfl_sync(0xFFFFFFFFu, incl, 31);
      if (k > RS_MAXV) break;
    }
    __syncwarp();
    bool           fits = k <= RS_MAXV;
    uint32_t const per  = (k + 31) / 32;
    uint32_t       cnt  = 0;
    if (fits)
      for (uint32_t i = lane * per; i < k && i < lane * per + per; ++i) {
        uint32_t const v = p.vid[i];
        uint32_t       c = 0;
        for (uint64_t e = G.fh[v], end = G.fh[v + 1]; e < end; ++e) c += bt_get(G.und, a.fc[e]) ? 1u : 0u;
        p.comp[i] = static_cast<uint16_t>(c < RS_MAXE ? c : RS_MAXE);
        cnt += c;
      }
    uint32_t incl = cnt;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, incl, d);
      if (lane >= static_cast<unsigned>(d)) incl += y;
    }
    uint32_t const total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    fits                 = fits && total <= RS_MAXE;
    if (fits) {
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
        for (uint64_t e = G.fh[v], end = G.fh[v + 1]; e < end; ++e) {
          uint32_t const w = a.fc[e];
          if (bt_get(G.und, w)) p.adj[o++] = static_cast<uint16_t>(rs_local(p, k, w));
        }
      }
      __syncwarp();
      if (lane == 0) rs_tarjan(p, k);
      __syncwarp();
      for (uint32_t i = lane; i < k; i += 32) {
        uint32_t const v = p.vid[i];
        G.ids[v]         = p.vid[p.comp[i]];
        atomicAnd(G.und + (v >> 5), ~(1u << (v & 31)));
      }
      if (lane == 0) atomicAdd(a.ctr + 6, 1u);
    }
    if (lane == 0) g.S->flag = fits ? 1u : 0u;
  }
  g.sync();
  bool const ok = g.S->flag != 0;
  g.sync();
  return ok;
}

// One thread's iterative Tarjan (tarjan.hpp:20-136) over the undecided
// sub-graph in global memory: index in indeg, low in outdeg, the SCC stack
// in q0, the call stack's vertices in q1 and edge cursors in pos; on-stack
// flags in vis_a.  The last resort after the round cap; n + m steps.
__device__ void
bt_tarjan_serial(bt_args const& a, bt_graph const& G, bt_group const& g, uint64_t* pos)
{
  g.sync();
  for (uint32_t v = g.gt; v < G.n; v += g.GT) G.indeg[v] = BT_NONE;
  for (uint32_t w = g.gt; w < G.words; w += g.GT) G.va[w] = 0;
  g.sync();
  if (g.leader()) {
    atomicAdd(a.ctr + 7, 1u);
    uint32_t idx = 0, sp = 0, cp = 0;
    for (uint32_t r = 0; r < G.n; ++r) {
      if (!bt_get(G.und, r) || __ldcg(G.indeg + r) != BT_NONE) continue;
      G.indeg[r] = G.outdeg[r] = idx++;
      G.q0[sp++]               = r;
      G.va[r >> 5] |= 1u << (r & 31);
      G.q1[cp]  = r;
      pos[cp++] = G.fh[r];
      while (cp > 0) {
        uint32_t const v = G.q1[cp - 1];
        uint64_t const e = pos[cp - 1];
        if (e < G.fh[v + 1]) {
          pos[cp - 1]      = e + 1;
          uint32_t const w = a.fc[e];
          if (!bt_get(G.und, w)) continue;
          if (G.indeg[w] == BT_NONE) {
            G.indeg[w] = G.outdeg[w] = idx++;
            G.q0[sp++]               = w;
            G.va[w >> 5] |= 1u << (w & 31);
            G.q1[cp]  = w;
            pos[cp++] = G.fh[w];
          } else if (((G.va[w >> 5] >> (w & 31)) & 1u) && G.indeg[w] < G.outdeg[v]) G.outdeg[v] = G.indeg[w];
        } else {
          --cp;
          if (cp > 0) {
            uint32_t const u = G.q1[cp - 1];
            if (G.outdeg[v] < G.outdeg[u]) G.outdeg[u] = G.outdeg[v];
          }
          if (G.outdeg[v] == G.indeg[v]) {
            uint32_t j = sp, mn = v;
            do {
              --j;
              if (G.q0[j] < mn) mn = G.q0[j];
            } while (G.q0[j] != v);
            for (uint32_t t = j; t < sp; ++t) {
              uint32_t const x = G.q0[t];
              G.va[x >> 5] &= ~(1u << (x & 31));
              G.ids[x] = mn;
              G.und[x >> 5] &= ~(1u << (x & 31));
            }
            sp = j;
          }
        }
      }
    }
  }
  g.sync();
}

__device__ void
bt_solve(bt_args const& a, uint32_t gi, bt_group const& g, rs_piece& piece)
{
  bt_graph G;
  G.vo     = a.vtx_off[gi];
  G.n      = static_cast<uint32_t>(a.vtx_off[gi + 1] - G.vo);
  G.words  = (G.n + 31) / 32;
  G.fh     = a.fh + G.vo;
  G.bh     = a.bh + G.vo;
  G.und    = a.und + a.word_off[gi];
  G.va     = a.vis_a + a.word_off[gi];
  G.vb     = a.vis_b + a.word_off[gi];
  G.indeg  = a.indeg + G.vo;
  G.outdeg = a.outdeg + G.vo;
  G.ids    = a.scc_id + G.vo;
  G.q0     = a.q0 + G.vo;
  G.q1     = a.q1 + G.vo;
  G.q2     = a.q2 + G.vo;
  uint64_t* const pos = a.pos + G.vo;

  uint64_t t = g.leader() ? bt_now() : 0;
  // init: all undecided, live degrees = raw degrees, in/out = 0 decided
  for (uint32_t w = g.gt; w < G.words; w += g.GT) {
    uint32_t const tail = G.n - w * 32;
    G.und[w]            = tail >= 32 ? 0xFFFFFFFFu : (1u << tail) - 1u;
    G.va[w] = G.vb[w] = 0;
  }
  if (g.leader()) g.S->cnt = 0;
  g.sync();
  for (uint32_t v = g.gt; v < G.n; v += g.GT) {
    uint32_t const o = static_cast<uint32_t>(G.fh[v + 1] - G.fh[v]);
    uint32_t const i = static_cast<uint32_t>(G.bh[v + 1] - G.bh[v]);
    G.outdeg[v]      = o;
    G.indeg[v]       = i;
    if (o == 0 || i == 0) {
      G.ids[v] = v;
      atomicAnd(G.und + (v >> 5), ~(1u << (v & 31)));
      G.q0[bt_slot(&g.S->cnt)] = v;
    } else G.ids[v] = UNDECIDED;
  }
  g.sync();
  uint32_t  qn   = g.S->cnt;
  uint32_t  rem  = G.n - qn;
  uint32_t* seed = G.q0;
  g.sync();
  bt_phase(a, g, 0, t);
  for (uint32_t round = 0;; ++round) {
    rem -= bt_trim(a, G, g, seed, qn);
    bt_phase(a, g, 1, t);
    if (rem == 0) break;
    if (rem <= a.rem_tarjan && bt_tarjan_smem(a, G, g, piece)) {
      bt_phase(a, g, 4, t);
      break;
    }
    if (round >= a.max_rounds) {
      bt_tarjan_serial(a, G, g, pos);
      bt_phase(a, g, 4, t);
      break;
    }
    // FW-BW from the largest live in * out
    uint32_t const p = bt_pivot(G, g);
    bt_phase(a, g, 2, t);
    if (p == BT_NONE) {
      if (g.leader()) atomicExch(a.ctr + 4, 1u);
      break;
    }
    uint32_t nf, nb;
    uint32_t* scc = G.q2; // the SCC's members
    if (a.joint) {
      uint2 const c = bt_reach_joint(a, G, g, p);
      nf            = c.x;
      // members: BW-reached vertices also FW-reached, compacted into q0
      if (g.leader()) g.S->cnt = 0;
      g.sync();
      for (uint32_t i = g.gt; i < c.y; i += g.GT) {
        uint32_t const v = __ldcg(G.q2 + i);
        if (bt_get(G.va, v)) G.q0[bt_slot(&g.S->cnt)] = v;
        atomicAnd(G.vb + (v >> 5), ~(1u << (v & 31))); // vis_b cleared through its own list
      }
      g.sync();
      nb  = g.S->cnt;
      scc = G.q0;
      g.sync();
    } else {
      nf = bt_reach(a, G, g, G.fh, a.fc, G.bh, a.bc, nullptr, G.va, G.q1, p, rem);
      nb = bt_reach(a, G, g, G.bh, a.bc, G.fh, a.fc, G.va, G.vb, G.q2, p, nf);
    }
    // the SCC: smallest member, ids, und; vis_a cleared through q1
    if (g.leader()) g.S->minid = 0xFFFFFFFFu;
    g.sync();
    uint32_t mn = 0xFFFFFFFFu;
    for (uint32_t i = g.gt; i < nb; i += g.GT) mn = min(mn, __ldcg(scc + i));
    mn = __reduce_min_sync(0xFFFFFFFFu, mn);
    if ((threadIdx.x & 31) == 0 && mn != 0xFFFFFFFFu) atomicMin(&g.S->minid, mn);
    g.sync();
    uint32_t const id = g.S->minid;
    for (uint32_t i = g.gt; i < nb; i += g.GT) {
      uint32_t const v = __ldcg(scc + i);
      G.ids[v]         = id;
      atomicAnd(G.und + (v >> 5), ~(1u << (v & 31)));
      atomicAnd(G.vb + (v >> 5), ~(1u << (v & 31)));
    }
    for (uint32_t i = g.gt; i < nf; i += g.GT) {
      uint32_t const v = __ldcg(G.q1 + i);
      atomicAnd(G.va + (v >> 5), ~(1u << (v & 31)));
    }
    if (g.leader()) atomicAdd(a.ctr + 5, 1u);
    g.sync();
    bt_phase(a, g, 3, t);
    rem -= nb;
    if (rem == 0) break;
    // the SCC's members seed the next trim
    seed = scc;
    qn   = nb;
  }
  g.sync();
}

// Persistent groups over one queue of graphs (a.order[first, first + *count)),
// claimed through *claim.  Launched with a cluster dimension (or none: a
// group of one block).
__global__ void __launch_bounds__(BT_THREADS, 3) // 3 blocks per SM: the path is latency-bound, graphs in flight count most
k_batch_group(bt_args a, uint32_t first_slot, uint32_t count_slot, uint32_t claim_slot)
{
  extern __shared__ __align__(16) unsigned char bt_dyn[];
  rs_piece&          piece = *reinterpret_cast<rs_piece*>(bt_dyn);
  __shared__ bt_smem s;
  bt_group           g{ cg::this_cluster(), nullptr, 0, 0, false };
  uint32_t const     csize = g.cl.num_blocks();
  g.one                    = csize == 1;
  g.S                      = g.one ? &s : g.cl.map_shared_rank(&s, 0);
  g.gt                     = g.cl.block_rank() * BT_THREADS + threadIdx.x;
  g.GT                     = csize * BT_THREADS;
  uint32_t const first     = first_slot == BT_NONE ? 0u : __ldcg(a.ctr + first_slot);
  uint32_t const count     = __ldcg(a.ctr + count_slot);
  g.sync(); // every block of the cluster has started (its shared memory exists)
  for (;;) {
    if (g.leader()) g.S->g = atomicAdd(a.ctr + claim_slot, 1u);
    g.sync();
    uint32_t const i = g.S->g;
    g.sync();
    if (i >= count) break;
    bt_solve(a, a.order[first + i], g, piece);
  }
  g.sync(); // no block leaves while another may still reach its shared memory
}

} // namespace

// ---------------------------------------------------------------- host
namespace {

struct batch_plan
{
  void*     base = nullptr; // one allocation: keys, vals, alt, words, word_off, hist, partials
  size_t    bytes = 0;
  uint32_t* keys = nullptr;
  uint32_t* order = nullptr;
  uint32_t* kalt = nullptr;
  uint32_t* valt = nullptr;
  uint32_t* words = nullptr;
  uint64_t* word_off = nullptr;
  uint32_t* hist = nullptr;
  uint32_t* part = nullptr;
  uint64_t* part64 = nullptr;
  uint32_t* und = nullptr;
  uint32_t* vis_a = nullptr;
  uint32_t* vis_b = nullptr;
  uint32_t* indeg = nullptr;
  uint32_t* outdeg = nullptr;
  uint32_t* q0 = nullptr;
  uint32_t* q1 = nullptr;
  uint32_t* q2 = nullptr;
  uint64_t* pos = nullptr;
  uint32_t* ctr = nullptr; // 32 words
};

} // namespace

struct batch_cache
{
  batch_plan      plan;
  cudaGraph_t     graph = nullptr;
  cudaGraphExec_t exec  = nullptr;
  void const*     key[6] = {};
  uint32_t        G = 0;
  uint64_t        N = 0;
  uint32_t        max_rounds = 0, rem_tarjan = 0, block_blocks = 0, cluster_size = 0, cluster_blocks = 0;
  uint64_t        cluster_min = 0;
  uint32_t        joint       = 0;
  cudaStream_t    cap_stream = nullptr;
};

void
batch_release(kspn_context* ctx)
{
  batch_cache* c = ctx->batch;
  if (!c) return;
  if (c->exec) cudaGraphExecDestroy(c->exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  if (c->plan.base) cudaFree(c->plan.base);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  delete c;
  ctx->batch = nullptr;
}

namespace {

void
carve_plan(batch_plan& p, char* base, uint32_t G, uint64_t N, size_t* bytes_out)
{
  size_t off  = 0;
  auto   take = [&](size_t bytes) {
    off           = (off + 255) & ~size_t(255);
    char* const q = base ? base + off : nullptr;
    off += bytes;
    return q;
  };
  size_t const hist_n = radix_hist_entries(G);
  size_t const part_n = scan_partial_entries(hist_n > G + 1 ? hist_n : G + 1);
  size_t const words  = N / 32 + G + 2; // every graph rounds up to whole words
  p.keys     = reinterpret_cast<uint32_t*>(take(4 * (G + 1)));
  p.order    = reinterpret_cast<uint32_t*>(take(4 * (G + 1)));
  p.kalt     = reinterpret_cast<uint32_t*>(take(4 * (G + 1)));
  p.valt     = reinterpret_cast<uint32_t*>(take(4 * (G + 1)));
  p.words    = reinterpret_cast<uint32_t*>(take(4 * (G + 1)));
  p.word_off = reinterpret_cast<uint64_t*>(take(8 * (G + 1)));
  p.hist     = reinterpret_cast<uint32_t*>(take(4 * hist_n));
  p.part     = reinterpret_cast<uint32_t*>(take(4 * part_n));
  p.part64   = reinterpret_cast<uint64_t*>(take(8 * part_n));
  p.und      = reinterpret_cast<uint32_t*>(take(4 * words));
  p.vis_a    = reinterpret_cast<uint32_t*>(take(4 * words));
  p.vis_b    = reinterpret_cast<uint32_t*>(take(4 * words));
  p.indeg    = reinterpret_cast<uint32_t*>(take(4 * (N + 1)));
  p.outdeg   = reinterpret_cast<uint32_t*>(take(4 * (N + 1)));
  p.q0       = reinterpret_cast<uint32_t*>(take(4 * (N + 1)));
  p.q1       = reinterpret_cast<uint32_t*>(take(4 * (N + 1)));
  p.q2       = reinterpret_cast<uint32_t*>(take(4 * (N + 1)));
  p.pos      = reinterpret_cast<uint64_t*>(take(8 * (N + 1)));
  p.ctr      = reinterpret_cast<uint32_t*>(take(4 * 64)); // [32..64): u64 phase times (bt_phase)
  *bytes_out = (off + 255) & ~size_t(255);
}

// The whole call as stream work (captured once per batch and settings).
void
enqueue_batch(kspn_context* ctx, batch_cache& c, bt_args const& a0)
{
  cudaStream_t const s = ctx->stream;
  batch_plan&        p = c.plan;
  uint32_t const     G = c.G;
  KSPN_CUDA(cudaMemsetAsync(p.ctr, 0, 64 * sizeof(uint32_t), s));
  unsigned const cgrid = div_up(G, 256);
  k_bt_classify<<<cgrid < 1 ? 1 : cgrid, 256, 0, s>>>(G, a0.vtx_off, a0.fh, c.cluster_min, p.keys, p.order, p.words, p.ctr);
  KSPN_CHECK_LAUNCH();
  exclusive_scan<uint64_t>(s, f_words{ p.words }, G, p.word_off, p.part64, nullptr);
  radix_sort_pairs(ctx, p.keys, p.order, p.kalt, p.valt, G, 0, 32, p.hist, p.part);
  bt_args a    = a0;
  a.word_off   = p.word_off;
  a.und        = p.und;
  a.vis_a      = p.vis_a;
  a.vis_b      = p.vis_b;
  a.indeg      = p.indeg;
  a.outdeg     = p.outdeg;
  a.q0         = p.q0;
  a.q1         = p.q1;
  a.q2         = p.q2;
  a.pos        = p.pos;
  a.order      = p.order;
  a.ctr        = p.ctr;
  a.max_rounds = c.max_rounds;
  a.rem_tarjan = c.rem_tarjan;
  a.joint      = c.joint;
  // large graphs: clusters of c.cluster_size blocks; medium: single blocks
  if (c.cluster_size > 1) {
    cudaLaunchConfig_t   cfg{};
    cudaLaunchAttribute  attr[1];
    attr[0].id               = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = c.cluster_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim              = dim3(c.cluster_blocks);
    cfg.blockDim             = dim3(BT_THREADS);
    cfg.dynamicSmemBytes     = sizeof(rs_piece);
    cfg.stream               = s;
    cfg.attrs                = attr;
    cfg.numAttrs             = 1;
    KSPN_CUDA(cudaLaunchKernelEx(&cfg, k_batch_group, a, BT_NONE, 2u, 0u));
  } else k_batch_group<<<c.block_blocks, BT_THREADS, sizeof(rs_piece), s>>>(a, BT_NONE, 2u, 0u);
  k_batch_group<<<c.block_blocks, BT_THREADS, sizeof(rs_piece), s>>>(a, 2u, 9u, 10u);
  k_batch_small<<<148 * 4, BS_WARPS * 32, BS_WARPS * sizeof(rs_piece), s>>>(a);
  KSPN_CHECK_LAUNCH();
}

} // namespace

void
scc_batched(kspn_context* ctx, uint32_t G, uint64_t N, uint64_t const* vtx_off, uint64_t const* fh, uint32_t const* fc, uint64_t const* bh, uint32_t const* bc, uint32_t* scc_id,
            kspn_batch_options const& opt, kspn_batch_stats* st)
{
  if (G == 0) return;
  uint32_t const rem = opt.rem_tarjan ? opt.rem_tarjan : RS_MAXV;
  if (rem > RS_MAXV) throw error{ KSPN_ERR_INVALID_ARGUMENT, "scc_batched: rem_tarjan > 512" };
  uint32_t const rounds = opt.max_rounds ? opt.max_rounds : 64;
  uint32_t const csize  = opt.cluster_size ? opt.cluster_size : 1;
  uint64_t const cmin   = csize == 1 ? ~0ull : (opt.cluster_min ? opt.cluster_min : (1ull << 16));
  if (csize > 8) throw error{ KSPN_ERR_INVALID_ARGUMENT, "scc_batched: cluster_size > 8" };
  uint32_t const joint = opt.search == 1 ? 1u : 0u; // 1: joint searches; 0 (default), 2: FW then BW
  batch_cache*&  cp     = ctx->batch;
  if (!cp) cp = new batch_cache{};
  batch_cache&      c   = *cp;
  void const* const key[6] = { vtx_off, fh, fc, bh, bc, scc_id };
  bool              same   = c.exec && c.G == G && c.N == N && c.max_rounds == rounds && c.rem_tarjan == rem && c.cluster_size == csize && c.cluster_min == cmin && c.joint == joint;
  for (int i = 0; i < 6 && same; ++i) same = c.key[i] == key[i];
  if (!same) {
    if (c.exec) cudaGraphExecDestroy(c.exec), c.exec = nullptr;
    if (c.graph) cudaGraphDestroy(c.graph), c.graph = nullptr;
    size_t bytes = 0;
    carve_plan(c.plan, nullptr, G, N, &bytes);
    if (bytes > c.plan.bytes) {
      if (c.plan.base) {
        KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
        cudaFree(c.plan.base);
        c.plan = {};
      }
      void* b = nullptr;
      if (cudaMalloc(&b, bytes) != cudaSuccess) {
        cudaGetLastError();
        throw error{ KSPN_ERR_OOM, "batched workspace of " + std::to_string(bytes) + " bytes" };
      }
      c.plan.base  = b;
      c.plan.bytes = bytes;
    }
    size_t const keep = c.plan.bytes;
    void* const  base = c.plan.base;
    carve_plan(c.plan, static_cast<char*>(base), G, N, &bytes);
    c.plan.base  = base;
    c.plan.bytes = keep;
    c.G = G, c.N = N, c.max_rounds = rounds, c.rem_tarjan = rem, c.cluster_size = csize, c.cluster_min = cmin, c.joint = joint;
    for (int i = 0; i < 6; ++i) c.key[i] = key[i];
    int bps = 0, sms = 0;
    KSPN_CUDA(cudaFuncSetAttribute(k_batch_small, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(BS_WARPS * sizeof(rs_piece))));
    KSPN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_batch_group, BT_THREADS, sizeof(rs_piece)));
    KSPN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    c.block_blocks = static_cast<uint32_t>(std::max(1, bps) * sms);
    c.cluster_blocks = c.block_blocks;
    if (csize > 1) {
      cudaLaunchConfig_t  cfg{};
      cudaLaunchAttribute attr[1];
      attr[0].id               = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = csize;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.gridDim              = dim3(c.block_blocks / csize * csize);
      cfg.blockDim             = dim3(BT_THREADS);
      cfg.dynamicSmemBytes     = sizeof(rs_piece);
      cfg.attrs                = attr;
      cfg.numAttrs             = 1;
      int clusters             = 0;
      KSPN_CUDA(cudaOccupancyMaxActiveClusters(&clusters, k_batch_group, &cfg));
      if (clusters < 1) throw error{ KSPN_ERR_CUDA, "scc_batched: no cluster of that size fits" };
      c.cluster_blocks = static_cast<uint32_t>(clusters) * csize;
    }
    bt_args a{};
    a.G       = G;
    a.vtx_off = vtx_off;
    a.fh = fh, a.fc = fc, a.bh = bh, a.bc = bc;
    a.scc_id = scc_id;
    // capture the call (plan + solve) once, on a private stream (the
    // context's stream may be the legacy default stream, which cannot be
    // captured); later calls replay it on the context's stream
    if (!c.cap_stream) KSPN_CUDA(cudaStreamCreateWithFlags(&c.cap_stream, cudaStreamNonBlocking));
    cudaStream_t const user = ctx->stream;
    KSPN_CUDA(cudaStreamSynchronize(user));
    ctx->stream = c.cap_stream;
    KSPN_CUDA(cudaStreamBeginCapture(c.cap_stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_batch(ctx, c, a);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(c.cap_stream, &g);
      if (g) cudaGraphDestroy(g);
      ctx->stream = user;
      throw;
    }
    cudaError_t const ec = cudaStreamEndCapture(c.cap_stream, &c.graph);
    ctx->stream          = user;
    KSPN_CUDA(ec);
    KSPN_CUDA(cudaGraphInstantiate(&c.exec, c.graph, 0));
  }
  KSPN_CUDA(cudaGraphLaunch(c.exec, ctx->stream));
  ctx->launches += 1;
  uint32_t h[64];
  KSPN_CUDA(cudaMemcpyAsync(h, c.plan.ctr, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h[4]) throw error{ KSPN_ERR_TIMEOUT, "scc_batched: a level or round bound was reached" };
  if (st) {
    st->graphs_small     = h[3];
    st->graphs_large     = h[2] + h[9];
    st->graphs_cluster   = h[2];
    st->cluster_size     = csize;
    st->fwbw_rounds      = h[5];
    st->tarjan_smem      = h[6];
    st->tarjan_serial    = h[7];
    st->trim_levels      = h[8];
    uint64_t ph[5];
    std::memcpy(ph, h + 32, sizeof(ph));
    for (int k = 0; k < 5; ++k) st->phase_ms[k] = static_cast<float>(ph[k] * 1e-6);
  }
}

} // namespace kspn
