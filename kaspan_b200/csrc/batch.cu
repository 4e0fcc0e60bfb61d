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
//  * k_batch_big: one block per large graph, claimed from the queue:
//    init (degrees, in/out = 0 decided), then rounds of {trim-1 push
//    levels, FW-BW from the largest live in*out (SCC named by its smallest
//    member, its members seed the next trim)} until the remainder has at
//    most `rem_tarjan` vertices -- then Tarjan in shared memory -- or the
//    round cap is reached -- then one thread's Tarjan in global memory.
// Every loop is bounded; a round / level cap sets the error word.
#include "kspn_internal.cuh"
#include "prim.cuh"
#include "tarjan_smem.cuh"

namespace kspn {

namespace {

constexpr int      BT_THREADS = 512;
constexpr int      BT_WARPS   = BT_THREADS / 32;
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
  uint32_t const* order; // graphs sorted: large ones first (n_big of them), then the small ones
  uint32_t*       ctr;   // [0] large claimed, [1] small claimed, [2] n_big, [3] n_small, [4] err,
                         // [5] FW-BW rounds, [6] shared-memory Tarjans, [7] serial Tarjans, [8] trim levels
  uint32_t        max_rounds; // FW-BW rounds per graph before the serial Tarjan
  uint32_t        rem_tarjan; // remainder size that goes to the shared-memory Tarjan (<= RS_MAXV)
};

__device__ __forceinline__ bool
bt_get(uint32_t const* bm, uint32_t v)
{
  return (__ldcg(bm + (v >> 5)) >> (v & 31)) & 1u;
}

// ---------------------------------------------------------------- plan
// Per graph: class key for the sort (large: ~(n + m) so the largest sort
// first; small: all ones, last) and its bitmap word count.
__global__ void
k_bt_classify(uint32_t G, uint64_t const* __restrict__ vtx_off, uint64_t const* __restrict__ fh, uint32_t* keys, uint32_t* vals, uint32_t* words, uint32_t* ctr)
{
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
    uint64_t const vo = vtx_off[g], n = vtx_off[g + 1] - vo;
    uint64_t const m  = fh[vo + n] - fh[vo];
    bool const     small = n <= RS_MAXV && m <= RS_MAXE;
    uint64_t const size  = n + m;
    keys[g]  = small ? 0xFFFFFFFFu : 0xFFFFFFFEu - static_cast<uint32_t>(size < 0xFFFFFFFEull ? size : 0xFFFFFFFEull);
    vals[g]  = g;
    words[g] = static_cast<uint32_t>((n + 31) / 32);
    atomicAdd(ctr + (small ? 3 : 2), 1u);
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
  uint32_t const nb   = __ldcg(a.ctr + 2), ns = __ldcg(a.ctr + 3);
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

// ---------------------------------------------------------------- large graphs
struct bt_smem
{
  uint32_t           g, qn, rem, cnt, minid, lo, hi, flag;
  unsigned long long best;
  unsigned long long wbest[BT_WARPS];
};

// One graph's view for the block.
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
// qin.  Returns the vertices decided.
__device__ uint32_t
bt_trim(bt_args const& a, bt_graph const& G, bt_smem& s, uint32_t* qin, uint32_t qn)
{
  uint32_t  total = 0;
  uint32_t* bufs[2];
  if (qin == G.q0) bufs[0] = G.q1, bufs[1] = G.q2;
  else if (qin == G.q1) bufs[0] = G.q0, bufs[1] = G.q2;
  else bufs[0] = G.q0, bufs[1] = G.q1;
  uint32_t levels = 0;
  for (uint32_t lvl = 0; qn > 0; ++lvl) {
    if (lvl > G.n + 1) {
      if (threadIdx.x == 0) atomicExch(a.ctr + 4, 1u);
      break;
    }
    uint32_t* const qout = bufs[lvl & 1];
    if (threadIdx.x == 0) s.cnt = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < qn; i += BT_THREADS) {
      uint32_t const u = __ldcg(qin + i);
#pragma unroll 1
      for (int dir = 0; dir < 2; ++dir) {
        uint64_t const* head = dir ? G.bh : G.fh;
        uint32_t const* adj  = dir ? a.bc : a.fc;
        uint32_t*       deg  = dir ? G.outdeg : G.indeg;
        for (uint64_t e = head[u], end = head[u + 1]; e < end; ++e) {
          uint32_t const w = adj[e];
          if (bt_get(G.und, w) && atomicSub(deg + w, 1u) == 1u && bit_take(G.und, w)) {
            G.ids[w]              = w;
            qout[atomicAdd(&s.cnt, 1u)] = w;
          }
        }
      }
    }
    __syncthreads();
    qn = s.cnt;
    total += qn;
    qin = qout;
    ++levels;
    __syncthreads();
  }
  if (threadIdx.x == 0 && levels) atomicAdd(a.ctr + 8, levels);
  return total;
}

// Level-synchronous reach from `root` over head/adj rows, among vertices
// whose bit is set in `cand` (nullptr: among undecided vertices), claiming
// bits of `mark`; every reached vertex is appended to `list`.  Returns how
// many were reached.
__device__ uint32_t
bt_reach(bt_args const& a, bt_graph const& G, bt_smem& s, uint64_t const* head, uint32_t const* adj, uint32_t const* cand, uint32_t* mark, uint32_t* list, uint32_t root)
{
  if (threadIdx.x == 0) {
    list[0] = root;
    atomicOr(mark + (root >> 5), 1u << (root & 31));
    s.lo = 0;
    s.hi = 1;
    s.cnt = 1;
  }
  __syncthreads();
  for (uint32_t lvl = 0;; ++lvl) {
    uint32_t const lo = s.lo, hi = s.hi;
    if (lo == hi) break;
    if (lvl > G.n + 1) {
      if (threadIdx.x == 0) atomicExch(a.ctr + 4, 1u);
      break;
    }
    for (uint32_t i = lo + threadIdx.x; i < hi; i += BT_THREADS) {
      uint32_t const u = __ldcg(list + i);
      for (uint64_t e = head[u], end = head[u + 1]; e < end; ++e) {
        uint32_t const w = adj[e];
        if ((cand ? bt_get(cand, w) : bt_get(G.und, w)) && bit_claim(mark, w)) list[atomicAdd(&s.cnt, 1u)] = w;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) s.lo = hi, s.hi = s.cnt;
    __syncthreads();
  }
  __syncthreads();
  uint32_t const c = s.cnt;
  __syncthreads();
  return c;
}

// argmax over undecided v of live in * out (lowest id on ties) into s.best
// as (prod << 32 | ~id) when prod < 2^32, else saturated
__device__ uint32_t
bt_pivot(bt_graph const& G, bt_smem& s)
{
  unsigned long long best = 0;
  for (uint32_t v = threadIdx.x; v < G.n; v += BT_THREADS) {
    if (!bt_get(G.und, v)) continue;
    uint64_t const     p   = static_cast<uint64_t>(__ldcg(G.indeg + v)) * __ldcg(G.outdeg + v);
    unsigned long long key = (static_cast<unsigned long long>(p < 0xFFFFFFFFull ? p : 0xFFFFFFFFull) << 32) | (0xFFFFFFFFu - v);
    best                   = key > best ? key : best;
  }
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) {
    unsigned long long const o = __shfl_xor_sync(0xFFFFFFFFu, best, sh);
    best                       = o > best ? o : best;
  }
  if ((threadIdx.x & 31) == 0) s.wbest[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long b = 0;
    for (int w = 0; w < BT_WARPS; ++w) b = s.wbest[w] > b ? s.wbest[w] : b;
    s.best = b;
  }
  __syncthreads();
  unsigned long long const b = s.best;
  __syncthreads();
  return b ? 0xFFFFFFFFu - static_cast<uint32_t>(b & 0xFFFFFFFFu) : BT_NONE;
}

// The remaining (undecided) vertices of a graph in id order into the
// piece, if there are at most RS_MAXV of them with at most RS_MAXE edges
// among them; warp 0 then runs Tarjan and writes ids.  Returns false (and
// changes nothing) when they do not fit.
__device__ bool
bt_tarjan_smem(bt_args const& a, bt_graph const& G, bt_smem& s, rs_piece& p)
{
  unsigned const lane = threadIdx.x & 31u;
  if (threadIdx.x < 32) {
    // ordered compaction of the und words (warp 0)
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
    }
    __syncwarp();
    bool fits = k <= RS_MAXV;
    // internal out-edges per listed vertex
    uint32_t const per = (k + 31) / 32;
    uint32_t       cnt = 0;
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
    fits             = fits && total <= RS_MAXE;
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
    if (lane == 0) s.flag = fits ? 1u : 0u;
  }
  __syncthreads();
  bool const ok = s.flag != 0;
  __syncthreads();
  return ok;
}

// One thread's iterative Tarjan (tarjan.hpp:20-136) over the undecided
// sub-graph in global memory: index in indeg, low in outdeg, the SCC stack
// in q0, the call stack's vertices in q1 and edge cursors in pos; on-stack
// flags in vis_a.  The last resort after the round cap; bounded by n + m
// steps.
__device__ void
bt_tarjan_serial(bt_args const& a, bt_graph const& G, uint64_t* pos)
{
  __syncthreads();
  for (uint32_t v = threadIdx.x; v < G.n; v += BT_THREADS) G.indeg[v] = BT_NONE;
  for (uint32_t w = threadIdx.x; w < G.words; w += BT_THREADS) G.va[w] = 0;
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(a.ctr + 7, 1u);
    uint32_t idx = 0, sp = 0, cp = 0;
    for (uint32_t r = 0; r < G.n; ++r) {
      if (!bt_get(G.und, r) || G.indeg[r] != BT_NONE) continue;
      G.indeg[r] = G.outdeg[r] = idx++;
      G.q0[sp++]             = r;
      G.va[r >> 5] |= 1u << (r & 31);
      G.q1[cp] = r;
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
            G.q0[sp++]             = w;
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
  __syncthreads();
}

__device__ void
bt_solve(bt_args const& a, uint32_t g, bt_smem& s, rs_piece& piece)
{
  bt_graph G;
  G.vo     = a.vtx_off[g];
  G.n      = static_cast<uint32_t>(a.vtx_off[g + 1] - G.vo);
  G.words  = (G.n + 31) / 32;
  G.fh     = a.fh + G.vo;
  G.bh     = a.bh + G.vo;
  G.und    = a.und + a.word_off[g];
  G.va     = a.vis_a + a.word_off[g];
  G.vb     = a.vis_b + a.word_off[g];
  G.indeg  = a.indeg + G.vo;
  G.outdeg = a.outdeg + G.vo;
  G.ids    = a.scc_id + G.vo;
  G.q0     = a.q0 + G.vo;
  G.q1     = a.q1 + G.vo;
  G.q2     = a.q2 + G.vo;
  uint64_t* const pos = a.pos + G.vo;

  // init: all undecided, live degrees = raw degrees, in/out = 0 decided
  for (uint32_t w = threadIdx.x; w < G.words; w += BT_THREADS) {
    uint32_t const tail = G.n - w * 32;
    G.und[w]            = tail >= 32 ? 0xFFFFFFFFu : (1u << tail) - 1u;
    G.va[w] = G.vb[w] = 0;
  }
  if (threadIdx.x == 0) s.cnt = 0;
  __syncthreads();
  for (uint32_t v = threadIdx.x; v < G.n; v += BT_THREADS) {
    uint32_t const o = static_cast<uint32_t>(G.fh[v + 1] - G.fh[v]);
    uint32_t const i = static_cast<uint32_t>(G.bh[v + 1] - G.bh[v]);
    G.outdeg[v]      = o;
    G.indeg[v]       = i;
    if (o == 0 || i == 0) {
      G.ids[v] = v;
      atomicAnd(G.und + (v >> 5), ~(1u << (v & 31)));
      G.q0[atomicAdd(&s.cnt, 1u)] = v;
    } else G.ids[v] = UNDECIDED;
  }
  __syncthreads();
  uint32_t qn  = s.cnt;
  uint32_t rem = G.n - qn;
  uint32_t* seed = G.q0;
  __syncthreads();
  for (uint32_t round = 0;; ++round) {
    rem -= bt_trim(a, G, s, seed, qn);
    if (rem == 0) break;
    if (rem <= a.rem_tarjan && bt_tarjan_smem(a, G, s, piece)) break;
    if (round >= a.max_rounds) {
      bt_tarjan_serial(a, G, pos);
      break;
    }
    // FW-BW from the largest live in * out
    uint32_t const p = bt_pivot(G, s);
    if (p == BT_NONE) {
      if (threadIdx.x == 0) atomicExch(a.ctr + 4, 1u);
      break;
    }
    uint32_t const nf = bt_reach(a, G, s, G.fh, a.fc, nullptr, G.va, G.q1, p);
    uint32_t const nb = bt_reach(a, G, s, G.bh, a.bc, G.va, G.vb, G.q2, p);
    // the SCC (q2): smallest member, ids, und; vis_a cleared through q1
    uint32_t mn = 0xFFFFFFFFu;
    for (uint32_t i = threadIdx.x; i < nb; i += BT_THREADS) mn = min(mn, __ldcg(G.q2 + i));
    mn = __reduce_min_sync(0xFFFFFFFFu, mn);
    if (threadIdx.x == 0) s.minid = 0xFFFFFFFFu;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicMin(&s.minid, mn);
    __syncthreads();
    uint32_t const id = s.minid;
    for (uint32_t i = threadIdx.x; i < nb; i += BT_THREADS) {
      uint32_t const v = __ldcg(G.q2 + i);
      G.ids[v]         = id;
      atomicAnd(G.und + (v >> 5), ~(1u << (v & 31)));
      atomicAnd(G.vb + (v >> 5), ~(1u << (v & 31)));
    }
    for (uint32_t i = threadIdx.x; i < nf; i += BT_THREADS) {
      uint32_t const v = __ldcg(G.q1 + i);
      atomicAnd(G.va + (v >> 5), ~(1u << (v & 31)));
    }
    if (threadIdx.x == 0) atomicAdd(a.ctr + 5, 1u);
    __syncthreads();
    rem -= nb;
    if (rem == 0) break;
    // the SCC's members seed the next trim
    seed = G.q2;
    qn   = nb;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(BT_THREADS)
k_batch_big(bt_args a)
{
  extern __shared__ __align__(16) unsigned char bt_dyn[];
  rs_piece&         piece = *reinterpret_cast<rs_piece*>(bt_dyn);
  __shared__ bt_smem s;
  uint32_t const     nb = __ldcg(a.ctr + 2);
  for (;;) {
    if (threadIdx.x == 0) s.g = atomicAdd(a.ctr + 0, 1u);
    __syncthreads();
    uint32_t const i = s.g;
    __syncthreads();
    if (i >= nb) break;
    bt_solve(a, a.order[i], s, piece);
  }
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
  uint32_t        max_rounds = 0, rem_tarjan = 0, big_blocks = 0;
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
  p.ctr      = reinterpret_cast<uint32_t*>(take(4 * 32));
  *bytes_out = (off + 255) & ~size_t(255);
}

// The whole call as stream work (captured once per batch and settings).
void
enqueue_batch(kspn_context* ctx, batch_cache& c, bt_args const& a0)
{
  cudaStream_t const s = ctx->stream;
  batch_plan&        p = c.plan;
  uint32_t const     G = c.G;
  KSPN_CUDA(cudaMemsetAsync(p.ctr, 0, 32 * sizeof(uint32_t), s));
  unsigned const cg = div_up(G, 256);
  k_bt_classify<<<cg < 1 ? 1 : cg, 256, 0, s>>>(G, a0.vtx_off, a0.fh, p.keys, p.order, p.words, p.ctr);
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
  k_batch_big<<<c.big_blocks, BT_THREADS, sizeof(rs_piece), s>>>(a);
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
  batch_cache*&  cp     = ctx->batch;
  if (!cp) cp = new batch_cache{};
  batch_cache&      c   = *cp;
  void const* const key[6] = { vtx_off, fh, fc, bh, bc, scc_id };
  bool              same   = c.exec && c.G == G && c.N == N && c.max_rounds == rounds && c.rem_tarjan == rem;
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
    c.G = G, c.N = N, c.max_rounds = rounds, c.rem_tarjan = rem;
    for (int i = 0; i < 6; ++i) c.key[i] = key[i];
    int bps = 0, sms = 0;
    KSPN_CUDA(cudaFuncSetAttribute(k_batch_small, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(BS_WARPS * sizeof(rs_piece))));
    KSPN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_batch_big, BT_THREADS, sizeof(rs_piece)));
    KSPN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    c.big_blocks = static_cast<uint32_t>(std::max(1, bps) * sms);
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
  uint32_t h[32];
  KSPN_CUDA(cudaMemcpyAsync(h, c.plan.ctr, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  if (h[4]) throw error{ KSPN_ERR_TIMEOUT, "scc_batched: a level or round bound was reached" };
  if (st) {
    st->graphs_small     = h[3];
    st->graphs_large     = h[2];
    st->fwbw_rounds      = h[5];
    st->tarjan_smem      = h[6];
    st->tarjan_serial    = h[7];
    st->trim_levels      = h[8];
  }
}

} // namespace kspn
