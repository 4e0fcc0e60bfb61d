// One warp's Tarjan on a small graph held in shared memory (the residual
// finish and the batched path's small graphs and remainders).
//
// Reference: tarjan (kaspan/scc/tarjan.hpp:20-136), iterative with explicit
// stacks; here on local indices of at most RS_MAXV vertices and RS_MAXE
// edges, every SCC named by its smallest local index.
#pragma once

#include <cstdint>

namespace kspn {

constexpr uint32_t RS_MAXV = 512;  // vertices of a piece decomposed in shared memory
constexpr uint32_t RS_MAXE = 2048; // its internal edges
constexpr uint16_t RS_NONE = 0xFFFF;

// Shared memory of one warp's piece.
struct rs_piece
{
  uint32_t vid[RS_MAXV];       // global ids, ascending
  uint16_t off[RS_MAXV + 2];   // local CSR offsets
  uint16_t adj[RS_MAXE];       // local neighbour indices
  uint16_t index[RS_MAXV], low[RS_MAXV], stk[RS_MAXV], cs_v[RS_MAXV], cs_e[RS_MAXV], comp[RS_MAXV];
  uint8_t  onst[RS_MAXV];
};

// local index of global id v in vid[0, k) (present by construction)
__device__ __forceinline__ uint32_t
rs_local(rs_piece const& p, uint32_t k, uint32_t v)
{
  uint32_t lo = 0, hi = k;
  while (lo + 1 < hi) {
    uint32_t const mid = (lo + hi) / 2;
    if (p.vid[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Iterative Tarjan over the piece (lane 0): comp[i] = smallest local index
// of i's SCC.
__device__ inline void
rs_tarjan(rs_piece& p, uint32_t k)
{
  for (uint32_t i = 0; i < k; ++i) p.index[i] = RS_NONE, p.onst[i] = 0;
  uint32_t idx = 0, sp = 0, cp = 0;
  for (uint32_t s = 0; s < k; ++s) {
    if (p.index[s] != RS_NONE) continue;
    p.index[s] = p.low[s] = static_cast<uint16_t>(idx++);
    p.stk[sp++]           = static_cast<uint16_t>(s);
    p.onst[s]             = 1;
    p.cs_v[cp]            = static_cast<uint16_t>(s);
    p.cs_e[cp++]          = p.off[s];
    while (cp > 0) {
      uint32_t const v = p.cs_v[cp - 1];
      uint32_t const e = p.cs_e[cp - 1];
      if (e < p.off[v + 1]) {
        p.cs_e[cp - 1]   = static_cast<uint16_t>(e + 1);
        uint32_t const w = p.adj[e];
        if (p.index[w] == RS_NONE) {
          p.index[w] = p.low[w] = static_cast<uint16_t>(idx++);
          p.stk[sp++]           = static_cast<uint16_t>(w);
          p.onst[w]             = 1;
          p.cs_v[cp]            = static_cast<uint16_t>(w);
          p.cs_e[cp++]          = p.off[w];
        } else if (p.onst[w] && p.index[w] < p.low[v]) p.low[v] = p.index[w];
      } else {
        --cp;
        if (cp > 0) {
          uint32_t const u = p.cs_v[cp - 1];
          if (p.low[v] < p.low[u]) p.low[u] = p.low[v];
        }
        if (p.low[v] == p.index[v]) {
          // v's SCC: the stack down to v; named by its smallest local index
          uint32_t j = sp, mn = v;
          do {
            --j;
            if (p.stk[j] < mn) mn = p.stk[j];
          } while (p.stk[j] != v);
          for (uint32_t t = j; t < sp; ++t) {
            p.onst[p.stk[t]] = 0;
            p.comp[p.stk[t]] = static_cast<uint16_t>(mn);
          }
          sp = j;
        }
      }
    }
  }
}

} // namespace kspn
