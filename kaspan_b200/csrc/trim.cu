// Trim phases and pivot selection.
//
//  trim_1_first      kaspan/scc/trim_1_local.hpp:12-46
//  trim_1_normal     kaspan/scc/trim_1_local.hpp:48-73
//  trim_exhaustive_first / trim_fixpoint
//                    kaspan/scc/trim_1_exhaustive.hpp:14-131 (live in/out
//                    degrees; a vertex whose degree drops to 0 is decided and
//                    its neighbours' degrees drop in turn).  On the device the
//                    reference's LIFO frontier becomes a level-synchronous
//                    queue; every directional fixpoint is order-free, so the
//                    decided sets are the same.
//  trim_2            exact size-2 trim (an addition, no reference row)
//  select_pivot_*    kaspan/scc/trim_1_local.hpp:24-45, kaspan/scc/pivot.hpp:53-74
//
// Work per launch is one thread per vertex (streaming passes) or one thread
// per queued vertex with rows of 32+ entries taken by the whole warp.
#include "expand.cuh"

#include <cstring>
#include <tuple>

namespace kspn {

namespace {

constexpr int      T_THREADS = 256;
constexpr uint32_t NONE      = 0xFFFFFFFFu;
constexpr int      WARP_BIG  = 32;
constexpr unsigned HEAVY_GRID = 148 * 8; // blocks of the heavy-row kernels

// Heavy rows in the trim kernels: a vertex with a row longer than HEAVY_ROW
// is listed by the per-vertex kernel and its rows are walked in slices by
// every warp of a follow-up kernel (k_live_heavy, k_push_heavy).
__device__ __forceinline__ bool
row_heavy(uint64_t b, uint64_t e)
{
  return e - b > HEAVY_ROW;
}

// Live (undecided) neighbours in the listed vertices' rows, added to
// outdeg (out-rows) and indeg (in-rows); the listing kernel zeroed both.
__global__ void __launch_bounds__(T_THREADS)
k_live_heavy(uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint64_t const* __restrict__ bh, uint32_t const* __restrict__ bc, uint32_t const* __restrict__ und, uint32_t const* list,
             uint32_t const* list_n, uint32_t* indeg, uint32_t* outdeg)
{
  unsigned const lane = threadIdx.x & 31u;
  uint32_t const cnt  = *list_n;
#pragma unroll 1
  for (int dir = 0; dir < 2; ++dir) {
    uint32_t const* adj = dir ? bc : fc;
    uint32_t*       deg = dir ? indeg : outdeg;
    heavy_slices(list, cnt, dir ? bh : fh, [&](uint32_t, uint32_t v, uint64_t b, uint64_t e) {
      uint32_t c = 0;
      for (uint64_t x = b + lane; x < e; x += 32) c += bit_get(und, adj[x]);
#pragma unroll
      for (int sh = 16; sh; sh >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, sh);
      if (lane == 0 && c) atomicAdd(deg + v, c);
    });
  }
}

// Push step of the listed heavy rows: out-rows of list_out lower their
// neighbours' indeg, in-rows of list_in their outdeg; a neighbour reaching
// 0 is decided and queued (qout).
__device__ __forceinline__ void
push_heavy(uint64_t const* __restrict__ fh,
           uint32_t const* __restrict__ fc,
           uint64_t const* __restrict__ bh,
           uint32_t const* __restrict__ bc,
           uint32_t* __restrict__ und,
           uint32_t* __restrict__ scc_id,
           uint32_t* __restrict__ indeg,
           uint32_t* __restrict__ outdeg,
           uint32_t const* list_out,
           uint32_t const* list_in,
           uint32_t const* list_n, // [0] out-rows, [1] in-rows
           uint32_t* __restrict__ qout,
           uint32_t* __restrict__ qout_n,
           uint32_t* __restrict__ decided)
{
  unsigned const lane = threadIdx.x & 31u;
  uint32_t       dec  = 0;
#pragma unroll 1
  for (int dir = 0; dir < 2; ++dir) {
    uint32_t const* adj = dir ? bc : fc;
    uint32_t*       deg = dir ? outdeg : indeg;
    heavy_slices<true>(dir ? list_in : list_out, list_n[dir], dir ? bh : fh, [&](uint32_t, uint32_t, uint64_t b, uint64_t e) {
      for (uint64_t x = b + lane; x < e; x += 32) {
        uint32_t const w = adj[x];
        if (bit_get(und, w) && atomicSub(deg + w, 1u) == 1u && bit_take(und, w)) {
          scc_id[w] = w;
          ++dec;
          warp_push_active(w, qout, qout_n);
        }
      }
    });
  }
  if (dec) atomicAdd(decided, dec);
}

__global__ void __launch_bounds__(T_THREADS)
k_push_heavy(uint64_t const* __restrict__ fh,
             uint32_t const* __restrict__ fc,
             uint64_t const* __restrict__ bh,
             uint32_t const* __restrict__ bc,
             uint32_t* __restrict__ und,
             uint32_t* __restrict__ scc_id,
             uint32_t* __restrict__ indeg,
             uint32_t* __restrict__ outdeg,
             uint32_t const* list_out,
             uint32_t const* list_in,
             uint32_t const* list_n,
             uint32_t* __restrict__ qout,
             uint32_t* __restrict__ qout_n,
             uint32_t* __restrict__ decided)
{
  push_heavy(fh, fc, bh, bc, und, scc_id, indeg, outdeg, list_out, list_in, list_n, qout, qout_n, decided);
}

unsigned
stream_grid(uint64_t items)
{
  uint64_t const b = (items + T_THREADS - 1) / T_THREADS;
  return static_cast<unsigned>(b < 148ull * 16 ? (b ? b : 1) : 148ull * 16);
}

// (product, id) pairs: larger product wins, then smaller id
struct pv
{
  uint64_t prod;
  uint32_t id;
};
__device__ __forceinline__ pv
pv_best(pv a, pv b)
{
  if (b.prod > a.prod || (b.prod == a.prod && b.id < a.id)) return b;
  return a;
}
__device__ __forceinline__ pv
pv_warp_reduce(pv x)
{
#pragma unroll
  for (int d = 16; d; d >>= 1) {
    pv y;
    y.prod = __shfl_down_sync(0xFFFFFFFFu, x.prod, d);
    y.id   = __shfl_down_sync(0xFFFFFFFFu, x.id, d);
    x      = pv_best(x, y);
  }
  return x;
}
// block reduction of x into out_prod[slot] / out_id[slot]
__device__ __forceinline__ void
pv_block_store_at(pv x, uint64_t* out_prod, uint32_t* out_id, uint32_t slot)
{
  __shared__ uint64_t sp[T_THREADS / 32];
  __shared__ uint32_t si[T_THREADS / 32];
  x = pv_warp_reduce(x);
  if ((threadIdx.x & 31) == 0) sp[threadIdx.x >> 5] = x.prod, si[threadIdx.x >> 5] = x.id;
  __syncthreads();
  if (threadIdx.x < 32) {
    pv y = { 0, NONE };
    if (threadIdx.x < T_THREADS / 32) y = { sp[threadIdx.x], si[threadIdx.x] };
    y = pv_warp_reduce(y);
    if (threadIdx.x == 0) out_prod[slot] = y.prod, out_id[slot] = y.id;
  }
}
__device__ __forceinline__ void
pv_block_store(pv x, uint64_t* out_prod, uint32_t* out_id)
{
  pv_block_store_at(x, out_prod, out_id, blockIdx.x);
}

// Final reduction of per-block pairs; result id in out_id[0] (NONE if no
// pair had a product > min_prod... the caller interprets).
__global__ void
k_pv_final(uint32_t nb, uint64_t* prod, uint32_t* id)
{
  pv x = { 0, NONE };
  for (uint32_t i = threadIdx.x; i < nb; i += 32) x = pv_best(x, pv{ prod[i], id[i] });
  x = pv_warp_reduce(x);
  if (threadIdx.x == 0) prod[0] = x.prod, id[0] = x.id;
}

// ---------------------------------------------------------------- trim_1_first
constexpr int TF_ITEMS = 4; // vertices per thread per pass of k_trim_first

__global__ void __launch_bounds__(T_THREADS)
k_trim_first(uint32_t n,
             uint64_t const* __restrict__ fh,
             uint64_t const* __restrict__ bh,
             uint32_t* __restrict__ und,
             uint32_t* __restrict__ scc_id,
             uint32_t* __restrict__ indeg,
             uint32_t* __restrict__ outdeg,
             uint32_t* __restrict__ queue,
             uint32_t* __restrict__ ctr,
             uint64_t* __restrict__ blk_prod,
             uint32_t* __restrict__ blk_id)
{
  __shared__ uint32_t s_buf[DENSE_BUF];
  __shared__ uint32_t s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  block_queue    bq{ s_buf, &s_n };
  pv             best = { 0, NONE };
  uint32_t       dec  = 0;
  // a pass covers TF_ITEMS slices of T_THREADS vertices; all offset loads
  // of a pass are issued before any is used
  uint64_t const pass     = static_cast<uint64_t>(T_THREADS) * TF_ITEMS;
  for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * pass; base < n; base += static_cast<uint64_t>(gridDim.x) * pass) {
    uint64_t f0[TF_ITEMS], f1[TF_ITEMS], b0[TF_ITEMS], b1[TF_ITEMS];
#pragma unroll
    for (int k = 0; k < TF_ITEMS; ++k) {
      uint64_t const t = base + k * T_THREADS + threadIdx.x;
      f0[k] = f1[k] = b0[k] = b1[k] = 0;
      if (t < n) f0[k] = fh[t], f1[k] = fh[t + 1], b0[k] = bh[t], b1[k] = bh[t + 1];
    }
#pragma unroll
    for (int k = 0; k < TF_ITEMS; ++k) {
      uint64_t const t       = base + k * T_THREADS + threadIdx.x;
      uint32_t const v       = static_cast<uint32_t>(t);
      bool const     valid   = t < n;
      uint64_t const out     = f1[k] - f0[k];
      uint64_t const in      = b1[k] - b0[k];
      bool const     trimmed = valid && (in == 0 || out == 0);
      bool const     live    = valid && !trimmed;
      unsigned const word    = __ballot_sync(0xFFFFFFFFu, live);
      if ((threadIdx.x & 31) == 0 && t < n) und[v >> 5] = word; // t = the warp's first vertex
      if (valid && scc_id) scc_id[v] = trimmed ? v : UNDECIDED; // scc_id null: the caller writes ids later
      if (live) {
        if (indeg) indeg[v] = static_cast<uint32_t>(in);
        if (outdeg) outdeg[v] = static_cast<uint32_t>(out);
        uint64_t const prod = in * out;
        if (prod > best.prod) best = { prod, v }; // ascending v: first strict max wins
      }
      if (queue) {
        bq.push(trimmed, v);
        __syncthreads();
        if (s_n > DENSE_BUF - T_THREADS) bq.flush(queue, ctr + CTR_Q0, &s_base);
      }
      dec += trimmed;
    }
  }
  if (queue) bq.flush(queue, ctr + CTR_Q0, &s_base);
  // decided count
  unsigned d = dec;
#pragma unroll
  for (int s = 16; s; s >>= 1) d += __shfl_down_sync(0xFFFFFFFFu, d, s);
  if ((threadIdx.x & 31) == 0 && d) atomicAdd(ctr + CTR_DECIDED, d);
  pv_block_store(best, blk_prod, blk_id);
  // the last block to finish reduces every block's pair into PV_FINAL, so a
  // later launch can read the pivot without a host round trip
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(ctr + CTR_PV_TICKET, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  pv x = { 0, NONE };
  for (uint32_t i = threadIdx.x; i < gridDim.x; i += T_THREADS) x = pv_best(x, pv{ __ldcg(blk_prod + i), __ldcg(blk_id + i) });
  pv_block_store_at(x, blk_prod, blk_id, PV_FINAL);
  if (threadIdx.x == 0) ctr[CTR_PV_TICKET] = 0;
}

// ---------------------------------------------------------------- trim_1_normal
__global__ void __launch_bounds__(T_THREADS)
k_trim_normal(uint32_t n,
              uint64_t const* __restrict__ fh,
              uint32_t const* __restrict__ fc,
              uint64_t const* __restrict__ bh,
              uint32_t const* __restrict__ bc,
              uint32_t* __restrict__ und,
              uint32_t* __restrict__ scc_id,
              uint32_t* __restrict__ ctr)
{
  uint32_t dec = 0;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < n; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint32_t const v = static_cast<uint32_t>(t);
    if (!bit_get(und, v)) continue;
    bool has = false;
    for (uint64_t e = fh[v], end = fh[v + 1]; e < end && !has; ++e) has = bit_get(und, fc[e]);
    for (uint64_t e = bh[v], end = bh[v + 1]; e < end && !has; ++e) has = bit_get(und, bc[e]);
    if (!has && bit_take(und, v)) {
      scc_id[v] = v;
      ++dec;
    }
  }
  if (dec) atomicAdd(ctr + CTR_DECIDED, dec);
}

// ---------------------------------------------------------------- live degrees (pull)
// For every undecided v: indeg/outdeg = undecided neighbours (with
// multiplicity).  Counting only; k_seed_dead decides in a second launch so
// every count sees the same undecided set (a vertex decided while others
// still count would be subtracted twice by the push levels).
__global__ void __launch_bounds__(T_THREADS)
k_live_degrees(uint32_t n,
               uint64_t const* __restrict__ fh,
               uint32_t const* __restrict__ fc,
               uint64_t const* __restrict__ bh,
               uint32_t const* __restrict__ bc,
               uint32_t const* __restrict__ und,
               uint32_t* __restrict__ indeg,
               uint32_t* __restrict__ outdeg,
               uint32_t* heavy,
               uint32_t* heavy_n)
{
  unsigned const lane = threadIdx.x & 31u;
  uint64_t const span = (static_cast<uint64_t>(n) + 31) & ~31ull;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint32_t const v    = static_cast<uint32_t>(t);
    bool           have = t < n && bit_get(und, v);
    uint64_t       fb = 0, fe = 0, bb = 0, be = 0;
    if (have) fb = fh[v], fe = fh[v + 1], bb = bh[v], be = bh[v + 1];
    bool const hv = have && (row_heavy(fb, fe) || row_heavy(bb, be));
    if (hv) indeg[v] = outdeg[v] = 0; // counted by k_live_heavy
    warp_push(hv, v, heavy, heavy_n);
    have &= !hv;
    uint32_t   outc  = 0, inc = 0;
    bool const small = have && (fe - fb) < WARP_BIG && (be - bb) < WARP_BIG;
    if (small) {
      for (uint64_t e = fb; e < fe; ++e) outc += bit_get(und, fc[e]);
      for (uint64_t e = bb; e < be; ++e) inc += bit_get(und, bc[e]);
    }
    unsigned todo = __ballot_sync(0xFFFFFFFFu, have && !small);
    while (todo) {
      unsigned const l = __ffs(todo) - 1;
      todo &= todo - 1;
      uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, fb, l), e0 = __shfl_sync(0xFFFFFFFFu, fe, l);
      uint64_t const b1 = __shfl_sync(0xFFFFFFFFu, bb, l), e1 = __shfl_sync(0xFFFFFFFFu, be, l);
      uint32_t       a = 0, c = 0;
      for (uint64_t e = b0 + lane; e < e0; e += 32) a += bit_get(und, fc[e]);
      for (uint64_t e = b1 + lane; e < e1; e += 32) c += bit_get(und, bc[e]);
#pragma unroll
      for (int s = 16; s; s >>= 1) a += __shfl_xor_sync(0xFFFFFFFFu, a, s), c += __shfl_xor_sync(0xFFFFFFFFu, c, s);
      if (lane == l) outc = a, inc = c;
    }
    if (have) {
      indeg[v]  = inc;
      outdeg[v] = outc;
    }
  }
}

// Decides (and queues) every undecided vertex whose live in- or out-degree is 0.
__global__ void __launch_bounds__(T_THREADS)
k_seed_dead(uint32_t n, uint32_t* __restrict__ und, uint32_t* __restrict__ scc_id, uint32_t const* __restrict__ indeg, uint32_t const* __restrict__ outdeg, uint32_t* __restrict__ queue, uint32_t* __restrict__ ctr)
{
  __shared__ uint32_t s_buf[DENSE_BUF];
  __shared__ uint32_t s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  block_queue    bq{ s_buf, &s_n };
  uint64_t const span = (static_cast<uint64_t>(n) + T_THREADS - 1) / T_THREADS * T_THREADS;
  for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * T_THREADS; base < span; base += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint64_t const t    = base + threadIdx.x;
    uint32_t const v    = static_cast<uint32_t>(t);
    bool const     dead = t < n && bit_get(und, v) && (indeg[v] == 0 || outdeg[v] == 0);
    bool const     won  = dead && bit_take(und, v);
    if (won) scc_id[v] = v;
    bq.push(won, v);
    __syncthreads();
    if (s_n > DENSE_BUF - T_THREADS) bq.flush(queue, ctr + CTR_Q0, &s_base);
  }
  bq.flush(queue, ctr + CTR_Q0, &s_base);
}

// ---------------------------------------------------------------- push-based trim level
// Each queued (just decided) u lowers the live in-degree of its undecided
// out-neighbours (dirs & 1) and the live out-degree of its undecided
// in-neighbours (dirs & 2); a neighbour reaching 0 is decided and queued.
template<int DIRS>
__global__ void __launch_bounds__(T_THREADS)
k_trim_push(uint64_t const* __restrict__ fh,
            uint32_t const* __restrict__ fc,
            uint64_t const* __restrict__ bh,
            uint32_t const* __restrict__ bc,
            uint32_t* __restrict__ und,
            uint32_t* __restrict__ scc_id,
            uint32_t* __restrict__ indeg,
            uint32_t* __restrict__ outdeg,
            uint32_t const* __restrict__ qin,
            uint32_t qn,
            uint32_t* __restrict__ qout,
            uint32_t* __restrict__ qout_n,
            uint32_t* __restrict__ ctr,
            unsigned long long* __restrict__ edges,
            uint32_t* heavy_out,
            uint32_t* heavy_in,
            uint32_t* heavy_n)
{
  unsigned const lane = threadIdx.x & 31u;
  uint64_t const span = (static_cast<uint64_t>(qn) + 31) & ~31ull;
  uint32_t       dec  = 0;
  uint64_t       ne   = 0;
  auto const     hit  = [&](uint32_t w, uint32_t* deg) {
    if (bit_get(und, w) && atomicSub(deg + w, 1u) == 1u && bit_take(und, w)) {
      scc_id[w] = w;
      ++dec;
      warp_push_active(w, qout, qout_n);
    }
  };
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    if (!(DIRS & (1 << dir))) continue;
    uint64_t const* head = dir == 0 ? fh : bh;
    uint32_t const* adj  = dir == 0 ? fc : bc;
    uint32_t*       deg  = dir == 0 ? indeg : outdeg;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
      bool const     have = t < qn;
      uint32_t const u    = have ? qin[t] : 0;
      uint64_t       b = 0, e = 0;
      if (have) b = head[u], e = head[u + 1];
      bool const hv  = have && row_heavy(b, e); // k_push_heavy walks it
      bool const big = have && !hv && (e - b) >= WARP_BIG;
      ne += e - b;
      warp_push(hv, u, dir == 0 ? heavy_out : heavy_in, heavy_n + dir);
      if (have && !big && !hv)
        for (uint64_t x = b; x < e; ++x) hit(adj[x], deg);
      unsigned todo = __ballot_sync(0xFFFFFFFFu, big);
      while (todo) {
        unsigned const l = __ffs(todo) - 1;
        todo &= todo - 1;
        uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, b, l), e0 = __shfl_sync(0xFFFFFFFFu, e, l);
        for (uint64_t x = b0 + lane; x < e0; x += 32) hit(adj[x], deg);
      }
    }
  }
  if (dec) atomicAdd(ctr + CTR_DECIDED, dec);
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) ne += __shfl_down_sync(0xFFFFFFFFu, ne, sh);
  if (lane == 0 && ne) atomicAdd(edges, static_cast<unsigned long long>(ne));
}

// Reference-exact seeding of trim_1_exhaustive_first's sweeps
// (kaspan/scc/trim_1_exhaustive.hpp:82-97 and :108-123): over the vertices
// still undecided, deg = raw degree in this direction; raw 0 => decided now.
__global__ void __launch_bounds__(T_THREADS)
k_seed_raw(uint32_t n, uint64_t const* __restrict__ head, uint32_t* __restrict__ und, uint32_t* __restrict__ scc_id, uint32_t* __restrict__ deg, uint32_t* __restrict__ queue, uint32_t* __restrict__ ctr)
{
  __shared__ uint32_t s_buf[DENSE_BUF];
  __shared__ uint32_t s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  block_queue    bq{ s_buf, &s_n };
  uint64_t const span = (static_cast<uint64_t>(n) + T_THREADS - 1) / T_THREADS * T_THREADS;
  uint32_t       dec  = 0;
  for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * T_THREADS; base < span; base += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint64_t const t    = base + threadIdx.x;
    uint32_t const v    = static_cast<uint32_t>(t);
    bool const     have = t < n && bit_get(und, v);
    bool           won  = false;
    if (have) {
      uint64_t const d = head[v + 1] - head[v];
      if (d > 0) deg[v] = static_cast<uint32_t>(d);
      else if (bit_take(und, v)) {
        scc_id[v] = v;
        won       = true;
        ++dec;
      }
    }
    bq.push(won, v);
    __syncthreads();
    if (s_n > DENSE_BUF - T_THREADS) bq.flush(queue, ctr + CTR_Q0, &s_base);
  }
  bq.flush(queue, ctr + CTR_Q0, &s_base);
  if (dec) atomicAdd(ctr + CTR_DECIDED, dec);
}

// ---------------------------------------------------------------- trim-2
// one[v] = the single distinct undecided neighbour of v in a direction, or
// NONE (zero or several distinct ones).
__global__ void __launch_bounds__(T_THREADS)
k_unique_neighbour(uint32_t n, uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint64_t const* __restrict__ bh, uint32_t const* __restrict__ bc, uint32_t const* __restrict__ und, uint32_t* __restrict__ out_one, uint32_t* __restrict__ in_one)
{
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < n; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint32_t const v = static_cast<uint32_t>(t);
    if (!bit_get(und, v)) continue;
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      uint64_t const* head = dir ? bh : fh;
      uint32_t const* adj  = dir ? bc : fc;
      uint32_t        one  = NONE;
      bool            many = false;
      for (uint64_t e = head[v], end = head[v + 1]; e < end; ++e) {
        uint32_t const w = adj[e];
        if (!bit_get(und, w)) continue;
        if (one == NONE) one = w;
        else if (w != one) {
          many = true;
          break;
        }
      }
      (dir ? in_one : out_one)[v] = many ? NONE : one;
    }
  }
}

__global__ void __launch_bounds__(T_THREADS)
k_trim2_decide(uint32_t n, uint32_t const* __restrict__ out_one, uint32_t const* __restrict__ in_one, uint32_t* __restrict__ und, uint32_t* __restrict__ scc_id, uint32_t* __restrict__ ctr)
{
  uint32_t dec = 0;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < n; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint32_t const u = static_cast<uint32_t>(t);
    if (!bit_get(und, u)) continue;
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
      uint32_t const* one = dir ? in_one : out_one;
      uint32_t const  v   = one[u];
      if (v == NONE || v <= u || v >= n) continue;
      if (one[v] != u) continue;
      // u < v, each the other's only undecided neighbour in this direction:
      // {u, v} is closed under that direction, so it is an SCC
      if (bit_take(und, u)) {
        bit_take(und, v);
        scc_id[u] = u;
        scc_id[v] = u;
        dec += 2;
      }
    }
  }
  if (dec) atomicAdd(ctr + CTR_DECIDED, dec);
}

// ---------------------------------------------------------------- pivots / counts
__global__ void __launch_bounds__(T_THREADS)
k_pivot_live(uint32_t n, uint32_t const* __restrict__ und, uint32_t const* __restrict__ indeg, uint32_t const* __restrict__ outdeg, uint64_t* __restrict__ blk_prod, uint32_t* __restrict__ blk_id)
{
  pv best = { 0, NONE };
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < n; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint32_t const v = static_cast<uint32_t>(t);
    if (!bit_get(und, v)) continue;
    pv const c = { static_cast<uint64_t>(outdeg[v]) * indeg[v] + 1, v }; // +1: any undecided vertex beats none
    best       = pv_best(best, c);
  }
  pv_block_store(best, blk_prod, blk_id);
}

__global__ void __launch_bounds__(T_THREADS)
k_popcount(uint32_t words, uint32_t n, uint32_t const* __restrict__ bm, uint32_t* __restrict__ out)
{
  uint32_t c = 0;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < words; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint32_t w = bm[t];
    if ((t + 1) * 32 > n) {
      uint32_t const valid = n - static_cast<uint32_t>(t) * 32;
      w &= valid >= 32 ? 0xFFFFFFFFu : ((1u << valid) - 1u);
    }
    c += __popc(w);
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, s);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// ---------------------------------------------------------------- device-driven trim fixpoint
// Control block of one trim fixpoint (workspace, after the FW-BW block).
struct trim_state
{
  uint32_t           cur;    // queue selector (fio)
  uint32_t           qn[2];  // queue lengths
  uint32_t           level;  // push levels run
  uint32_t           cap;    // level cap
  uint32_t           err;    // 1: cap hit
  uint32_t           decided;
  uint32_t           list_n; // undecided vertices at the start
  unsigned long long edges;  // edges pushed along
  uint32_t           heavy_n[3]; // heavy rows listed: push out-rows, push in-rows (this level), live counts
};

// The level's heavy rows (listed by k_t_push) into the same output queue.
__global__ void __launch_bounds__(T_THREADS)
k_t_push_heavy(uint64_t const* __restrict__ fh,
               uint32_t const* __restrict__ fc,
               uint64_t const* __restrict__ bh,
               uint32_t const* __restrict__ bc,
               uint32_t* __restrict__ und,
               uint32_t* __restrict__ scc_id,
               uint32_t* __restrict__ indeg,
               uint32_t* __restrict__ outdeg,
               fio f,
               trim_state* st,
               uint32_t const* heavy_out,
               uint32_t const* heavy_in)
{
  push_heavy(fh, fc, bh, bc, und, scc_id, indeg, outdeg, heavy_out, heavy_in, st->heavy_n, f.out(), f.out_n(), &st->decided);
}

__global__ void
k_t_init(trim_state* st)
{
  uint32_t const cap = st->cap;
  st->cur = st->qn[0] = st->qn[1] = st->level = st->err = st->decided = st->list_n = 0;
  st->heavy_n[0] = st->heavy_n[1] = st->heavy_n[2] = 0;
  st->edges = 0;
  st->cap   = cap;
}

// Undecided vertex ids -> list (one bitmap word per thread, block scan of
// popcounts, one global atomic per block).
__global__ void __launch_bounds__(T_THREADS)
k_t_compact(uint32_t n, uint32_t const* __restrict__ und, uint32_t* __restrict__ list, trim_state* st)
{
  __shared__ uint32_t s_base;
  uint32_t const      words = (n + 31) / 32;
  for (uint32_t wbase = blockIdx.x * T_THREADS; wbase < words; wbase += gridDim.x * T_THREADS) {
    uint32_t const w    = wbase + threadIdx.x;
    uint32_t       word = w < words ? und[w] : 0u;
    if (w == words - 1 && (n & 31)) word &= (1u << (n & 31)) - 1u;
    uint32_t total;
    uint32_t off = block_exclusive_scan<uint32_t, T_THREADS>(static_cast<uint32_t>(__popc(word)), &total);
    if (threadIdx.x == 0) s_base = total ? atomicAdd(&st->list_n, total) : 0;
    __syncthreads();
    uint32_t j = s_base + off;
    while (word) {
      uint32_t const b = __ffs(word) - 1;
      word &= word - 1;
      list[j++] = w * 32 + b;
    }
    __syncthreads();
  }
}

// Live degrees of the listed (undecided) vertices; rows of WARP_BIG+ by
// the whole warp.
__global__ void __launch_bounds__(T_THREADS)
k_t_live(uint64_t const* __restrict__ fh, uint32_t const* __restrict__ fc, uint64_t const* __restrict__ bh, uint32_t const* __restrict__ bc, uint32_t const* __restrict__ und, uint32_t const* __restrict__ list,
         trim_state* st, uint32_t* __restrict__ indeg, uint32_t* __restrict__ outdeg, uint32_t* heavy)
{
  unsigned const lane = threadIdx.x & 31u;
  uint32_t const ln   = st->list_n;
  uint64_t const span = (static_cast<uint64_t>(ln) + 31) & ~31ull;
  for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    bool           have = t < ln;
    uint32_t const v    = have ? list[t] : 0u;
    uint64_t       fb = 0, fe = 0, bb = 0, be = 0;
    if (have) fb = fh[v], fe = fh[v + 1], bb = bh[v], be = bh[v + 1];
    bool const hv = have && (row_heavy(fb, fe) || row_heavy(bb, be));
    if (hv) indeg[v] = outdeg[v] = 0; // counted by k_live_heavy
    warp_push(hv, v, heavy, &st->heavy_n[2]);
    have &= !hv;
    uint32_t   outc  = 0, inc = 0;
    bool const small = have && (fe - fb) < WARP_BIG && (be - bb) < WARP_BIG;
    if (small) {
      for (uint64_t e = fb; e < fe; ++e) outc += bit_get(und, fc[e]);
      for (uint64_t e = bb; e < be; ++e) inc += bit_get(und, bc[e]);
    }
    unsigned todo = __ballot_sync(0xFFFFFFFFu, have && !small);
    while (todo) {
      unsigned const l = __ffs(todo) - 1;
      todo &= todo - 1;
      uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, fb, l), e0 = __shfl_sync(0xFFFFFFFFu, fe, l);
      uint64_t const b1 = __shfl_sync(0xFFFFFFFFu, bb, l), e1 = __shfl_sync(0xFFFFFFFFu, be, l);
      uint32_t       a = 0, c = 0;
      for (uint64_t e = b0 + lane; e < e0; e += 32) a += bit_get(und, fc[e]);
      for (uint64_t e = b1 + lane; e < e1; e += 32) c += bit_get(und, bc[e]);
#pragma unroll
      for (int s = 16; s; s >>= 1) a += __shfl_xor_sync(0xFFFFFFFFu, a, s), c += __shfl_xor_sync(0xFFFFFFFFu, c, s);
      if (lane == l) outc = a, inc = c;
    }
    if (have) {
      indeg[v]  = inc;
      outdeg[v] = outc;
    }
  }
}

// Listed vertices with a live degree of 0 are decided and queued (q0).
__global__ void __launch_bounds__(T_THREADS)
k_t_seed(uint32_t* __restrict__ und, uint32_t* __restrict__ scc_id, uint32_t const* __restrict__ indeg, uint32_t const* __restrict__ outdeg, uint32_t const* __restrict__ list, trim_state* st, uint32_t* __restrict__ q0)
{
  __shared__ uint32_t s_buf[DENSE_BUF];
  __shared__ uint32_t s_n, s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  block_queue    bq{ s_buf, &s_n };
  uint32_t const ln   = st->list_n;
  uint64_t const span = (static_cast<uint64_t>(ln) + T_THREADS - 1) / T_THREADS * T_THREADS;
  uint32_t       dec  = 0;
  for (uint64_t base = static_cast<uint64_t>(blockIdx.x) * T_THREADS; base < span; base += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
    uint64_t const t    = base + threadIdx.x;
    uint32_t const v    = t < ln ? list[t] : 0u;
    bool const     dead = t < ln && (indeg[v] == 0 || outdeg[v] == 0);
    bool const     won  = dead && bit_take(und, v);
    if (won) {
      scc_id[v] = v;
      ++dec;
    }
    bq.push(won, v);
    __syncthreads();
    if (s_n > DENSE_BUF - T_THREADS) bq.flush(q0, &st->qn[0], &s_base);
  }
  bq.flush(q0, &st->qn[0], &s_base);
  if (dec) atomicAdd(&st->decided, dec);
}

// One push level (both directions) from the fio input queue to its output.
__global__ void __launch_bounds__(T_THREADS)
k_t_push(uint64_t const* __restrict__ fh,
         uint32_t const* __restrict__ fc,
         uint64_t const* __restrict__ bh,
         uint32_t const* __restrict__ bc,
         uint32_t* __restrict__ und,
         uint32_t* __restrict__ scc_id,
         uint32_t* __restrict__ indeg,
         uint32_t* __restrict__ outdeg,
         fio f,
         trim_state* st,
         uint32_t* heavy_out,
         uint32_t* heavy_in)
{
  unsigned const  lane   = threadIdx.x & 31u;
  uint32_t const* qin    = f.in();
  uint32_t const  qn     = f.in_n();
  uint32_t* const qout   = f.out();
  uint32_t* const qout_n = f.out_n();
  uint64_t const  span   = (static_cast<uint64_t>(qn) + 31) & ~31ull;
  uint32_t        dec    = 0;
  uint64_t        ne     = 0;
  auto const      hit    = [&](uint32_t w, uint32_t* deg) {
    if (bit_get(und, w) && atomicSub(deg + w, 1u) == 1u && bit_take(und, w)) {
      scc_id[w] = w;
      ++dec;
      warp_push_active(w, qout, qout_n);
    }
  };
#pragma unroll
  for (int dir = 0; dir < 2; ++dir) {
    uint64_t const* head = dir == 0 ? fh : bh;
    uint32_t const* adj  = dir == 0 ? fc : bc;
    uint32_t*       deg  = dir == 0 ? indeg : outdeg;
    for (uint64_t t = static_cast<uint64_t>(blockIdx.x) * T_THREADS + threadIdx.x; t < span; t += static_cast<uint64_t>(gridDim.x) * T_THREADS) {
      bool const     have = t < qn;
      uint32_t const u    = have ? qin[t] : 0;
      uint64_t       b = 0, e = 0;
      if (have) b = head[u], e = head[u + 1];
      bool const hv  = have && row_heavy(b, e); // k_t_push_heavy walks it
      bool const big = have && !hv && (e - b) >= WARP_BIG;
      ne += e - b;
      warp_push(hv, u, dir == 0 ? heavy_out : heavy_in, &st->heavy_n[dir]);
      if (have && !big && !hv)
        for (uint64_t x = b; x < e; ++x) hit(adj[x], deg);
      unsigned todo = __ballot_sync(0xFFFFFFFFu, big);
      while (todo) {
        unsigned const l = __ffs(todo) - 1;
        todo &= todo - 1;
        uint64_t const b0 = __shfl_sync(0xFFFFFFFFu, b, l), e0 = __shfl_sync(0xFFFFFFFFu, e, l);
        for (uint64_t x = b0 + lane; x < e0; x += 32) hit(adj[x], deg);
      }
    }
  }
  if (dec) atomicAdd(&st->decided, dec);
#pragma unroll
  for (int sh = 16; sh; sh >>= 1) ne += __shfl_down_sync(0xFFFFFFFFu, ne, sh);
  if (lane == 0 && ne) atomicAdd(&st->edges, static_cast<unsigned long long>(ne));
}

__global__ void
k_t_advance(trim_state* st, cudaGraphConditionalHandle h, int in_graph)
{
  st->level += 1;
  st->heavy_n[0] = st->heavy_n[1] = 0; // the level's heavy rows were walked
  st->cur ^= 1u;
  st->qn[(st->cur & 1u) ^ 1u] = 0; // next level's output
  unsigned cond = st->qn[st->cur & 1u] > 0;
  if (cond && st->level >= st->cap) {
    st->err = 1;
    cond    = 0;
  }
  if (in_graph) cudaGraphSetConditional(h, cond);
}

template<typename... KArgs, typename... Vals>
cudaGraphNode_t
t_add_kernel(cudaGraph_t g, cudaGraphNode_t dep, void (*fn)(KArgs...), unsigned grid, unsigned block, Vals... vals)
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
  p.kernelParams         = params;
  cudaGraphNode_t node   = nullptr;
  KSPN_CUDA(cudaGraphAddKernelNode(&node, g, dep ? &dep : nullptr, dep ? 1 : 0, &p));
  return node;
}

trim_state*
trim_state_dev(kspn_context* ctx)
{
  return reinterpret_cast<trim_state*>(static_cast<char*>(ctx->ws.rstate) + 512);
}
trim_state*
trim_state_host(kspn_context* ctx)
{
  return reinterpret_cast<trim_state*>(static_cast<char*>(ctx->h_state) + 512);
}

void
build_trim_graph(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id)
{
  auto&          ws    = ctx->ws;
  trim_state*    st    = trim_state_dev(ctx);
  uint32_t const words = (g.n + 31) / 32;
  cudaGraph_t    graph = nullptr;
  KSPN_CUDA(cudaGraphCreate(&graph, 0));
  try {
    unsigned const  wgrid = stream_grid(words);
    unsigned const  vgrid = stream_grid(g.n);
    cudaGraphNode_t dep   = nullptr;
    dep = t_add_kernel(graph, dep, &k_t_init, 1, 1, st);
    dep = t_add_kernel(graph, dep, &k_t_compact, wgrid, T_THREADS, g.n, und, ws.q1, st);
    uint32_t* const h_out  = ws.heavy;
    uint32_t* const h_in   = ws.heavy + ws.heavy_cap;
    uint32_t* const h_live = ws.heavy + 2 * ws.heavy_cap;
    dep = t_add_kernel(graph, dep, &k_t_live, vgrid, T_THREADS, g.fh, g.fc, g.bh, g.bc, und, ws.q1, st, ws.indeg, ws.outdeg, h_live);
    dep = t_add_kernel(graph, dep, &k_live_heavy, HEAVY_GRID, T_THREADS, g.fh, g.fc, g.bh, g.bc, und, h_live, &st->heavy_n[2], ws.indeg, ws.outdeg);
    dep = t_add_kernel(graph, dep, &k_t_seed, vgrid, T_THREADS, und, scc_id, ws.indeg, ws.outdeg, ws.q1, st, ws.q0);
    cudaGraphConditionalHandle h;
    KSPN_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type                = cudaGraphNodeTypeConditional;
    cp.conditional.handle  = h;
    cp.conditional.type    = cudaGraphCondTypeWhile;
    cp.conditional.size    = 1;
    cudaGraphNode_t loop   = nullptr;
    KSPN_CUDA(cudaGraphAddNode(&loop, graph, &dep, 1, &cp));
    cudaGraph_t     body = cp.conditional.phGraph_out[0];
    fio const       f{ ws.q0, ws.q1, &st->qn[0], &st->qn[1], &st->cur };
    cudaGraphNode_t bdep = t_add_kernel(body, nullptr, &k_t_push, vgrid, T_THREADS, g.fh, g.fc, g.bh, g.bc, und, scc_id, ws.indeg, ws.outdeg, f, st, h_out, h_in);
    bdep                 = t_add_kernel(body, bdep, &k_t_push_heavy, HEAVY_GRID, T_THREADS, g.fh, g.fc, g.bh, g.bc, und, scc_id, ws.indeg, ws.outdeg, f, st, (uint32_t const*)h_out, (uint32_t const*)h_in);
    t_add_kernel(body, bdep, &k_t_advance, 1, 1, st, h, 1);
    cudaGraphExec_t exec = nullptr;
    KSPN_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    ctx->trim.graph = graph;
    ctx->trim.exec  = exec;
  } catch (...) {
    cudaGraphDestroy(graph);
    throw;
  }
}

uint32_t
pv_result(kspn_context* ctx, unsigned nb, uint64_t* min_prod_out)
{
  auto&     ws   = ctx->ws;
  uint64_t* prod = ws.pivot;
  uint32_t* id   = reinterpret_cast<uint32_t*>(ws.pivot + 4096);
  k_pv_final<<<1, 32, 0, ctx->stream>>>(nb, prod, id);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  uint64_t hp = 0;
  uint32_t hi = 0;
  KSPN_CUDA(cudaMemcpyAsync(&hp, prod, sizeof(hp), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaMemcpyAsync(&hi, id, sizeof(hi), cudaMemcpyDeviceToHost, ctx->stream));
  KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
  if (min_prod_out) *min_prod_out = hp;
  return hi;
}

// Runs push levels from the queue in q0 (size qn) until no vertex is
// decided; returns the number decided by the levels.
template<int DIRS>
uint32_t
run_push_levels(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t qn)
{
  auto&    ws    = ctx->ws;
  uint32_t total = 0;
  uint32_t* qa = ws.q0, *qb = ws.q1;
  uint32_t const cap = g.n + 2;
  for (uint32_t level = 0; qn > 0; ++level) {
    if (level > cap) throw error{ KSPN_ERR_TIMEOUT, "trim: level cap exceeded" };
    KSPN_CUDA(cudaMemsetAsync(ws.ctr + CTR_Q1, 0, sizeof(uint32_t), ctx->stream));
    KSPN_CUDA(cudaMemsetAsync(ws.ctr + CTR_DECIDED, 0, sizeof(uint32_t), ctx->stream));
    KSPN_CUDA(cudaMemsetAsync(ws.ctr + CTR_TRIM_HEAVY, 0, 2 * sizeof(uint32_t), ctx->stream));
    uint64_t const e0 = ctx->h_ctr64[2];
    prof_start(ctx);
    k_trim_push<DIRS><<<stream_grid(qn), T_THREADS, 0, ctx->stream>>>(g.fh, g.fc, g.bh, g.bc, und, scc_id, ws.indeg, ws.outdeg, qa, qn, qb, ws.ctr + CTR_Q1, ws.ctr,
                                                                       reinterpret_cast<unsigned long long*>(ws.ctr64 + 2), ws.heavy, ws.heavy + ws.heavy_cap, ws.ctr + CTR_TRIM_HEAVY);
    k_push_heavy<<<HEAVY_GRID, T_THREADS, 0, ctx->stream>>>(g.fh, g.fc, g.bh, g.bc, und, scc_id, ws.indeg, ws.outdeg, ws.heavy, ws.heavy + ws.heavy_cap, ws.ctr + CTR_TRIM_HEAVY, qb, ws.ctr + CTR_Q1,
                                                            ws.ctr + CTR_DECIDED);
    prof_stop(ctx);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 2;
    read_counters(ctx);
    // per queued vertex and direction: queue entry + offset pair; per edge:
    // id + degree atomic; per decided vertex: id write + queue write
    int const ndir = (DIRS & 1) + ((DIRS >> 1) & 1);
    prof_add(ctx, 0, KSPN_KERNEL_TRIM, 20ull * ndir * qn + 8 * (ctx->h_ctr64[2] - e0) + 8ull * ctx->h_ctr[CTR_DECIDED]);
    qn = ctx->h_ctr[CTR_Q1];
    total += ctx->h_ctr[CTR_DECIDED];
    uint32_t* t = qa;
    qa          = qb;
    qb          = t;
  }
  // leave the workspace queues in their canonical order for the next user
  return total;
}

} // namespace

uint32_t
trim_1_first(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t* queue_out, uint32_t* queue_count_host, bool init_degrees)
{
  auto& ws = ctx->ws;
  zero_counters(ctx);
  unsigned const nb = pivot_candidates(g.n);
  prof_start(ctx);
  k_trim_first<<<nb, T_THREADS, 0, ctx->stream>>>(g.n, g.fh, g.bh, und, scc_id, init_degrees ? ws.indeg : nullptr, init_degrees ? ws.outdeg : nullptr, queue_out, ws.ctr, ws.pivot, reinterpret_cast<uint32_t*>(ws.pivot + 4096));
  prof_stop(ctx);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  uint64_t       prod  = 0;
  uint32_t const pivot = pv_result(ctx, nb, &prod);
  read_counters(ctx);
  {
    // both offset arrays streamed (8 B per vertex each), id + bitmap written,
    // live degrees written, trimmed vertices queued
    uint64_t const dec  = ctx->h_ctr[CTR_DECIDED];
    uint64_t const live = g.n - dec;
    prof_add(ctx, 0, KSPN_KERNEL_STREAM, 16ull * (g.n + 1) + 4ull * g.n + g.n / 8 + (init_degrees ? 8 * live : 0) + (queue_out ? 4 * dec : 0));
  }
  if (queue_count_host) *queue_count_host = ctx->h_ctr[CTR_Q0];
  ctx->h_ctr[CTR_AUX] = ctx->h_ctr[CTR_DECIDED];
  // no undecided vertex: the reference returns n (trim_1_local.hpp:21,44)
  return (prod == 0 || pivot == NONE) ? g.n : pivot;
}

unsigned
pivot_candidates(uint32_t n)
{
  // k_trim_first's grid, which is also the number of per-block pivot
  // candidates: one wave of resident blocks (blocks per SM x SMs), so no
  // partial last wave leaves SMs idle, or fewer blocks for a small graph
  static unsigned const wave = [] {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trim_first, T_THREADS, 0) != cudaSuccess || per_sm <= 0) per_sm = 4;
    return static_cast<unsigned>(std::min(sms * per_sm, static_cast<int>(PV_FINAL)));
  }();
  uint64_t const b = (static_cast<uint64_t>(n) + static_cast<uint64_t>(T_THREADS) * TF_ITEMS - 1) / (static_cast<uint64_t>(T_THREADS) * TF_ITEMS);
  return static_cast<unsigned>(b < wave ? (b ? b : 1) : wave);
}

// (the caller has zeroed ws.ctr; ids are not written: the resident
// launch that follows writes every vertex's id at its end)
void
trim_1_first_async(kspn_context* ctx, dgraph const& g, uint32_t* und)
{
  auto& ws = ctx->ws;
  prof_start(ctx);
  k_trim_first<<<pivot_candidates(g.n), T_THREADS, 0, ctx->stream>>>(g.n, g.fh, g.bh, und, nullptr, nullptr, nullptr, nullptr, ws.ctr, ws.pivot, reinterpret_cast<uint32_t*>(ws.pivot + 4096));
  prof_stop(ctx);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
}

uint32_t
trim_1_normal(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id)
{
  zero_counters(ctx);
  k_trim_normal<<<stream_grid(g.n), T_THREADS, 0, ctx->stream>>>(g.n, g.fh, g.fc, g.bh, g.bc, und, scc_id, ctx->ws.ctr);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  read_counters(ctx);
  return ctx->h_ctr[CTR_DECIDED];
}

// Full trim-1 fixpoint on the undecided sub-graph.  degrees_from_first:
// the live degrees and the seed queue (seed_count entries in q0) come from
// trim_1_first; otherwise they are counted here (pull) first.
uint32_t
trim_fixpoint(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, bool degrees_from_first, uint32_t seed_count)
{
  auto&    ws    = ctx->ws;
  uint32_t total = 0, qn = seed_count;
  if (!degrees_from_first && !ctx->prof) {
    // one graph launch: compact the undecided set, live degrees, seeds, and
    // a device-driven loop of push levels
    trim_state* hs = trim_state_host(ctx);
    std::memset(hs, 0, sizeof(trim_state));
    hs->cap = g.n + 2;
    KSPN_CUDA(cudaMemcpyAsync(trim_state_dev(ctx), hs, sizeof(trim_state), cudaMemcpyHostToDevice, ctx->stream));
    graph_key const key{ g.fh, g.fc, g.bh, g.bc, und, scc_id, ws.base, g.n, g.m };
    if (!ctx->trim.exec || !(ctx->trim.key == key)) {
      if (ctx->trim.exec) cudaGraphExecDestroy(ctx->trim.exec);
      if (ctx->trim.graph) cudaGraphDestroy(ctx->trim.graph);
      ctx->trim = {};
      build_trim_graph(ctx, g, und, scc_id);
      ctx->trim.key = key;
    }
    KSPN_CUDA(cudaGraphLaunch(ctx->trim.exec, ctx->stream));
    KSPN_CUDA(cudaMemcpyAsync(hs, trim_state_dev(ctx), sizeof(trim_state), cudaMemcpyDeviceToHost, ctx->stream));
    KSPN_CUDA(cudaStreamSynchronize(ctx->stream));
    if (hs->err) throw error{ KSPN_ERR_TIMEOUT, "trim: level cap exceeded" };
    ctx->launches += 5 + 3ull * hs->level;
    return hs->decided;
  }
  if (!degrees_from_first) {
    zero_counters(ctx);
    k_live_degrees<<<stream_grid(g.n), T_THREADS, 0, ctx->stream>>>(g.n, g.fh, g.fc, g.bh, g.bc, und, ws.indeg, ws.outdeg, ws.heavy, ws.ctr + CTR_TRIM_HEAVY + 3);
    k_live_heavy<<<HEAVY_GRID, T_THREADS, 0, ctx->stream>>>(g.fh, g.fc, g.bh, g.bc, und, ws.heavy, ws.ctr + CTR_TRIM_HEAVY + 3, ws.indeg, ws.outdeg);
    k_seed_dead<<<stream_grid(g.n), T_THREADS, 0, ctx->stream>>>(g.n, und, scc_id, ws.indeg, ws.outdeg, ws.q0, ws.ctr);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 3;
    read_counters(ctx);
    qn    = ctx->h_ctr[CTR_Q0];
    total = qn;
  }
  total += run_push_levels<3>(ctx, g, und, scc_id, qn);
  return total;
}

uint32_t
trim_exhaustive_first(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t* outdeg, uint32_t* indeg)
{
  auto&    ws    = ctx->ws;
  uint32_t total = 0;
  // every vertex starts undecided
  KSPN_CUDA(cudaMemsetAsync(und, 0xFF, (static_cast<size_t>(g.n) + 31) / 32 * 4, ctx->stream));
  KSPN_CUDA(cudaMemsetAsync(scc_id, 0xFF, static_cast<size_t>(g.n) * 4, ctx->stream));
  uint32_t* save_in = ws.indeg, *save_out = ws.outdeg;
  ws.indeg  = indeg;
  ws.outdeg = outdeg;
  try {
    // in-degree sweep: raw in-degree 0 decided, decrements along out-edges
    zero_counters(ctx);
    k_seed_raw<<<stream_grid(g.n), T_THREADS, 0, ctx->stream>>>(g.n, g.bh, und, scc_id, indeg, ws.q0, ws.ctr);
    KSPN_CHECK_LAUNCH();
    read_counters(ctx);
    total += ctx->h_ctr[CTR_DECIDED];
    total += run_push_levels<1>(ctx, g, und, scc_id, ctx->h_ctr[CTR_Q0]);
    // out-degree sweep over the survivors: raw out-degree, decrements along in-edges
    zero_counters(ctx);
    k_seed_raw<<<stream_grid(g.n), T_THREADS, 0, ctx->stream>>>(g.n, g.fh, und, scc_id, outdeg, ws.q0, ws.ctr);
    KSPN_CHECK_LAUNCH();
    read_counters(ctx);
    total += ctx->h_ctr[CTR_DECIDED];
    total += run_push_levels<2>(ctx, g, und, scc_id, ctx->h_ctr[CTR_Q0]);
    ctx->launches += 2;
  } catch (...) {
    ws.indeg  = save_in;
    ws.outdeg = save_out;
    throw;
  }
  ws.indeg  = save_in;
  ws.outdeg = save_out;
  return total;
}

uint32_t
trim_2(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id)
{
  auto& ws = ctx->ws;
  zero_counters(ctx);
  k_unique_neighbour<<<stream_grid(g.n), T_THREADS, 0, ctx->stream>>>(g.n, g.fh, g.fc, g.bh, g.bc, und, ws.indeg, ws.outdeg);
  k_trim2_decide<<<stream_grid(g.n), T_THREADS, 0, ctx->stream>>>(g.n, ws.indeg, ws.outdeg, und, scc_id, ws.ctr);
  KSPN_CHECK_LAUNCH();
  ctx->launches += 2;
  read_counters(ctx);
  return ctx->h_ctr[CTR_DECIDED];
}

// argmax over undecided v of live outdeg*indeg, lowest id on ties; n if no
// vertex is undecided.  Degrees must be current (after a trim fixpoint).
uint32_t
select_pivot_live(kspn_context* ctx, dgraph const& g, uint32_t const* und)
{
  auto&          ws = ctx->ws;
  unsigned const nb = stream_grid(g.n);
  k_pivot_live<<<nb, T_THREADS, 0, ctx->stream>>>(g.n, und, ws.indeg, ws.outdeg, ws.pivot, reinterpret_cast<uint32_t*>(ws.pivot + 4096));
  KSPN_CHECK_LAUNCH();
  ctx->launches += 1;
  uint64_t       prod = 0;
  uint32_t const p    = pv_result(ctx, nb, &prod);
  return (prod == 0 || p == NONE) ? g.n : p;
}

uint32_t
count_undecided(kspn_context* ctx, uint32_t n, uint32_t const* und)
{
  uint32_t const words = (n + 31) / 32;
  zero_counters(ctx);
  if (words) {
    k_popcount<<<stream_grid(words), T_THREADS, 0, ctx->stream>>>(words, n, und, ctx->ws.ctr + CTR_AUX);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 1;
  }
  read_counters(ctx);
  return ctx->h_ctr[CTR_AUX];
}

} // namespace kspn
