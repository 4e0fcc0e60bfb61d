// Internal declarations shared by the kspn CUDA sources (not installed).
//
// Device data layout (one graph, one GPU):
//   fw_head u64[n+1], fw_csr u32[m]   out-edges (CSR)
//   bw_head u64[n+1], bw_csr u32[m]   in-edges  (transpose, "CSC")
//   und     u32[ceil(n/32)]           bit v%32 of word v/32 set = v undecided;
//                                     byte-identical to the reference's u64
//                                     bitset words on a little-endian host
//   scc_id  u32[n]                    member id of v's component, UNDECIDED
//                                     (0xFFFFFFFF) while v is undecided
#pragma once

#include "../../include/kspn.h"

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>
#include <utility>

namespace kspn {

constexpr uint32_t UNDECIDED = 0xFFFFFFFFu;

// ---------------------------------------------------------------- errors
struct error
{
  int         code;
  std::string what;
};

#define KSPN_CUDA(call)                                                                                  \
  do {                                                                                                   \
    cudaError_t const e_ = (call);                                                                       \
    if (e_ != cudaSuccess) throw ::kspn::error{ KSPN_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_) }; \
  } while (0)

#define KSPN_CHECK_LAUNCH() KSPN_CUDA(cudaGetLastError())

inline unsigned
div_up(uint64_t a, uint64_t b)
{
  return static_cast<unsigned>((a + b - 1) / b);
}

// ---------------------------------------------------------------- device helpers
__device__ __forceinline__ bool
bit_get(uint32_t const* bm, uint32_t v)
{
  return (bm[v >> 5] >> (v & 31)) & 1u;
}

// Clears bit v; true iff this call cleared it (exactly one caller wins).
__device__ __forceinline__ bool
bit_take(uint32_t* bm, uint32_t v)
{
  uint32_t const mask = 1u << (v & 31);
  return (atomicAnd(bm + (v >> 5), ~mask) & mask) != 0;
}

// Sets bit v without waiting for the old word (no result: the atomic is
// issued and the thread goes on).
__device__ __forceinline__ void
bit_set_async(uint32_t* bm, uint32_t v)
{
  atomicOr(bm + (v >> 5), 1u << (v & 31));
}

// Sets bit v; true iff this call set it.
__device__ __forceinline__ bool
bit_claim(uint32_t* bm, uint32_t v)
{
  uint32_t const mask = 1u << (v & 31);
  return (atomicOr(bm + (v >> 5), mask) & mask) == 0;
}

// GPU-scope acquire load (coherent across SMs, never hoisted by the
// compiler): polls of words other blocks update inside one launch.
__device__ __forceinline__ uint32_t
ld_acquire(uint32_t const* p)
{
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned
lane_id()
{
  return threadIdx.x & 31u;
}

// Warp-aggregated append: every lane of the (fully active) warp calls it;
// lanes with pred append v.  One atomic per warp.
__device__ __forceinline__ void
warp_push(bool pred, uint32_t v, uint32_t* queue, uint32_t* count)
{
  unsigned const ballot = __ballot_sync(0xFFFFFFFFu, pred);
  if (!ballot) return;
  unsigned const lane   = lane_id();
  unsigned const leader = __ffs(ballot) - 1;
  uint32_t       base   = 0;
  if (lane == leader) base = atomicAdd(count, static_cast<uint32_t>(__popc(ballot)));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  if (pred) queue[base + __popc(ballot & ((1u << lane) - 1u))] = v;
}

// Same, for lanes that may be inactive (uses the active mask).
__device__ __forceinline__ void
warp_push_active(uint32_t v, uint32_t* queue, uint32_t* count)
{
  unsigned const mask   = __activemask();
  unsigned const lane   = lane_id();
  unsigned const leader = __ffs(mask) - 1;
  uint32_t       base   = 0;
  if (lane == leader) base = atomicAdd(count, static_cast<uint32_t>(__popc(mask)));
  base = __shfl_sync(mask, base, leader);
  queue[base + __popc(mask & ((1u << lane) - 1u))] = v;
}

// ---------------------------------------------------------------- heavy rows
// A row longer than HEAVY_ROW edges is never walked by one thread or one
// warp alone (on skewed graphs one such row would serialise a whole
// phase): it is listed, and every warp of the grid takes slices of
// HEAVY_SLICE edges of every listed row.
constexpr uint32_t HEAVY_ROW   = 2048;
constexpr uint32_t HEAVY_SLICE = 1024;
// Worklist items that the passes of every warp of the persistent search can
// push around its switch to exact takes: two passes of at most 32 lanes x 8
// finds for each of AW_GRID_MAX blocks x 8 warps.
constexpr int    AW_GRID_MAX = 1024;
constexpr size_t AW_STALE    = size_t(2) * AW_GRID_MAX * 8 * 32 * 8;

// Entries of one heavy list: a list holds each vertex at most once per
// direction, and only vertices with a row longer than HEAVY_ROW (at most
// m / HEAVY_ROW per direction).
inline uint64_t
heavy_capacity(uint32_t n, uint64_t m)
{
  uint64_t const c = 2 * (m / HEAVY_ROW);
  return (c < 2ull * n ? c : 2ull * n) + 32;
}

// fn(i, v, b, e) for the slices of the listed rows that fall to this warp:
// the slices of the whole list are numbered in list order (entry i's slices
// follow entry i-1's) and global slice g goes to warp g mod W of the grid's
// W warps; [b, e) is one slice of v's row in `head`.  HEAVY_ONLY: rows of at
// most HEAVY_ROW entries are skipped (their owner walks them).  All lanes of
// every warp call it; fn is called warp-uniformly.  A warp reads the list
// HS_BATCHES x 32 entries at a time (independent loads), numbers the
// batch's slices with a warp scan and finds the entry of each slice it owns
// with a ballot, so its cost is count / 32 scan steps plus its own slices.
// Entries are read through L2 (the list was written by other blocks of the
// same launch).
constexpr uint32_t HS_BATCHES = 2;

template<bool HEAVY_ONLY = false, class F>
__device__ __forceinline__ void
heavy_slices(uint32_t const* list, uint32_t count, uint64_t const* __restrict__ head, F&& fn)
{
  unsigned const lane = threadIdx.x & 31u;
  uint32_t const W    = gridDim.x * (blockDim.x >> 5);
  // offset of this warp's next slice from the start of the current batch
  uint64_t nxt = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (uint32_t base = 0; base < count; base += 32 * HS_BATCHES) {
    uint32_t v[HS_BATCHES];
    uint64_t b[HS_BATCHES], e[HS_BATCHES];
#pragma unroll
    for (uint32_t k = 0; k < HS_BATCHES; ++k) {
      uint32_t const i = base + 32 * k + lane;
      v[k]             = i < count ? __ldcg(list + i) : 0u;
    }
#pragma unroll
    for (uint32_t k = 0; k < HS_BATCHES; ++k) {
      bool const in = base + 32 * k + lane < count;
      b[k]          = in ? head[v[k]] : 0ull;
      e[k]          = in ? head[v[k] + 1] : 0ull;
    }
#pragma unroll
    for (uint32_t k = 0; k < HS_BATCHES; ++k) {
      uint64_t const len = e[k] - b[k];
      uint32_t const ns  = HEAVY_ONLY && len <= HEAVY_ROW ? 0u : static_cast<uint32_t>((len + HEAVY_SLICE - 1) / HEAVY_SLICE);
      uint32_t       inc = ns; // inclusive scan of the batch's slice counts
#pragma unroll
      for (unsigned sh = 1; sh < 32; sh <<= 1) {
        uint32_t const t = __shfl_up_sync(0xFFFFFFFFu, inc, sh);
        if (lane >= sh) inc += t;
      }
      uint32_t const total = __shfl_sync(0xFFFFFFFFu, inc, 31);
      for (; nxt < total; nxt += W) {
        uint32_t const o  = static_cast<uint32_t>(nxt);
        unsigned const j  = __popc(__ballot_sync(0xFFFFFFFFu, inc <= o)); // entry holding slice o
        uint32_t const vj = __shfl_sync(0xFFFFFFFFu, v[k], j);
        uint64_t const bj = __shfl_sync(0xFFFFFFFFu, b[k], j), ej = __shfl_sync(0xFFFFFFFFu, e[k], j);
        uint32_t const s  = o - __shfl_sync(0xFFFFFFFFu, inc - ns, j);
        uint64_t const sb = bj + static_cast<uint64_t>(s) * HEAVY_SLICE;
        fn(base + 32 * k + j, vj, sb, sb + HEAVY_SLICE < ej ? sb + HEAVY_SLICE : ej);
      }
      nxt -= total;
    }
  }
}

// Block-aggregated append: pushes collected in shared memory during a tile (or sweep step)
// are reserved in the global queue with ONE atomic per block and copied out
// coalesced (a per-warp atomic on one counter serialises in L2 when a level
// discovers millions of vertices).
struct block_queue
{
  uint32_t* s_buf; // EX_TILE entries
  uint32_t* s_n;
  __device__ __forceinline__ void push(bool pred, uint32_t v)
  {
    unsigned const ballot = __ballot_sync(0xFFFFFFFFu, pred);
    if (!ballot) return;
    unsigned const lane   = threadIdx.x & 31u;
    unsigned const leader = __ffs(ballot) - 1;
    uint32_t       base   = 0;
    if (lane == leader) base = atomicAdd(s_n, static_cast<uint32_t>(__popc(ballot)));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (pred) s_buf[base + __popc(ballot & ((1u << lane) - 1u))] = v;
  }
  // all threads; leaves s_n == 0 for the next tile
  __device__ __forceinline__ void flush(uint32_t* queue, uint32_t* count, uint32_t* s_base)
  {
    __syncthreads();
    uint32_t const cnt = *s_n;
    if (cnt) {
      if (threadIdx.x == 0) *s_base = atomicAdd(count, cnt);
      __syncthreads();
      uint32_t const b = *s_base;
      for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) queue[b + i] = s_buf[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) *s_n = 0;
    __syncthreads();
  }
};

// Dense vertex sweeps push through a block_queue of DENSE_BUF entries and
// flush when fewer than one step's worth of slots is left.
constexpr int DENSE_BUF = 2048;

__device__ __forceinline__ uint32_t
rotr32(uint32_t x, int r)
{
  return __funnelshift_r(x, x, r & 31);
}
__device__ __forceinline__ uint32_t
rotl32(uint32_t x, int r)
{
  return __funnelshift_l(x, x, r & 31);
}

// ---------------------------------------------------------------- graph + context
struct dgraph
{
  uint32_t        n  = 0;
  uint64_t        m  = 0;
  uint64_t const* fh = nullptr; // fw head
  uint32_t const* fc = nullptr; // fw csr
  uint64_t const* bh = nullptr; // bw head
  uint32_t const* bc = nullptr; // bw csr
};

// Device counters (one cache line each would be nicer; they are few).
enum ctr_slot : int
{
  CTR_Q0 = 0,   // queue 0 size
  CTR_Q1,       // queue 1 size
  CTR_DECIDED,  // vertices decided by the running phase
  CTR_AUX,      // phase-specific
  CTR_ERR,      // error word (bounds checks, caps)
  CTR_COUNT = 16, // slots 5.. are phase-specific (8: expansion tile count)
  CTR_RES_HEAVY  = 5, // residual: heavy rows listed by k_res_hook
  CTR_TRIM_HEAVY = 6, // trim push levels (host-driven): heavy out-rows at 6, in-rows at 7; live counts: 9
  CTR_PV_TICKET = 15 // trim_1_first: blocks finished (the last one reduces the pivot)
};

// ws.pivot holds per-block (product, id) pivot candidates: products at
// [0, 4096), ids as u32 from ws.pivot + 4096.  trim_1_first's last block
// leaves the grid-wide best in slot PV_FINAL of both.
constexpr uint32_t PV_FINAL = 4095;

// Scratch owned by a context, sized for the largest graph seen.
struct workspace
{
  uint32_t n_cap = 0;
  uint64_t m_cap = 0;
  void*    base  = nullptr;
  size_t   bytes = 0;

  uint32_t* q0       = nullptr; // n
  uint32_t* q1       = nullptr; // n
  uint32_t* vis_a    = nullptr; // bitmap
  uint32_t* vis_b    = nullptr; // bitmap
  uint32_t* mark     = nullptr; // bitmap
  uint32_t* fresh    = nullptr; // bitmap: vertices found by the last bottom-up sweep (FW search)
  uint32_t* fresh_bw = nullptr; // the same for the BW search of the persistent FW-BW
  uint32_t* cand_bw  = nullptr; // bitmap: BW candidates of a joint worklist search (FW and BW at once)
  uint32_t* label    = nullptr; // n
  uint32_t* indeg    = nullptr; // n
  uint32_t* outdeg   = nullptr; // n
  uint64_t* prefix   = nullptr; // n+1 (u64 scan output)
  uint64_t* prefix2  = nullptr; // n+1 (second frontier of the persistent FW-BW)
  uint64_t* blocks   = nullptr; // scan partials
  uint32_t* ctr      = nullptr; // CTR_COUNT
  uint64_t* ctr64    = nullptr; // 8 (64-bit counters)
  uint64_t* pivot    = nullptr; // per-block pivot keys (4096 u64 products + 4096 u32 ids)
  uint32_t* tile_start  = nullptr; // m / 2048 + 4 (frontier expansion)
  uint32_t* tile_start2 = nullptr; // m / 2048 + 4 (second frontier of the persistent FW-BW)
  // the BW search's frontier pair in the persistent FW-BW (FW and BW run side by side)
  uint32_t* q2          = nullptr; // n
  uint32_t* q3          = nullptr; // n
  uint64_t* prefix3     = nullptr; // n+1
  uint64_t* prefix4     = nullptr; // n+1
  uint32_t* tile_start3 = nullptr; // m / 2048 + 4
  uint32_t* tile_start4 = nullptr; // m / 2048 + 4
  uint32_t* tile_zero   = nullptr; // m / 2048 + 4 zeros: tile starts of a one-vertex frontier
  uint32_t* seed_q      = nullptr; // 4: the pivot as a one-vertex frontier
  uint64_t* seed_prefix = nullptr; // 4
  void*     gbar        = nullptr; // 4 KiB: grid barrier of the persistent FW-BW at 0, worklist counters at 1024 (zeroed at creation)
  void*     aw          = nullptr; // aw_entries u64: worklist of the asynchronous search tail (zeroed at creation, zero outside a phase)
  size_t    aw_entries  = 0;       // 4 (n + 2) + 2 AW_STALE vertex items (FW and BW at once, duplicate pushes) + 4 m / HEAVY_SLICE + 128 row-slice items
  void*     rstate      = nullptr; // 4 KiB device control blocks (FW-BW at 0, trim at 512, search stamps at 2048)
  uint32_t* heavy       = nullptr; // 4 heavy lists of heavy_cap entries (persistent FW-BW: trim seed, two trim push levels, cut bottom-up rows)
  uint64_t  heavy_cap   = 0;
  uint32_t* cutmap      = nullptr; // bitmaps: vertices on a cut list, FW search then BW search (2 x words; zero outside a search)
  // owned graph storage (host inputs, or a CSC built on device)
  uint64_t* g_fh = nullptr;
  uint32_t* g_fc = nullptr;
  uint64_t* g_bh = nullptr;
  uint32_t* g_bc = nullptr;
  uint32_t* g_out = nullptr;
  uint32_t* und   = nullptr; // bitmap
  size_t    g_bytes = 0;
  void*     g_base  = nullptr;
};

} // namespace kspn

namespace kspn {
// Identity of a cached CUDA graph: the buffers its kernel arguments name.
struct graph_key
{
  void const* a[7] = {};
  uint32_t    n    = 0;
  uint64_t    m    = 0;
  graph_key() = default;
  graph_key(void const* p0, void const* p1, void const* p2, void const* p3, void const* p4, void const* p5, void const* p6, uint32_t n_, uint64_t m_)
    : a{ p0, p1, p2, p3, p4, p5, p6 }
    , n(n_)
    , m(m_)
  {
  }
  bool operator==(graph_key const& o) const
  {
    for (int i = 0; i < 7; ++i)
      if (a[i] != o.a[i]) return false;
    return n == o.n && m == o.m;
  }
};
// A device buffer owned by a context, grown on demand and reused by later
// calls (host-pointer calls, graph construction scratch).
struct dev_buffer
{
  void*  p     = nullptr;
  size_t bytes = 0;
};
enum buffer_slot : int
{
  BUF_HOST_GRAPH = 0, // device copy of a host graph + output (kspn_scc)
  BUF_BUILD      = 1, // radix-sort scratch (transpose, build_csr)
  BUF_TRANSPOSE  = 2, // transpose built for kspn_scc_device without bw
  BUF_GEN        = 3, // generator scratch (RGG points and cells)
  BUF_SHARD      = 4, // counters of the sharded steps (shard.cu)
  BUF_SEEDS      = 5, // learned seed order of the label searches: score bucket per vertex (label.cu)
  BUF_UNION      = 6, // the batch mix as one graph (batch_union.cu)
  BUF_COUNT      = 7
};

struct cached_graph
{
  graph_key       key;
  cudaGraph_t     graph = nullptr;
  cudaGraphExec_t exec  = nullptr;
};
} // namespace kspn

namespace kspn {
struct batch_cache; // batched path: plan buffers and the captured call (batch.cu)
}

struct kspn_context
{
  int                device     = 0;
  cudaStream_t       stream     = nullptr;
  bool               own_stream = false;
  kspn::workspace    ws;
  uint32_t*          h_ctr      = nullptr; // pinned mirror of ws.ctr
  uint64_t*          h_ctr64    = nullptr;
  int                rotation   = 0; // label-search calls made by this context
  cudaEvent_t        ev[KSPN_PHASES + 2] = {};
  uint64_t           launches   = 0;
  uint64_t           td_edges   = 0; // top-down reachability edges (host tally; the rest count on device)
  std::string        last_error;
  // kernel-class timing (kspn_options.profile): two event pairs in flight
  kspn_stats*        prof       = nullptr;
  cudaEvent_t        pe[4]      = {};
  void*              h_state    = nullptr; // pinned 4 KiB mirror of ws.rstate
  unsigned           search_grid = 0;      // blocks of the persistent FW-BW launch
  unsigned           resume_grid = 0;      // blocks of its resume launch (the worklist phase)
  unsigned           bar_grid    = 0;      // grid of the last launch on the workspace's grid barrier
  bool               union_route = false;  // the pipeline runs on a batch mix as one graph: no second FW-BW
  alignas(16) unsigned char fwbw_last[1024] = {}; // arguments of the last persistent FW-BW launch (a resume launch reuses them)
  cudaEvent_t        fwbw_after  = nullptr; // event the last launch records after its kernel (re-recorded after a resume)
  float*             pivot_model = nullptr; // device copy of the pivot MLP (kspn_set_pivot_model)
  kspn::cached_graph trim;                 // one-launch trim fixpoint graph
  kspn::batch_cache* batch      = nullptr;  // batched path (kspn_scc_batched)
  kspn::dev_buffer   bufs[kspn::BUF_COUNT];
  cudaStream_t       copy_stream = nullptr; // host-graph upload (upload_transpose)
  cudaEvent_t        copy_ev     = nullptr;
};

namespace kspn {

// Kernel-class timing: prof_start/prof_stop bracket launches on the stream;
// prof_add (after the stream was synchronised) books the elapsed time and
// the algorithmic bytes of the bracketed work.
inline void
prof_start(kspn_context* ctx, int pair = 0)
{
  if (ctx->prof) cudaEventRecord(ctx->pe[2 * pair], ctx->stream);
}
inline void
prof_stop(kspn_context* ctx, int pair = 0)
{
  if (ctx->prof) cudaEventRecord(ctx->pe[2 * pair + 1], ctx->stream);
}
inline float
prof_add(kspn_context* ctx, int pair, int cls, uint64_t bytes, uint64_t calls = 1)
{
  if (!ctx->prof) return 0.f;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, ctx->pe[2 * pair], ctx->pe[2 * pair + 1]) != cudaSuccess) {
    cudaGetLastError();
    return 0.f;
  }
  ctx->prof->kernel_ms[cls] += ms;
  ctx->prof->kernel_bytes[cls] += bytes;
  ctx->prof->kernel_calls[cls] += calls;
  return ms;
}

// workspace / context helpers (context.cu)
void  ensure_workspace(kspn_context* ctx, uint32_t n, uint64_t m);
void* context_buffer(kspn_context* ctx, int slot, size_t bytes); // grown on demand, kept
void read_counters(kspn_context* ctx); // D2H of ws.ctr / ws.ctr64 + stream sync
void zero_counters(kspn_context* ctx);
int  fail(kspn_context* ctx, error const& e);

// Runs an entry point's body: KSPN_OK, or the status of the error it threw
// (detail kept for kspn_last_error).  No exception crosses the C ABI.
template<class F>
int
run_guarded(kspn_context* ctx, F&& body)
{
  try {
    body();
    return KSPN_OK;
  } catch (error const& e) {
    return fail(ctx, e);
  } catch (...) {
    return fail(ctx, error{ KSPN_ERR_INTERNAL, "unexpected exception" });
  }
}

// trim.cu
// reach.cu: the resident start of the FAST pipeline -- FW-BW from
// trim_1_first's pivot (left on the device) and the trim-1 fixpoint in one
// persistent launch, which then writes every vertex's id (trim_1_first_async
// writes none); no host sync; results after the stream synchronised.
struct resident_result
{
  uint32_t pivot = 0, fwbw_decided = 0, trim_decided = 0, trim_levels = 0, und_left = 0;
  double   fwbw_share     = 1.0;   // FW-BW's share of the launch's device time
  bool     pivot_rejected = false;
  bool     resumed        = false; // the worklist phase ran in a resume launch (after one more host round trip) // the pivot model rejected trim_1_first's pivot: the launch ended after its first level
};
bool            resident_fits(dgraph const& g);
void            fw_bw_trim_async(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, kspn_options const& opt, kspn_stats* st, cudaEvent_t after_kernel);
resident_result fw_bw_trim_result(kspn_context* ctx, dgraph const& g, kspn_options const& opt, kspn_stats* st);
// FW-BW from `pivot` and the trim-1 fixpoint of the remainder in one
// resident launch, ids written as decided; (FW-BW decided, trim decided)
std::pair<uint32_t, uint32_t> fw_bw_trim(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t pivot, kspn_options const& opt, kspn_stats* st);

uint32_t trim_1_first(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t* queue_out, uint32_t* queue_count_host, bool init_degrees);
void     trim_1_first_async(kspn_context* ctx, dgraph const& g, uint32_t* und); // ws.ctr zeroed by the caller; writes no ids; no host sync: decided in ws.ctr, pivot in PV_FINAL
uint32_t trim_1_normal(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id);
uint32_t trim_fixpoint(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, bool degrees_from_first, uint32_t seed_count);
uint32_t trim_exhaustive_first(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t* outdeg, uint32_t* indeg);
uint32_t trim_2(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id);
uint32_t select_pivot_live(kspn_context* ctx, dgraph const& g, uint32_t const* und);
uint32_t union_build(kspn_context* ctx, uint32_t count, uint64_t n, uint64_t m, uint64_t const* vtx_off, uint64_t const* fh_in, uint32_t const* fc_in, uint64_t const* bh_in,
                     uint32_t const* bc_in, uint64_t* fh, uint32_t* fc, uint64_t* bh, uint32_t* bc, uint32_t* piv, uint32_t* p_dev, unsigned long long* maxprod_dev,
                     unsigned long long* maxprod);
void     union_rename(kspn_context* ctx, uint32_t count, uint64_t n, uint64_t const* vtx_off, uint32_t const* uid, uint32_t* scc_id);
void     scc_batched(kspn_context* ctx, uint32_t G, uint64_t N, uint64_t const* vtx_off, uint64_t const* fh, uint32_t const* fc, uint64_t const* bh, uint32_t const* bc, uint32_t* scc_id,
                     kspn_batch_options const& opt, kspn_batch_stats* st);
void     batch_release(kspn_context* ctx);
void     manifest_read(char const* path, kspn_manifest* out);
void     manifest_load(kspn_context* ctx, kspn_manifest const& mf, uint64_t* fh, uint32_t* fc, uint64_t* bh, uint32_t* bc);
void     manifest_write(char const* dir, char const* name, uint32_t n, uint64_t m, uint64_t const* fh, uint32_t const* fc, uint64_t const* bh, uint32_t const* bc, uint32_t head_bytes,
                        uint32_t csr_bytes, int big_endian, int self_loops, int duplicate_edges);
void     batch_shape(uint32_t count, uint64_t seed, uint32_t log2_min, uint32_t log2_max, float deg_min, float deg_max, uint32_t* n_out, uint64_t* draws_out);
void     gen_batch(kspn_context* ctx, uint32_t count, uint64_t seed, uint64_t const* vtx_off, uint64_t const* draw_off, uint32_t const* ids, uint64_t total_draws, uint32_t* src, uint32_t* dst);
void     batch_localize(kspn_context* ctx, uint32_t count, uint64_t N, uint64_t const* vtx_off, uint64_t const* head, uint32_t* csr);
// trim.cu: k_trim_first's grid = the number of per-block pivot candidates
unsigned pivot_candidates(uint32_t n);
// mlp.cu: the learned pivot model (KSPN_MLP_PARAMS FP32 parameters)
void mlp_features(kspn_context* ctx, dgraph const& g, uint32_t count, uint32_t const* vs, float* feat);
void mlp_forward(kspn_context* ctx, uint32_t count, float const* feat, float const* params, float* out);
void mlp_grad(kspn_context* ctx, uint32_t count, float const* feat, float const* y, float const* params, float* grad, float* loss);
void mlp_adam(kspn_context* ctx, float* params, float const* grad, float* m, float* v, float lr, int step);
void learned_pivot(kspn_context* ctx, dgraph const& g, float const* params, bool check = true);
// residual.cu: Tarjan per weakly connected undecided piece that fits a warp's
// shared memory; returns vertices decided, *pieces_left = pieces left over
uint32_t residual(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t* pieces_left);
uint32_t count_undecided(kspn_context* ctx, uint32_t n, uint32_t const* und);

// reach.cu
size_t reach_state_bytes();
void   release_graphs(kspn_context* ctx);
// min_ids: name the SCC after its smallest member (else the pivot, as the reference does)
uint32_t fw_bw(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, uint32_t pivot, kspn_options const& opt, kspn_stats* st, bool min_ids);

// label.cu
uint32_t label_search(kspn_context* ctx, dgraph const& g, uint32_t* und, uint32_t* scc_id, int rotation, kspn_options const& opt, kspn_stats* st);

// canon.cu
// members: every id is a member of its own class (pipeline output); else
// arbitrary ids < n (normalise_scc_id semantics).
void canonicalise(kspn_context* ctx, uint32_t n, uint32_t* scc_id, uint32_t* scratch, bool members);

// csr.cu
void     transpose(kspn_context* ctx, uint32_t n, uint64_t m, uint64_t const* fh, uint32_t const* fc, uint64_t* bh, uint32_t* bc, uint32_t* scratch_n);
// Upload of a host CSR in chunks of `chunk` edges (0: UPLOAD_CHUNK) on the
// context's copy stream, with the CSC built on the context's stream while
// later chunks are still in flight: each arrived chunk's (target, source)
// pairs are radix-sorted, every entry gets its offset inside its CSC row
// (entries of earlier chunks first, so rows stay ascending), and after the
// last chunk one scan gives the heads and one pass places the entries.
// Leaves (dfh, dfc) = the host CSR and (dbh, dbc) = the same CSC as
// transpose(); work queued on the context's stream sees all of it.
constexpr uint64_t UPLOAD_CHUNK = 8ull << 20;
void     upload_transpose(kspn_context* ctx, uint32_t n, uint64_t m, uint64_t const* h_fh, uint32_t const* h_fc, uint64_t* dfh, uint32_t* dfc, uint64_t* dbh, uint32_t* dbc, uint64_t chunk);
uint64_t build_csr(kspn_context* ctx, uint32_t n, uint64_t m_raw, uint32_t* src, uint32_t* dst, uint64_t* head, uint32_t* csr);
void     validate(kspn_context* ctx, dgraph const& g);

// gen.cu
void gen_gnm(kspn_context* ctx, uint32_t n, uint64_t draws, uint64_t seed, uint32_t* src, uint32_t* dst);
void gen_rmat(kspn_context* ctx, int scale, uint64_t draws, uint64_t seed, uint64_t ta, uint64_t tab, uint64_t tabc, int do_perm, uint32_t* src, uint32_t* dst);
// edge count; the edges are written when src is given and count <= cap
uint64_t gen_rgg(kspn_context* ctx, uint32_t n, uint64_t seed, uint32_t g, uint64_t r2, uint32_t* src, uint32_t* dst, uint64_t cap);

} // namespace kspn
