/*
 * kspn -- strongly connected components of a directed graph on one NVIDIA
 * B200, as a drop-in for the `scc` entry point of rawbby/KaSpan.
 *
 * C ABI: plain pointers and sizes, no exceptions cross it, every entry point
 * returns a status (KSPN_OK or a KSPN_ERR_* code, see kspn_strerror).
 *
 * Graph layout everywhere: n vertices with u32 ids; forward CSR
 * fw_head[n+1] (u64 offsets) / fw_csr[m] (u32 neighbour ids) and its
 * transpose bw_head / bw_csr.  This is the reference's
 * bidi_graph_part_view at one rank built with KASPAN_INDEX64
 * (kaspan/graph/bidi_graph_part.hpp:12-28, kaspan/graph/base.hpp:18-28).
 * Duplicate edges and self-loops are allowed, as in the reference.
 *
 * Output contract: scc_id[v] is the MINIMUM vertex id of v's strongly
 * connected component.  The reference promises "some member of the
 * component" (tool/bench_kaspan/src/main.cpp:74-80); the minimum member is
 * one, and it is what kaspan::normalise_scc_id (kaspan/test/normalise_scc.hpp:10-25)
 * produces, so outputs compare bit for bit after that relabel.
 *
 * Vertex-state bitsets in the phase-level entry points use the reference's
 * bits layout: ceil(n/64) u64 words, bit v%64 of word v/64 set = vertex v
 * undecided (kaspan/memory/bits_ops.hpp).
 */
#ifndef KSPN_H
#define KSPN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define KSPN_OK 0
#define KSPN_ERR_INVALID_ARGUMENT 1 /* null pointer, bad size, unknown option */
#define KSPN_ERR_INVALID_GRAPH 2    /* offsets not monotone / out of range, id >= n */
#define KSPN_ERR_OOM 3              /* device or pinned allocation failed */
#define KSPN_ERR_TIMEOUT 4          /* an iteration cap or wait limit was hit */
#define KSPN_ERR_CUDA 5             /* a CUDA runtime call failed */
#define KSPN_ERR_NO_DEVICE 6        /* no usable CUDA device */
#define KSPN_ERR_INTERNAL 7         /* a device-side consistency check failed */

#define KSPN_UNDECIDED 0xFFFFFFFFu /* reference: scc_id_undecided, kaspan/graph/base.hpp:135 */

/* ---------------------------------------------------------------- options */
#define KSPN_PIPELINE_FAST 0      /* trim_1_first, pivot FW-BW, then rounds of trim fixpoint / trim-2 / label search */
#define KSPN_PIPELINE_REFERENCE 1 /* the phase order of kaspan::scc (kaspan/scc/scc.hpp:21-87) */
/* The reference's variants (kaspan/scc/variant/*.hpp), phase order at one
 * rank, where the n - n/P threshold of the residual variants is 0 (so their
 * FW-BW / colouring blocks do not run).  The residual step is the device
 * finish (kspn_residual); pieces too large for it, if any, are finished by
 * label rounds.  Every pipeline yields the same partition. */
#define KSPN_PIPELINE_HPC_LIKE 2               /* scc_hpc_like.hpp: trim_1_first, FW-BW, label rounds */
#define KSPN_PIPELINE_HPC_TRIM_EX 3            /* scc_hpc_trim_ex.hpp: exhaustive trim, degree pivot, FW-BW, label rounds */
#define KSPN_PIPELINE_ISPAN_LIKE 4             /* scc_ispan_like.hpp: trim_1_first, FW-BW, trim_1_normal x2, residual */
#define KSPN_PIPELINE_TRIM_EX 5                /* scc_trim_ex.hpp: exhaustive trim, degree pivot, FW-BW, trim, {label, trim} */
#define KSPN_PIPELINE_TRIM_EX_LIGHT_RESIDUAL 6 /* scc_trim_ex_light_residual.hpp: exhaustive trim, trim, residual */
#define KSPN_PIPELINE_TRIM_EX_RESIDUAL 7       /* scc_trim_ex_residual.hpp: exhaustive trim, residual */
#define KSPN_PIPELINE_COUNT 8

typedef struct kspn_options
{
  uint32_t struct_size;     /* sizeof(kspn_options); filled by kspn_options_default */
  int32_t  pipeline;        /* KSPN_PIPELINE_* */
  int32_t  trim2;           /* 1: run the exact size-2 trim in the fast pipeline */
  int32_t  validate;        /* 1: check the CSR (monotone offsets, ids < n) before running */
  uint32_t bu_enter_div;    /* reachability: go bottom-up when frontier > undecided / this */
  uint32_t bu_leave_div;    /* ... and back top-down when frontier < undecided / this */
  uint32_t max_levels;      /* cap on reachability levels per search (0 = n + 2) */
  uint32_t max_label_iters; /* cap on label-propagation sweeps per search (0 = n + 2) */
  uint32_t max_rounds;      /* cap on pipeline rounds (0 = n + 2) */
  int32_t  profile;         /* 1: time kernel classes with CUDA events (kspn_stats.kernel_*) */
  int32_t  trace;           /* 1: timestamp the phases of the persistent searches (kspn_stats.search_*) */
  int32_t  learned_pivot;   /* 1: FAST pipeline picks its FW-BW pivot with the context's pivot model
                               (kspn_set_pivot_model) instead of argmax in*out; same partition */
  /* Test hooks of the resident FW-BW launch; leave them 0 in production.
   *  wait_limit     polls a grid-barrier or worklist wait makes before it
   *                 gives up (KSPN_ERR_TIMEOUT); 0 = 2^22 (about half a second)
   *  drop_barrier   the launch's last block leaves at its k-th grid barrier
   *                 (k >= 1, counted from the launch start) without arriving,
   *                 so the other blocks' waits run out: a host-side stand-in
   *                 for a block that never arrives
   *  aw_exact_after worklist items after which the search tail's warps take
   *                 every find themselves instead of leaving the take to its
   *                 consumer; 0 = half the worklist */
  uint32_t wait_limit;
  uint32_t drop_barrier;
  uint32_t aw_exact_after;
  int32_t  learned_seeds;   /* 1: label searches order their seeds by the context's pivot model: vertices
                               the model scores higher get smaller labels (they win the min-label
                               propagation and become roots first); 0 = the reference's rotated ids.
                               Needs a model and n <= 2^31; same partition either way */
} kspn_options;

/* Per-call statistics (all fields written by a successful call). */
#define KSPN_PHASES 8
#define KSPN_PHASE_TRIM_FIRST 0
#define KSPN_PHASE_TRIM 1
#define KSPN_PHASE_FWBW 2
#define KSPN_PHASE_TRIM_NORMAL 3
#define KSPN_PHASE_LABEL 4
#define KSPN_PHASE_TRIM2 5
#define KSPN_PHASE_RESIDUAL 6
#define KSPN_PHASE_CANON 7
/* Kernel classes timed when kspn_options.profile is set.  Bytes follow the
 * algorithmic model: 16 B per adjacency row opened (two u64 offsets), 4 B
 * per neighbour id read, 4 B per state probe of that neighbour, 4 B per
 * queue entry read or written and per id written; bitmap sweeps n/8 B. */
#define KSPN_KERNEL_CLASSES 4
#define KSPN_KERNEL_EXPAND 0    /* top-down frontier expansion (reachability, labels) */
#define KSPN_KERNEL_BOTTOM_UP 1 /* bottom-up reachability sweep */
#define KSPN_KERNEL_TRIM 2      /* trim push levels + live-degree counting */
#define KSPN_KERNEL_STREAM 3    /* trim_1_first pass */
typedef struct kspn_stats
{
  uint32_t n;
  uint64_t m;
  uint64_t decided[KSPN_PHASES];       /* vertices decided per phase */
  double   ms[KSPN_PHASES];            /* device time per phase (CUDA events) */
  double   ms_total;                   /* device time of the whole call, inputs resident */
  uint64_t edges_scanned;              /* adjacency entries read by reachability + label kernels */
  uint32_t pivot;                      /* first FW-BW pivot (n if none) */
  uint32_t levels_fw, levels_bw;       /* reachability levels of the first FW-BW */
  uint32_t levels_bottom_up;           /* of those, bottom-up sweeps */
  uint32_t label_calls;                /* label searches run */
  uint32_t rounds;                     /* pipeline rounds after the first FW-BW */
  uint64_t kernel_launches;            /* kspn kernels launched by the call */
  double   kernel_ms[KSPN_KERNEL_CLASSES];       /* event-timed device ms per class */
  uint64_t kernel_bytes[KSPN_KERNEL_CLASSES];    /* algorithmic bytes per class */
  uint64_t kernel_calls[KSPN_KERNEL_CLASSES];    /* timed launches per class */
  /* Per-level trace of the first FW-BW, filled when kspn_options.profile is set. */
  uint32_t trace_levels;
  struct kspn_level_trace
  {
    uint32_t backward;       /* 0 FW, 1 BW */
    uint32_t bottom_up;      /* direction the level ran in */
    uint32_t frontier;       /* vertices expanded (top-down) / joined before it */
    uint32_t discovered;     /* vertices the level added */
    uint64_t frontier_edges; /* edges of the frontier (top-down direction) */
    uint64_t scanned;        /* adjacency entries read (bottom-up) */
    uint64_t candidates;     /* vertices swept (bottom-up) */
    float    ms;             /* event time of the level's expansion kernel */
    uint32_t pad;
  } trace[32];
  /* kspn_options.trace: %globaltimer stamps (ns) taken by block 0 of the
   * first FW-BW's persistent launch after each phase, and the phase that
   * ended there: 0 launch start, 8 init, 4 expansion level (top-down),
   * 5 sweep level (bottom-up), 7 frontier built from a sweep's bitmap,
   * 10 SCC written back, 11 trim live degrees + seeds, 12 trim push
   * level, 9 launch end. */
  uint32_t search_marks;
  uint32_t search_phase[128];
  uint64_t search_ns[128];
  /* The resident launch of the FAST pipeline (FW-BW, trim fixpoint and all
   * ids in one persistent kernel; 0 when the call did not run it): its
   * CUDA-event duration and its algorithmic DRAM traffic -- 16 B per
   * adjacency row opened (two u64 offsets), 4 B per neighbour id read,
   * n/8 B per pass over a vertex bitmap, 4 B per id written; probes of the
   * state bitmaps (n/8 B each, L2-resident) are not counted. */
  double   resident_ms;
  uint64_t resident_bytes;
  uint64_t resident_rows;          /* adjacency rows opened */
  uint64_t resident_edges;         /* neighbour ids read */
  uint32_t resident_bitmap_passes; /* passes over a vertex bitmap */
  uint32_t resident_pad;
  /* Heavy rows (over 2048 entries) in the resident launch: bottom-up rows
   * cut short and listed, fix-up steps that walked them, and trim vertices
   * whose heavy rows were counted in slices. */
  uint32_t heavy_cut_rows;
  uint32_t heavy_fixups;
  uint32_t heavy_trim_seeds;
  uint32_t trim_worklist;   /* 1: the resident trim tail finished on the worklist (long, thin peeling) */
  uint32_t fwbw_joint;      /* 1: the FW and BW searches of the resident launch ran side by side */
  uint32_t search_worklist; /* 1: the resident launch's searches finished on the worklist (high diameter) */
} kspn_stats;

typedef struct kspn_context kspn_context;

/* ---------------------------------------------------------------- lifetime */
int         kspn_options_default(kspn_options* opt);
/* sizeof(kspn_options) / sizeof(kspn_stats) as compiled into the library,
 * for FFI bindings to check their struct layouts. */
size_t      kspn_options_size(void);
size_t      kspn_stats_size(void);
const char* kspn_strerror(int status);
const char* kspn_last_error(const kspn_context* ctx); /* detail of the last failure on ctx */
/* device: a CUDA device ordinal, or KSPN_DEVICE_CURRENT for the calling
 * thread's current device (cudaGetDevice at creation). */
#define KSPN_DEVICE_CURRENT (-1)
int         kspn_context_create(int device, kspn_context** out);
/* Uses a caller stream (cudaStream_t passed as void*); NULL = a new stream. */
int         kspn_context_create_on_stream(int device, void* stream, kspn_context** out);
int         kspn_context_destroy(kspn_context* ctx);
int         kspn_context_synchronize(kspn_context* ctx);
/* Number of kspn kernel launches made on ctx since it was created. */
uint64_t    kspn_context_launches(const kspn_context* ctx);

/* ---------------------------------------------------------------- whole path */
/*
 * Replaces kaspan::scc(bidi_graph_part_view<single_part_view>, vertex_t*)
 * (kaspan/scc/scc.hpp:21-25).  HOST pointers: the graph is copied to the
 * device, the result copied back into scc_id[n].  bw_head/bw_csr may both be
 * NULL: the transpose is then built on the device (the reference's
 * backward_complement_graph, kaspan/scc/backward_complement.hpp:22-68).
 * ctx may be NULL (a context on device 0 is created for the call).
 */
int kspn_scc(kspn_context* ctx, uint32_t n, uint64_t m,
             const uint64_t* fw_head, const uint32_t* fw_csr,
             const uint64_t* bw_head, const uint32_t* bw_csr,
             uint32_t* scc_id, const kspn_options* opt, kspn_stats* stats);

/* Same with DEVICE pointers, on ctx's stream, inputs left untouched.
 * bw_head/bw_csr may be NULL (transpose built in ctx's workspace). */
int kspn_scc_device(kspn_context* ctx, uint32_t n, uint64_t m,
                    const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                    const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                    uint32_t* d_scc_id, const kspn_options* opt, kspn_stats* stats);

/* ---------------------------------------------------------------- phases */
/*
 * Phase-level entry points on DEVICE pointers.  Each mirrors one reference
 * function at one rank; `undecided` is the reference bitset (see top),
 * scc_id receives the same member ids the reference writes.
 */

/* trim_1_first (kaspan/scc/trim_1_local.hpp:12-46): decide in- or
 * out-degree-0 vertices (id = itself); *pivot = argmax in*out over the
 * rest, lowest id on ties, n if none.  undecided is written in full. */
int kspn_trim_1_first(kspn_context* ctx, uint32_t n, uint64_t m,
                      const uint64_t* d_fw_head, const uint64_t* d_bw_head,
                      uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* pivot);

/* cache_forward_backward_search / forward_backward_search
 * (kaspan/scc/cache_pivot_search.hpp:16-104, pivot_search.hpp:15-85). */
int kspn_forward_backward_search(kspn_context* ctx, uint32_t n, uint64_t m,
                                 const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                                 const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                                 uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t pivot,
                                 uint32_t* decided);

/* trim_1_normal (kaspan/scc/trim_1_local.hpp:48-73). */
int kspn_trim_1_normal(kspn_context* ctx, uint32_t n, uint64_t m,
                       const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                       const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                       uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided);

/* One cache_label_search_pull with map = rotr(., rotation)
 * (kaspan/scc/cache_multi_pivot_search_pull.hpp:40-244; the rotated
 * wrapper :246-266 draws rotation from a process-global counter, here the
 * caller passes it).  d_label (nullable, n entries) receives the labels. */
int kspn_label_search(kspn_context* ctx, uint32_t n, uint64_t m,
                      const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                      const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                      uint64_t* d_undecided, uint32_t* d_scc_id, int rotation,
                      uint32_t* d_label, uint32_t* decided);

/* trim_1_exhaustive_first (kaspan/scc/trim_1_exhaustive.hpp:71-131):
 * in-degree sweep to its fixpoint, then out-degree sweep; d_outdegree /
 * d_indegree receive the live degree arrays it leaves. */
int kspn_trim_1_exhaustive_first(kspn_context* ctx, uint32_t n, uint64_t m,
                                 const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                                 const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                                 uint64_t* d_undecided, uint32_t* d_scc_id,
                                 uint32_t* d_outdegree, uint32_t* d_indegree, uint32_t* decided);

/* Trim-1 to its fixpoint in both directions on the undecided sub-graph
 * (what alternating trim_1_exhaustive fw/bw converges to,
 * kaspan/scc/trim_1_exhaustive.hpp:48-69). */
int kspn_trim_1_fixpoint(kspn_context* ctx, uint32_t n, uint64_t m,
                         const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                         const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                         uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided);

/* Exact size-2 trim (no reference counterpart; an addition): decides
 * undecided pairs {u,v} where u's only undecided out-neighbour is v and v's
 * is u, or the same with in-neighbours. */
/* Residual device finish (the residual step of variant/scc_trim_ex_residual.hpp:110-127:
 * allgather_fw_sub_graph + tarjan): the sub-graph induced by the undecided
 * vertices is split into weakly connected pieces, and every piece of at most
 * 512 vertices and 2048 internal edges is decomposed by Tarjan in one warp's
 * shared memory; its SCCs get their smallest member as id and leave
 * `undecided`.  *decided = vertices decided, *pieces_left = pieces too large
 * (left undecided); both nullable. */
int kspn_residual(kspn_context* ctx, uint32_t n, uint64_t m,
                  const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                  uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided, uint32_t* pieces_left);
int kspn_trim_2(kspn_context* ctx, uint32_t n, uint64_t m,
                const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                uint64_t* d_undecided, uint32_t* d_scc_id, uint32_t* decided);

/* normalise_scc_id (kaspan/test/normalise_scc.hpp:10-25) on the device:
 * every id becomes the minimum vertex carrying it.  Ids must be < n. */
int kspn_normalise(kspn_context* ctx, uint32_t n, uint32_t* d_scc_id);

/* Canonical relabel that allocates nothing (no counterpart in the
 * reference).  Same result as kspn_normalise, for callers that cannot call
 * cudaMalloc at this point: their device memory is already handed out by
 * their own pool or caching allocator, or they cannot afford the device-wide
 * synchronisation an allocation may cause.  No context is needed: the
 * scratch is a file-scope device array for at most KSPN_NOALLOC_MAX_N
 * vertices (4 MiB, held by every GPU that loads the library until exit).
 *  - n > KSPN_NOALLOC_MAX_N: KSPN_ERR_INVALID_ARGUMENT, nothing runs.
 *  - An id >= n: KSPN_ERR_INVALID_ARGUMENT (kspn_normalise reports
 *    KSPN_ERR_INTERNAL there), and the array is left PARTLY relabelled: the
 *    ids >= n are unchanged, every id < n is already relabelled.
 *  - The first call on a device looks up the array's device address; make
 *    that first call before any stream capture.
 *  - All calls share the array: calls that overlap on the GPU race; serialise
 *    them.  Runs on `stream` (a cudaStream_t, NULL = default stream) and
 *    returns after the stream has finished. */
#define KSPN_NOALLOC_MAX_N (1u << 20)
int kspn_normalise_noalloc(uint32_t n, uint32_t* d_scc_id, void* stream);

/* backward_complement_graph (kaspan/scc/backward_complement.hpp:22-68) on
 * the device: d_bw_head[n+1] / d_bw_csr[m] receive the transpose with rows
 * in ascending order. */
int kspn_transpose(kspn_context* ctx, uint32_t n, uint64_t m,
                   const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                   uint64_t* d_bw_head, uint32_t* d_bw_csr);

/* Upload of a host CSR with its transpose built on the device while the
 * upload runs (what kspn_scc does when bw_head / bw_csr are NULL; the input
 * preparation the reference's graph adapters end with,
 * backward_complement_graph_part in kaspan/scc/adapter/kagen.hpp:38).
 * Host fw_head[n+1] / fw_csr[m]
 * are copied to d_fw_head / d_fw_csr in chunks of chunk_edges edges
 * (0 = 8 Mi) on the context's copy stream; as each chunk arrives its
 * (target, source) pairs are sorted on the context's stream, and after the
 * last one d_bw_head / d_bw_csr receive the transpose, rows ascending (the
 * same arrays as kspn_transpose).  Pinned host memory overlaps the copy
 * with the sorting.  m must be below 2^32 - 1; fw_head[0] != 0 or
 * fw_head[n] != m is KSPN_ERR_INVALID_GRAPH.  Returns after both are done. */
int kspn_upload_transpose(kspn_context* ctx, uint32_t n, uint64_t m,
                          const uint64_t* fw_head, const uint32_t* fw_csr,
                          uint64_t* d_fw_head, uint32_t* d_fw_csr,
                          uint64_t* d_bw_head, uint32_t* d_bw_csr, uint64_t chunk_edges);

/* ---------------------------------------------------------------- learned pivot
 * No reference counterpart.  An MLP 8 -> 32 -> 32 -> 1 (ReLU; BF16-rounded
 * weights, FP32 accumulation) scores pivot candidates by the odds that they
 * lie in the largest SCC; the FAST pipeline with kspn_options.learned_pivot
 * starts FW-BW from the best of trim_1_first's per-block candidates.  Only
 * the starting vertex changes, so the partition is the same.  Parameters:
 * W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3 (FP32). */
#define KSPN_MLP_PARAMS 1377
#define KSPN_MLP_FEATURES 8
/* Copies the model (host, KSPN_MLP_PARAMS floats) to the context's device;
 * NULL removes it. */
int kspn_set_pivot_model(kspn_context* ctx, const float* params);
/* Features (count x 8 FP32, device) of device vertex list d_vertices. */
int kspn_mlp_features(kspn_context* ctx, uint32_t n, uint64_t m,
                      const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                      const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                      uint32_t count, const uint32_t* d_vertices, float* d_features);
/* Logits of count feature rows with device parameters d_params. */
int kspn_mlp_forward(kspn_context* ctx, uint32_t count, const float* d_features, const float* d_params, float* d_logits);
/* Mean binary cross-entropy of sigmoid(logit) against d_labels (0 / 1) and
 * its gradient w.r.t. the FP32 parameters (through the BF16 rounding, as a
 * straight-through estimate): d_grad (KSPN_MLP_PARAMS), d_loss (1). */
int kspn_mlp_gradient(kspn_context* ctx, uint32_t count, const float* d_features, const float* d_labels,
                      const float* d_params, float* d_grad, float* d_loss);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8; step counts from 1) on the
 * device parameters, with moment buffers d_m, d_v (KSPN_MLP_PARAMS each). */
int kspn_mlp_adam(kspn_context* ctx, float* d_params, const float* d_grad, float* d_m, float* d_v, float lr, int step);

/* ---------------------------------------------------------------- batched */
/*
 * Many independent graphs in one call (no reference counterpart: the
 * reference decomposes one graph per `scc` call, kaspan/scc/scc.hpp:21-87;
 * each graph here gets the partition that call gives, min-member ids).
 * Graph g owns vertices [vtx_off[g], vtx_off[g+1]) of ONE concatenated CSR
 * (fw) and CSC (bw) over n_total = vtx_off[count] vertices: heads hold
 * global edge positions, rows hold LOCAL ids (0 .. n_g - 1).  Output:
 * scc_id[vtx_off[g] + v] = the local id of the smallest member of v's SCC.
 * Graphs of at most 512 vertices and 2048 edges are decomposed by one warp
 * each (Tarjan in shared memory), larger ones by one block or, from
 * n + m >= cluster_min, one thread-block cluster each (trim-1, FW-BW
 * rounds, Tarjan of the remainder), all in one captured CUDA graph
 * that later calls with the same arrays and settings replay.  Device
 * pointers; the context's stream; synchronous.
 */
typedef struct kspn_batch_options {
    uint32_t max_rounds;   /* FW-BW rounds per large graph before one thread's Tarjan finishes it (0: 64) */
    uint32_t rem_tarjan;   /* a large graph's remainder of at most this many vertices goes to the
                              shared-memory Tarjan (0: 512, the most it holds) */
    uint32_t cluster_size; /* blocks of the thread-block cluster a large graph gets (1..8; 0: 1, a block) */
    uint32_t reserved0;
    uint64_t cluster_min;  /* with cluster_size > 1: n + m from which a graph gets a cluster
                              instead of one block (0: 2^16) */
    uint32_t search;       /* 0 or 2: FW, then BW inside the FW set; 1: FW and BW searches of a
                              round at the same time (SCC = their intersection; half the levels,
                              more work: on C5 3% slower) */
    uint32_t route;        /* 0: the per-graph kernels above, one captured CUDA graph; 1: the mix as ONE
                              graph with global ids plus a super-source linked to every graph's
                              pivot, through the single-graph pipeline (one FW-BW decides a component
                              in every graph at once; host-driven, several synchronisations); falls
                              back to 0 when the super-source would not be the pipeline's pivot */
} kspn_batch_options;

typedef struct kspn_batch_stats {
    uint32_t graphs_small;  /* decomposed by one warp */
    uint32_t graphs_large;  /* decomposed by one block */
    uint32_t fwbw_rounds;   /* FW-BW rounds over all large graphs */
    uint32_t tarjan_smem;   /* remainders finished in shared memory */
    uint32_t tarjan_serial; /* remainders finished by one thread (round cap) */
    uint32_t trim_levels;   /* trim push levels over all large graphs */
    float    ms;            /* device time of the call (CUDA events) */
    uint32_t graphs_cluster; /* of the large ones: decomposed by a cluster of blocks */
    uint32_t cluster_size;
    float    phase_ms[5];   /* larger graphs, summed over their groups (group-leader clock):
                               init, trim, pivot, searches, remainder Tarjan; route 1: the
                               pipeline's trim_1_first, trim, (unused), FW-BW, residual + label
                               searches + relabel */
    uint32_t label_calls;   /* route 1: label searches the union needed */
    uint32_t reserved[1];
} kspn_batch_stats;

void kspn_batch_options_default(kspn_batch_options* opt);
int  kspn_scc_batched(kspn_context* ctx, uint32_t count, uint64_t n_total,
                      const uint64_t* d_vtx_off,
                      const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                      const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                      uint32_t* d_scc_id, const kspn_batch_options* opt, kspn_batch_stats* stats);

/* ---------------------------------------------------------------- autotuner */
/*
 * Picks the settings of a path by timing candidates on the caller's own
 * input (CUDA events, `reps` timed runs after one warm-up, the minimum
 * counts): coordinate descent from *base, one setting at a time, a
 * candidate kept when it is at least 2% faster.  Every candidate must give
 * the same ids as the first run (checked on the device; a mismatch is
 * KSPN_ERR_INTERNAL).  d_scc_id receives the ids.  No reference
 * counterpart: the reference's settings are compile-time constants.
 *  - kspn_autotune: FAST pipeline -- bu_enter_div, bu_leave_div (the
 *    top-down / bottom-up switch points), trim2 on/off, learned_pivot on/off
 *    (when the context holds a model);
 *  - kspn_autotune_batched: cluster_size / cluster_min (which graphs get a
 *    block or a thread-block cluster), rem_tarjan (FW-BW -> Tarjan switch
 *    point), max_rounds.
 */
typedef struct kspn_tune_report {
    uint32_t candidates;   /* settings timed */
    float    default_ms;   /* the base settings */
    float    best_ms;      /* the settings returned (<= default_ms) */
    uint32_t reserved[5];
} kspn_tune_report;

int kspn_autotune(kspn_context* ctx, uint32_t n, uint64_t m,
                  const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                  const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                  uint32_t* d_scc_id, const kspn_options* base, uint32_t reps,
                  kspn_options* best, kspn_tune_report* report);
int kspn_autotune_batched(kspn_context* ctx, uint32_t count, uint64_t n_total,
                          const uint64_t* d_vtx_off,
                          const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                          const uint64_t* d_bw_head, const uint32_t* d_bw_csr,
                          uint32_t* d_scc_id, const kspn_batch_options* base, uint32_t reps,
                          kspn_batch_options* best, kspn_tune_report* report);

/* The batch mix of uneven G(n,m) graphs (host, deterministic): graph i has
 * n_i = round(2^U[log2_min, log2_max]) vertices and round(n_i * U[deg_min,
 * deg_max]) edge draws, both drawn from SplitMix64 stream `seed` (the
 * per-graph key is draw i of that stream). */
void kspn_batch_shape(uint32_t count, uint64_t seed, uint32_t log2_min, uint32_t log2_max,
                      float deg_min, float deg_max, uint32_t* n_out, uint64_t* draws_out);
/* Its edge draws on the device, GLOBAL ids (vtx_off[g] + local): draw k of
 * graph g is (u, v) uniform in [0, n_g)^2; d_draw_off = prefix of draws_out.
 * d_graph_ids (nullable): graph g of this batch is graph d_graph_ids[g] of
 * the mix (a shard of it: the same graphs the whole mix holds). */
int  kspn_gen_batch(kspn_context* ctx, uint32_t count, uint64_t seed,
                    const uint64_t* d_vtx_off, const uint64_t* d_draw_off,
                    const uint32_t* d_graph_ids, uint32_t* d_src, uint32_t* d_dst);
/* Global ids -> local ids in every row of a concatenated CSR or CSC. */
int  kspn_batch_localize(kspn_context* ctx, uint32_t count, uint64_t n_total,
                         const uint64_t* d_vtx_off, const uint64_t* d_head, uint32_t* d_csr);

/* ---------------------------------------------------------------- one graph over several GPUs
 * One rank's device steps of the sharded decomposition (kaspan_b200/shard.py
 * drives them, one process per GPU, and runs the exchanges between ranks).
 * They replace the rank-local work of the reference's distributed
 * kaspan::scc (kaspan/scc/scc.hpp:21-87) on its 1D vertex partition: rank r
 * owns vertices [lo, lo + n_loc) of an n-vertex graph and their rows of the
 * CSR and the transpose with GLOBAL neighbour ids (the reference's
 * bidi_graph_part_view of one rank, kaspan/graph/bidi_graph_part.hpp:12-28);
 * heads hold local offsets (n_loc + 1 entries).  Local vertex state is a
 * bitmap over the local range (u32 words, bit v = global vertex lo + v);
 * scc_id holds global ids.  Device pointers; ctx's stream; each call returns
 * after its stream work has finished.
 */
/* trim_1_first on the local rows (kaspan/scc/trim_1_local.hpp:12-46):
 * d_und written in full, decided vertices get their own global id, the
 * others UNDECIDED; *best_prod / *best_id = the largest in * out among the
 * local survivors and its smallest global id (UNDECIDED when none). */
int kspn_shard_trim_first(kspn_context* ctx, uint32_t n_loc, uint32_t lo, const uint64_t* d_fw_head, const uint64_t* d_bw_head,
                          uint32_t* d_und, uint32_t* d_scc_id, uint64_t* best_prod, uint32_t* best_id, uint32_t* decided);
/* The pivot rule on the remaining graph (kaspan/scc/pivot.hpp:53-74, raw
 * degrees): largest in * out among the undecided local vertices. */
int kspn_shard_pivot(kspn_context* ctx, uint32_t n_loc, uint32_t lo, const uint64_t* d_fw_head, const uint64_t* d_bw_head,
                     const uint32_t* d_und, uint64_t* best_prod, uint32_t* best_id);
/* Start of an FW-BW search: candidates of both searches = und, reached = {},
 * the bitmaps of ids sent to other shards (n bits each) cleared. */
int kspn_shard_search_begin(kspn_context* ctx, uint32_t n_loc, uint32_t n, const uint32_t* d_und, uint32_t* d_cand_fw, uint32_t* d_cand_bw,
                            uint32_t* d_vis_fw, uint32_t* d_vis_bw, uint32_t* d_sent_fw, uint32_t* d_sent_bw);
/* One top-down level of one search over the local rows (the forward rows for
 * FW, the transposed ones for BW; cache_forward_backward_search,
 * kaspan/scc/cache_pivot_search.hpp:16-104): a local neighbour still in
 * d_cand is taken (set in d_vis, appended to d_next after the *next_n
 * entries already there; *next_n updated); a remote one is claimed once per
 * search in d_sent and sent to its owner: d_send receives the remote ids
 * grouped by owning shard (shard r owns [d_bounds[r], d_bounds[r + 1])),
 * counts[parts] (host) their number per shard -- the payload and counts of
 * the reference's frontier exchange (kaspan/scc/frontier.hpp:237-282).
 * d_remote (remote_cap entries) and d_counts (2 * parts) are scratch. */
int kspn_shard_expand(kspn_context* ctx, uint32_t n_loc, uint32_t lo, const uint64_t* d_head, const uint32_t* d_adj,
                      const uint32_t* d_frontier, uint32_t frontier_n, uint32_t* d_cand, uint32_t* d_vis, uint32_t* d_sent,
                      uint32_t* d_next, uint32_t next_cap, uint32_t* next_n, uint32_t* d_remote, uint32_t remote_cap,
                      uint32_t parts, const uint32_t* d_bounds, uint32_t* d_send, uint32_t* d_counts, uint32_t* counts);
/* Ids other shards sent this one (global ids in its range): taken as local
 * finds (appended to d_next after *next_n entries). */
int kspn_shard_receive(kspn_context* ctx, uint32_t n_loc, uint32_t lo, const uint32_t* d_recv, uint32_t recv_n, uint32_t* d_cand,
                       uint32_t* d_vis, uint32_t* d_next, uint32_t next_cap, uint32_t* next_n);
/* Smallest global id in FW & BW on this shard (UNDECIDED if none). */
int kspn_shard_scc_min(kspn_context* ctx, uint32_t n_loc, uint32_t lo, const uint32_t* d_vis_fw, const uint32_t* d_vis_bw, uint32_t* min_id);
/* The SCC FW & BW leaves d_und; its local members get id `id`. */
int kspn_shard_finalize(kspn_context* ctx, uint32_t n_loc, const uint32_t* d_vis_fw, const uint32_t* d_vis_bw, uint32_t* d_und,
                        uint32_t* d_scc_id, uint32_t id, uint32_t* decided);
/* The residual sub-graph's edges leaving this shard (the local part of
 * allgather_fw_sub_graph, kaspan/scc/allgather_sub_graph.hpp:253-301):
 * (lo + v, u) for every undecided local v and out-neighbour u undecided in
 * d_global_und (ceil(n / 32) words of the whole graph); *count = their
 * number, written while it stays below cap. */
int kspn_shard_residual(kspn_context* ctx, uint32_t n_loc, uint32_t lo, const uint64_t* d_fw_head, const uint32_t* d_fw_csr,
                        const uint32_t* d_und, const uint32_t* d_global_und, uint32_t* d_src, uint32_t* d_dst, uint64_t cap,
                        uint64_t* count);

/* ---------------------------------------------------------------- manifest graph files */
/*
 * The reference's on-disk graph format (kaspan/scc/adapter/manifest.hpp:
 * 19-245): a text manifest of `key value` lines (`%` starts a comment) and
 * four binary files -- fw/bw head (n + 1 entries) and fw/bw csr (m entries)
 * -- of dense unsigned integers, graph.head.bytes / graph.csr.bytes bytes
 * each (1..8), in graph.endian byte order.  Paths in the manifest are
 * relative to its directory.
 */
typedef struct kspn_manifest {
    uint32_t schema_version;
    int32_t  big_endian;        /* graph.endian: 0 little, 1 big */
    uint64_t node_count;        /* graph.node_count */
    uint64_t edge_count;        /* graph.edge_count */
    int32_t  self_loops;        /* graph.contains_self_loops */
    int32_t  duplicate_edges;   /* graph.contains_duplicate_edges */
    uint32_t head_bytes;        /* graph.head.bytes */
    uint32_t csr_bytes;         /* graph.csr.bytes */
    char     graph_code[64];
    char     graph_name[128];
    char     fw_head_path[1024];  /* resolved against the manifest's directory */
    char     fw_csr_path[1024];
    char     bw_head_path[1024];
    char     bw_csr_path[1024];
} kspn_manifest;

/* Parses a manifest (host only; every key the reference requires must be
 * present, widths 1..8, booleans true/false, endian little/big). */
int kspn_manifest_read(const char* path, kspn_manifest* out);
/* Loads its four files into device arrays (u64 heads of n + 1, u32 ids of
 * m entries): pinned host chunks, raw copies, a decode kernel on the
 * device.  Entries beyond m (heads) or >= n (ids) are KSPN_ERR_INVALID_GRAPH. */
int kspn_manifest_load(kspn_context* ctx, const kspn_manifest* mf,
                       uint64_t* d_fw_head, uint32_t* d_fw_csr,
                       uint64_t* d_bw_head, uint32_t* d_bw_csr);
/* Writes host arrays as <dir>/<name>.manifest + four .bin files with the
 * given entry widths and byte order (an entry that does not fit is an error). */
int kspn_manifest_write(const char* dir, const char* name, uint32_t n, uint64_t m,
                        const uint64_t* fw_head, const uint32_t* fw_csr,
                        const uint64_t* bw_head, const uint32_t* bw_csr,
                        uint32_t head_bytes, uint32_t csr_bytes, int big_endian,
                        int self_loops, int duplicate_edges);

/* ---------------------------------------------------------------- inputs */
/*
 * Seeded synthetic edge lists on the device (no reference counterpart:
 * they stand in for the KaGen generators the reference benchmarks with).
 * Draw i of a stream is SplitMix64's finaliser applied to key + (i+1)*gamma.
 */
int kspn_gen_gnm(kspn_context* ctx, uint32_t n, uint64_t draws, uint64_t seed,
                 uint32_t* d_src, uint32_t* d_dst);
int kspn_gen_rmat(kspn_context* ctx, int scale, uint64_t draws, uint64_t seed,
                  uint64_t t_a, uint64_t t_ab, uint64_t t_abc, int permute,
                  uint32_t* d_src, uint32_t* d_dst);
/* Random geometric graph in the unit square (stands in for KaGen's rgg2d):
 * n points on a g x g cell grid, squared radius r2 in units of 2^-60
 * (pass g = floor(1/r), r2 = floor(r^2 * 2^60)); each pair within the
 * radius becomes u->v, v->u, both or neither with probability 1/4 each.
 * *m_out = the edge count; the edges are written when d_src and d_dst are
 * given and hold `capacity` >= *m_out entries (otherwise, with buffers,
 * KSPN_ERR_INVALID_ARGUMENT and *m_out set). */
int kspn_gen_rgg(kspn_context* ctx, uint32_t n, uint64_t seed, uint32_t g, uint64_t r2,
                 uint32_t* d_src, uint32_t* d_dst, uint64_t capacity, uint64_t* m_out);
/* Edge list -> CSR with self-loops and duplicates removed, rows ascending.
 * d_src/d_dst are overwritten (used as scratch).  *m_out = edges kept. */
int kspn_build_csr(kspn_context* ctx, uint32_t n, uint64_t m_raw,
                   uint32_t* d_src, uint32_t* d_dst,
                   uint64_t* d_head, uint32_t* d_csr, uint64_t* m_out);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* KSPN_H */
