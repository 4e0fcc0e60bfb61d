/*
 * kspn oracle -- CPU CHECKER, TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's single-rank SCC path
 * (rawbby/KaSpan, kaspan/include/kaspan/...), used by tests/ and by the
 * bench's CPU-baseline leg to check and time the CUDA library.  The product
 * library (kaspan_b200/libkspn.so) never links, loads or calls this file.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's own code compiled from its sources (oracle/_ref, built by
 * oracle/Makefile) and against the known-answer fixtures in tests/golden.
 *
 * Conventions: n vertices with u32 ids, u64 CSR offsets ("head", n+1
 * entries), u32 neighbour ids ("csr"); fw = out-edges, bw = in-edges (the
 * transpose).  Vertex state "undecided" is one byte per vertex (1 =
 * undecided); the reference keeps a bitset, which changes nothing here.
 *
 * The synthetic-graph generators at the end are NOT reference code: they
 * restate, on the CPU, the seeded input definitions the CUDA generators in
 * kaspan_b200/csrc/gen.cu implement, so both sides build identical graphs.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define UNDECIDED 0xFFFFFFFFu

/* ------------------------------------------------------------------ */
/* Canonical relabel: kaspan/test/normalise_scc.hpp:10-25.  Each id is  */
/* replaced by the first vertex (in id order) that carries it, i.e. the */
/* minimum member of the component.  old2new is a dense table here.     */
/* ------------------------------------------------------------------ */
void
orc_normalise(uint32_t n, uint32_t* scc_id)
{
  uint32_t* old2new = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (uint32_t i = 0; i < n; ++i) old2new[i] = UNDECIDED;
  for (uint32_t u = 0; u < n; ++u) {
    uint32_t const id = scc_id[u];
    if (id >= n) { /* ids outside [0,n) are left as they are */
      continue;
    }
    if (old2new[id] == UNDECIDED) old2new[id] = u;
    scc_id[u] = old2new[id];
  }
  free(old2new);
}

/* ------------------------------------------------------------------ */
/* Iterative Tarjan: kaspan/scc/tarjan.hpp:20-122, with the SCC naming   */
/* of test_mpi/test_tarjan_vs_kaspan.cpp:37-45 (id = min member).       */
/* Returns the number of components.                                    */
/* ------------------------------------------------------------------ */
uint32_t
orc_tarjan(uint32_t n, uint64_t const* head, uint32_t const* csr, uint32_t* scc_id)
{
  uint32_t* index    = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t* low      = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint8_t*  on_stack = (uint8_t*)calloc(n + 1, 1);
  uint32_t* st       = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t* dfs_u    = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint64_t* dfs_it   = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  uint32_t  st_n = 0, dfs_n = 0, count = 0, comps = 0;

  for (uint32_t i = 0; i < n; ++i) index[i] = UNDECIDED;

  for (uint32_t root = 0; root < n; ++root) {
    if (index[root] != UNDECIDED) continue;
    index[root] = low[root] = count++;
    st[st_n++]              = root;
    on_stack[root]          = 1;
    dfs_u[dfs_n]            = root;
    dfs_it[dfs_n++]         = head[root];

    while (dfs_n) {
      uint32_t const u  = dfs_u[dfs_n - 1];
      uint64_t const it = dfs_it[dfs_n - 1];
      if (it < head[u + 1]) {
        uint32_t const v = csr[it];
        dfs_it[dfs_n - 1] += 1;
        if (index[v] == UNDECIDED) {
          index[v] = low[v] = count++;
          st[st_n++]        = v;
          on_stack[v]       = 1;
          dfs_u[dfs_n]      = v;
          dfs_it[dfs_n++]   = head[v];
        } else if (on_stack[v] && index[v] < low[u]) {
          low[u] = index[v];
        }
        continue;
      }
      if (low[u] == index[u]) {
        uint32_t const end = st_n;
        for (;;) {
          uint32_t const v = st[--st_n];
          on_stack[v]      = 0;
          if (v == u) break;
        }
        uint32_t id = UNDECIDED;
        for (uint32_t i = st_n; i < end; ++i)
          if (st[i] < id) id = st[i];
        for (uint32_t i = st_n; i < end; ++i) scc_id[st[i]] = id;
        ++comps;
      }
      --dfs_n;
      if (dfs_n) {
        uint32_t const p = dfs_u[dfs_n - 1];
        if (low[u] < low[p]) low[p] = low[u];
      }
    }
  }
  free(index);
  free(low);
  free(on_stack);
  free(st);
  free(dfs_u);
  free(dfs_it);
  return comps;
}

/* ------------------------------------------------------------------ */
/* trim_1_first: kaspan/scc/trim_1_local.hpp:12-46 at one rank.          */
/* Decides every vertex with in- or out-degree 0 (id = itself) and      */
/* returns the pivot argmax(in*out) over the rest, first (lowest) id on */
/* ties; n when every vertex was decided.                               */
/* ------------------------------------------------------------------ */
uint32_t
orc_trim_1_first(uint32_t n, uint64_t const* fwh, uint64_t const* bwh, uint8_t* undecided, uint32_t* scc_id, uint32_t* decided_count)
{
  uint64_t best  = 0;
  uint32_t pivot = n, dec = 0;
  for (uint32_t k = 0; k < n; ++k) {
    uint64_t const out = fwh[k + 1] - fwh[k];
    uint64_t const in  = bwh[k + 1] - bwh[k];
    if (in == 0 || out == 0) {
      undecided[k] = 0;
      scc_id[k]    = k;
      ++dec;
    } else {
      uint64_t const prod = in * out;
      if (best < prod) {
        best  = prod;
        pivot = k;
      }
    }
  }
  if (decided_count) *decided_count = dec;
  return pivot;
}

/* ------------------------------------------------------------------ */
/* trim_1_normal: kaspan/scc/trim_1_local.hpp:48-73.  Decides undecided  */
/* vertices with no undecided neighbour in either direction.  Two       */
/* adjacent undecided vertices can never both pass, so the reference's  */
/* in-pass updates do not change the outcome of this one-pass form.     */
/* ------------------------------------------------------------------ */
uint32_t
orc_trim_1_normal(uint32_t n, uint64_t const* fwh, uint32_t const* fwc, uint64_t const* bwh, uint32_t const* bwc, uint8_t* undecided, uint32_t* scc_id)
{
  uint32_t dec = 0;
  for (uint32_t k = 0; k < n; ++k) {
    if (!undecided[k]) continue;
    int has = 0;
    for (uint64_t e = fwh[k]; e < fwh[k + 1] && !has; ++e) has = undecided[fwc[e]];
    for (uint64_t e = bwh[k]; e < bwh[k + 1] && !has; ++e) has = undecided[bwc[e]];
    if (!has) {
      undecided[k] = 0;
      scc_id[k]    = k;
      ++dec;
    }
  }
  return dec;
}

/* ------------------------------------------------------------------ */
/* Single-pivot forward-backward search:                               */
/* kaspan/scc/cache_pivot_search.hpp:16-104 (== pivot_search.hpp:15-85  */
/* at one rank).  FW: vertices reachable from the pivot through         */
/* undecided vertices.  BW: of those, the ones that reach the pivot     */
/* through FW-reached vertices; each is decided with id = pivot.        */
/* Returns the number decided.                                          */
/* ------------------------------------------------------------------ */
uint32_t
orc_fw_bw(uint32_t n, uint64_t const* fwh, uint32_t const* fwc, uint64_t const* bwh, uint32_t const* bwc, uint8_t* undecided, uint32_t* scc_id, uint32_t pivot)
{
  uint8_t*  reached = (uint8_t*)calloc(n + 1, 1);
  uint32_t* stack   = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t  sp = 0, dec = 0;

  reached[pivot] = 1;
  stack[sp++]    = pivot;
  while (sp) {
    uint32_t const u = stack[--sp];
    for (uint64_t e = fwh[u]; e < fwh[u + 1]; ++e) {
      uint32_t const v = fwc[e];
      if (undecided[v] && !reached[v]) {
        reached[v]  = 1;
        stack[sp++] = v;
      }
    }
  }

  reached[pivot]   = 0;
  undecided[pivot] = 0;
  scc_id[pivot]    = pivot;
  ++dec;
  stack[sp++] = pivot;
  while (sp) {
    uint32_t const u = stack[--sp];
    for (uint64_t e = bwh[u]; e < bwh[u + 1]; ++e) {
      uint32_t const v = bwc[e];
      if (reached[v]) {
        reached[v]   = 0;
        undecided[v] = 0;
        scc_id[v]    = pivot;
        ++dec;
        stack[sp++] = v;
      }
    }
  }
  free(reached);
  free(stack);
  return dec;
}

static inline uint32_t
rotr32(uint32_t x, int r)
{
  r &= 31;
  return r ? (x >> r) | (x << (32 - r)) : x;
}
static inline uint32_t
rotl32(uint32_t x, int r)
{
  r &= 31;
  return r ? (x << r) | (x >> (32 - r)) : x;
}

/* ------------------------------------------------------------------ */
/* One multi-pivot label ("colour") search, pull form:                  */
/* kaspan/scc/cache_multi_pivot_search_pull.hpp:40-244 at one rank,    */
/* with map = rotr(., rotation), unmap = rotl(., rotation) as in        */
/* cache_rot_label_search_pull (:246-266).                              */
/*  FW: label[k] = min over undecided in-neighbours, to a fixpoint      */
/*      (= min map() over k's undecided ancestors, itself included).    */
/*  roots: label[k] == map(k), decided with id unmap(label) = k.        */
/*  BW: k joins if an out-neighbour was decided with the same label.    */
/* Returns the number decided (at least one while any is undecided).    */
/* ------------------------------------------------------------------ */
uint32_t
orc_label_search_pull(uint32_t n, uint64_t const* fwh, uint32_t const* fwc, uint64_t const* bwh, uint32_t const* bwc, uint8_t* undecided, uint32_t* scc_id, int rotation, uint32_t* label_out)
{
  uint32_t* label     = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t* stack     = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint8_t*  in_active = (uint8_t*)calloc(n + 1, 1);
  uint32_t  sp = 0, dec = 0;

  for (uint32_t k = 0; k < n; ++k) {
    if (undecided[k]) {
      label[k]     = rotr32(k, rotation);
      in_active[k] = 1;
      stack[sp++]  = k;
    } else {
      label[k] = UNDECIDED;
    }
  }
  while (sp) {
    uint32_t const k = stack[--sp];
    if (!undecided[k]) {
      in_active[k] = 0;
      continue;
    }
    uint32_t m = label[k];
    for (uint64_t e = bwh[k]; e < bwh[k + 1]; ++e) {
      uint32_t const v = bwc[e];
      if (undecided[v] && label[v] < m) m = label[v];
    }
    if (m < label[k]) {
      label[k] = m;
      for (uint64_t e = fwh[k]; e < fwh[k + 1]; ++e) {
        uint32_t const v = fwc[e];
        if (undecided[v] && !in_active[v]) {
          in_active[v] = 1;
          stack[sp++]  = v;
        }
      }
    }
    in_active[k] = 0;
  }

  /* roots, then the backward closure inside each label class */
  memset(in_active, 0, n + 1);
  uint8_t* root = (uint8_t*)calloc(n + 1, 1);
  for (uint32_t k = 0; k < n; ++k) {
    if (undecided[k] && label[k] == rotr32(k, rotation)) {
      undecided[k] = 0;
      scc_id[k]    = rotl32(label[k], rotation);
      root[k]      = 1;
      ++dec;
    }
  }
  for (uint32_t k = 0; k < n; ++k) {
    if (!root[k]) continue;
    for (uint64_t e = bwh[k]; e < bwh[k + 1]; ++e) {
      uint32_t const v = bwc[e];
      if (undecided[v] && !in_active[v]) {
        in_active[v] = 1;
        stack[sp++]  = v;
      }
    }
  }
  while (sp) {
    uint32_t const k = stack[--sp];
    if (!undecided[k]) {
      in_active[k] = 0;
      continue;
    }
    uint32_t const lk      = label[k];
    int            reached = 0;
    for (uint64_t e = fwh[k]; e < fwh[k + 1]; ++e) {
      uint32_t const v = fwc[e];
      if (!undecided[v] && label[v] == lk) reached = 1;
    }
    if (reached) {
      undecided[k] = 0;
      scc_id[k]    = rotl32(lk, rotation);
      ++dec;
      for (uint64_t e = bwh[k]; e < bwh[k + 1]; ++e) {
        uint32_t const v = bwc[e];
        if (undecided[v] && !in_active[v]) {
          in_active[v] = 1;
          stack[sp++]  = v;
        }
      }
    }
    in_active[k] = 0;
  }
  if (label_out) memcpy(label_out, label, sizeof(uint32_t) * n);
  free(root);
  free(label);
  free(stack);
  free(in_active);
  return dec;
}

/* ------------------------------------------------------------------ */
/* Exhaustive trim-1: kaspan/scc/trim_1_exhaustive.hpp:14-46 (one       */
/* direction) and :71-131 (first pass: in-degree sweep, then            */
/* out-degree sweep).  degree[] holds live degrees of undecided         */
/* vertices; a vertex whose degree reaches 0 is decided (id = itself).  */
/* ------------------------------------------------------------------ */
static uint32_t
trim_ex_dir(uint64_t const* head, uint32_t const* csr, uint8_t* undecided, uint32_t* scc_id, uint32_t* degree, uint32_t* queue, uint64_t qn)
{
  /* queue holds vertices whose (this-direction) degree must drop by one */
  uint32_t dec = 0;
  while (qn) {
    uint32_t const k = queue[--qn];
    if (undecided[k]) {
      if (--degree[k] == 0) {
        undecided[k] = 0;
        scc_id[k]    = k;
        ++dec;
        for (uint64_t e = head[k]; e < head[k + 1]; ++e) queue[qn++] = csr[e];
      }
    }
  }
  return dec;
}

uint32_t
orc_trim_1_exhaustive_first(uint32_t n, uint64_t m, uint64_t const* fwh, uint32_t const* fwc, uint64_t const* bwh, uint32_t const* bwc, uint8_t* undecided, uint32_t* scc_id, uint32_t* outdegree, uint32_t* indegree)
{
  /* each undecided vertex is pushed at most once per incident edge */
  uint32_t* queue = (uint32_t*)malloc(sizeof(uint32_t) * (m + 1));
  uint64_t  qn    = 0;
  uint32_t  dec   = 0;
  for (uint32_t k = 0; k < n; ++k) {
    uint64_t const d = bwh[k + 1] - bwh[k];
    if (d > 0) indegree[k] = (uint32_t)d;
    else {
      undecided[k] = 0;
      scc_id[k]    = k;
      ++dec;
      for (uint64_t e = fwh[k]; e < fwh[k + 1]; ++e) queue[qn++] = fwc[e];
    }
  }
  dec += trim_ex_dir(fwh, fwc, undecided, scc_id, indegree, queue, qn);
  qn = 0;
  for (uint32_t k = 0; k < n; ++k) {
    if (!undecided[k]) continue;
    uint64_t const d = fwh[k + 1] - fwh[k];
    if (d > 0) outdegree[k] = (uint32_t)d;
    else {
      undecided[k] = 0;
      scc_id[k]    = k;
      ++dec;
      for (uint64_t e = bwh[k]; e < bwh[k + 1]; ++e) queue[qn++] = bwc[e];
    }
  }
  dec += trim_ex_dir(bwh, bwc, undecided, scc_id, outdegree, queue, qn);
  free(queue);
  return dec;
}

/* ------------------------------------------------------------------ */
/* Full exhaustive trim to a fixpoint in both directions on the current */
/* undecided sub-graph (what the reference reaches by alternating       */
/* trim_1_exhaustive fw/bw, kaspan/scc/trim_1_exhaustive.hpp:48-69).    */
/* Used to check the device trim, which is order-free.                  */
/* ------------------------------------------------------------------ */
uint32_t
orc_trim_1_fixpoint(uint32_t n, uint64_t const* fwh, uint32_t const* fwc, uint64_t const* bwh, uint32_t const* bwc, uint8_t* undecided, uint32_t* scc_id)
{
  uint32_t* indeg  = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
  uint32_t* outdeg = (uint32_t*)calloc(n + 1, sizeof(uint32_t));
  uint32_t* queue  = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint8_t*  queued = (uint8_t*)calloc(n + 1, 1);
  uint32_t  qn = 0, dec = 0;
  for (uint32_t k = 0; k < n; ++k) {
    if (!undecided[k]) continue;
    for (uint64_t e = bwh[k]; e < bwh[k + 1]; ++e) indeg[k] += undecided[bwc[e]];
    for (uint64_t e = fwh[k]; e < fwh[k + 1]; ++e) outdeg[k] += undecided[fwc[e]];
    if (indeg[k] == 0 || outdeg[k] == 0) {
      queue[qn++] = k;
      queued[k]   = 1;
    }
  }
  while (qn) {
    uint32_t const k = queue[--qn];
    undecided[k]     = 0;
    scc_id[k]        = k;
    ++dec;
    for (uint64_t e = fwh[k]; e < fwh[k + 1]; ++e) {
      uint32_t const v = fwc[e];
      if (undecided[v] && !queued[v] && --indeg[v] == 0) {
        queue[qn++] = v;
        queued[v]   = 1;
      }
    }
    for (uint64_t e = bwh[k]; e < bwh[k + 1]; ++e) {
      uint32_t const v = bwc[e];
      if (undecided[v] && !queued[v] && --outdeg[v] == 0) {
        queue[qn++] = v;
        queued[v]   = 1;
      }
    }
  }
  free(indeg);
  free(outdeg);
  free(queue);
  free(queued);
  return dec;
}

/* ------------------------------------------------------------------ */
/* Default pipeline kaspan::scc, kaspan/scc/scc.hpp:21-87:              */
/* trim_1_first -> FW-BW(pivot) -> trim_1_normal -> repeated rotated    */
/* label searches (rotation 1, 2, 3, ... as the reference's counter     */
/* gives in a fresh process).  phase_decided (nullable, 4 entries)      */
/* receives the count each phase decided; returns the number of label   */
/* search calls.  scc_id holds member ids (not normalised).             */
/* ------------------------------------------------------------------ */
uint32_t
orc_scc(uint32_t n, uint64_t const* fwh, uint32_t const* fwc, uint64_t const* bwh, uint32_t const* bwc, uint32_t* scc_id, uint32_t* phase_decided)
{
  uint8_t* undecided = (uint8_t*)malloc(n + 1);
  memset(undecided, 1, n + 1);
  uint32_t pd[4] = { 0, 0, 0, 0 };
  uint32_t calls = 0;
  uint32_t dec   = 0;
  uint32_t pivot = orc_trim_1_first(n, fwh, bwh, undecided, scc_id, &pd[0]);
  dec += pd[0];
  if (dec < n) {
    pd[1] = orc_fw_bw(n, fwh, fwc, bwh, bwc, undecided, scc_id, pivot);
    dec += pd[1];
  }
  if (dec < n) {
    pd[2] = orc_trim_1_normal(n, fwh, fwc, bwh, bwc, undecided, scc_id);
    dec += pd[2];
  }
  int rotation = 0;
  while (dec < n) {
    ++rotation;
    uint32_t const d = orc_label_search_pull(n, fwh, fwc, bwh, bwc, undecided, scc_id, rotation, NULL);
    pd[3] += d;
    dec += d;
    ++calls;
  }
  if (phase_decided) memcpy(phase_decided, pd, sizeof(pd));
  free(undecided);
  return calls;
}

/* ================================================================== */
/* Synthetic inputs (not reference code; the CPU side of the seeded    */
/* generators the CUDA library implements in kaspan_b200/csrc/gen.cu). */
/* ================================================================== */

/* SplitMix64 (Steele, Lea, Flood 2014): state advanced by the golden   */
/* gamma, output through the variant-13 finaliser.  Counter-based use:  */
/* draw i of a stream with key K is fmix(K + (i+1)*gamma).              */
static inline uint64_t
fmix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
uint64_t
orc_seed_key(uint64_t seed)
{
  return fmix64(seed + 0x9E3779B97F4A7C15ull);
}
uint64_t
orc_draw(uint64_t key, uint64_t i)
{
  return fmix64(key + (i + 1) * 0x9E3779B97F4A7C15ull);
}

/* Directed G(n, draws): draw i gives u = lo32 * n >> 32, v = hi32 * n >> 32. */
void
orc_gen_gnm(uint32_t n, uint64_t draws, uint64_t seed, uint32_t* src, uint32_t* dst)
{
  uint64_t const key = orc_seed_key(seed);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)draws; ++i) {
    uint64_t const r = orc_draw(key, (uint64_t)i);
    src[i]           = (uint32_t)(((r & 0xFFFFFFFFull) * (uint64_t)n) >> 32);
    dst[i]           = (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
  }
}

/* Seeded bijection on [0, 2^scale): three rounds of add-key, multiply by */
/* an odd key, xorshift right, all mod 2^scale.                           */
uint32_t
orc_rmat_perm(uint32_t x, int scale, uint64_t pkey)
{
  uint32_t const mask = scale >= 32 ? 0xFFFFFFFFu : ((1u << scale) - 1u);
  int const      sh   = (scale + 1) / 2;
  for (int r = 0; r < 3; ++r) {
    uint64_t const k = orc_draw(pkey, (uint64_t)r);
    x                = (x + (uint32_t)k) & mask;
    x                = (x * ((uint32_t)(k >> 32) | 1u)) & mask;
    if (sh > 0) x ^= x >> sh;
  }
  return x & mask;
}

/* R-MAT: draw i descends `scale` levels; level l uses 32-bit word l&1  */
/* of stream value i*ceil(scale/2) + l/2 and picks quadrant a|b|c|d by  */
/* the integer thresholds t[0..2] (= floor(p * 2^32), cumulative).      */
/* Both endpoints then go through orc_rmat_perm with key draw(key', 0). */
void
orc_gen_rmat(int scale, uint64_t draws, uint64_t seed, uint64_t ta, uint64_t tab, uint64_t tabc, int permute, uint32_t* src, uint32_t* dst)
{
  uint64_t const key   = orc_seed_key(seed);
  uint64_t const pkey  = orc_seed_key(seed ^ 0x5045524D55544531ull);
  int const      words = (scale + 1) / 2;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)draws; ++i) {
    uint32_t u = 0, v = 0;
    uint64_t r = 0;
    for (int l = 0; l < scale; ++l) {
      if ((l & 1) == 0) r = orc_draw(key, (uint64_t)i * (uint64_t)words + (uint64_t)(l >> 1));
      uint64_t const x = (l & 1) ? (r >> 32) : (r & 0xFFFFFFFFull);
      uint32_t       bu, bv;
      if (x < ta) bu = 0, bv = 0;
      else if (x < tab) bu = 0, bv = 1;
      else if (x < tabc) bu = 1, bv = 0;
      else bu = 1, bv = 1;
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
    if (permute) {
      u = orc_rmat_perm(u, scale, pkey);
      v = orc_rmat_perm(v, scale, pkey);
    }
    src[i] = u;
    dst[i] = v;
  }
}

/* 2-D random geometric graph.  Point i: x = draw(key, 2i) >> 34,        */
/* y = draw(key, 2i+1) >> 34 (30-bit fixed point).  Cells: g = floor(1/r) */
/* per side, cell = (y*g>>30)*g + (x*g>>30); vertex ids are ranks in the  */
/* order (cell, i).  Each pair i<j (new ids) with dx^2+dy^2 <= r2 (fixed  */
/* point, r2 = floor(r^2 * 2^60)) draws h = draw(key2, i<<32|j): top two */
/* bits 0: i->j, 1: j->i, 2: both, 3: none.                                */
/* Phase 1 (orc_rgg_points) sorts the points; phase 2 (orc_rgg_edges)   */
/* counts (src == NULL) or writes the edges.                              */
typedef struct
{
  uint32_t* px;     /* by new id */
  uint32_t* py;     /* by new id */
  uint64_t* cell_start; /* g*g + 1 */
  uint32_t  g;
} orc_rgg_t;

static int
cmp_u64(void const* a, void const* b)
{
  uint64_t const x = *(uint64_t const*)a, y = *(uint64_t const*)b;
  return x < y ? -1 : x > y;
}

void
orc_rgg_points(uint32_t n, uint64_t seed, uint32_t g, uint32_t* px, uint32_t* py, uint64_t* cell_start)
{
  uint64_t const key  = orc_seed_key(seed);
  uint64_t*      keys = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
  uint32_t*      x0   = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t*      y0   = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    uint32_t const x = (uint32_t)(orc_draw(key, 2 * (uint64_t)i) >> 34);
    uint32_t const y = (uint32_t)(orc_draw(key, 2 * (uint64_t)i + 1) >> 34);
    uint64_t const cx = ((uint64_t)x * g) >> 30, cy = ((uint64_t)y * g) >> 30;
    x0[i]   = x;
    y0[i]   = y;
    keys[i] = ((cy * g + cx) << 32) | (uint64_t)i;
  }
  qsort(keys, n, sizeof(uint64_t), cmp_u64);
  memset(cell_start, 0, sizeof(uint64_t) * ((uint64_t)g * g + 1));
  for (uint32_t j = 0; j < n; ++j) {
    uint32_t const i = (uint32_t)(keys[j] & 0xFFFFFFFFull);
    px[j]            = x0[i];
    py[j]            = y0[i];
    cell_start[(keys[j] >> 32) + 1] += 1;
  }
  for (uint64_t c = 0; c < (uint64_t)g * g; ++c) cell_start[c + 1] += cell_start[c];
  free(keys);
  free(x0);
  free(y0);
}

/* Edges of vertex i (to partners j > i).  Writes at most cap entries.   */
static uint64_t
rgg_vertex_edges(uint32_t i, uint32_t const* px, uint32_t const* py, uint64_t const* cell_start, uint32_t g, uint64_t r2, uint64_t key2, uint32_t* src, uint32_t* dst)
{
  uint64_t       cnt = 0;
  uint64_t const cx = ((uint64_t)px[i] * g) >> 30, cy = ((uint64_t)py[i] * g) >> 30;
  for (int dy = -1; dy <= 1; ++dy) {
    int64_t const yy = (int64_t)cy + dy;
    if (yy < 0 || yy >= (int64_t)g) continue;
    for (int dx = -1; dx <= 1; ++dx) {
      int64_t const xx = (int64_t)cx + dx;
      if (xx < 0 || xx >= (int64_t)g) continue;
      uint64_t const c = (uint64_t)yy * g + (uint64_t)xx;
      for (uint64_t j = cell_start[c]; j < cell_start[c + 1]; ++j) {
        if (j <= i) continue;
        int64_t const  ddx = (int64_t)px[i] - (int64_t)px[j];
        int64_t const  ddy = (int64_t)py[i] - (int64_t)py[j];
        uint64_t const d2  = (uint64_t)(ddx * ddx) + (uint64_t)(ddy * ddy);
        if (d2 > r2) continue;
        uint64_t const h   = orc_draw(key2, ((uint64_t)i << 32) | j);
        unsigned const dir = (unsigned)(h >> 62);
        if (dir == 0 || dir == 2) {
          if (src) src[cnt] = i, dst[cnt] = (uint32_t)j;
          ++cnt;
        }
        if (dir == 1 || dir == 2) {
          if (src) src[cnt] = (uint32_t)j, dst[cnt] = i;
          ++cnt;
        }
      }
    }
  }
  return cnt;
}

/* Counts (src == NULL) or writes all edges; offsets[n+1] is filled by a  */
/* counting call and read by the writing call.                            */
uint64_t
orc_rgg_edges(uint32_t n, uint64_t seed, uint32_t g, uint64_t r2, uint32_t const* px, uint32_t const* py, uint64_t const* cell_start, uint64_t* offsets, uint32_t* src, uint32_t* dst)
{
  uint64_t const key2 = orc_seed_key(seed ^ 0x5247474544474553ull);
  if (!src) {
#pragma omp parallel for schedule(dynamic, 4096)
    for (int64_t i = 0; i < (int64_t)n; ++i)
      offsets[i + 1] = rgg_vertex_edges((uint32_t)i, px, py, cell_start, g, r2, key2, NULL, NULL);
    offsets[0] = 0;
    for (uint32_t i = 0; i < n; ++i) offsets[i + 1] += offsets[i];
    return offsets[n];
  }
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t i = 0; i < (int64_t)n; ++i)
    rgg_vertex_edges((uint32_t)i, px, py, cell_start, g, r2, key2, src + offsets[i], dst + offsets[i]);
  return offsets[n];
}

/* Edge list -> CSR with self-loops and duplicates removed and rows       */
/* sorted ascending: counting sort by source, then sort+unique per row.   */
/* head must hold n+1 entries, csr m_raw entries; returns m.             */
static int
cmp_u32(void const* a, void const* b)
{
  uint32_t const x = *(uint32_t const*)a, y = *(uint32_t const*)b;
  return x < y ? -1 : x > y;
}

uint64_t
orc_build_csr(uint32_t n, uint64_t m_raw, uint32_t const* src, uint32_t const* dst, uint64_t* head, uint32_t* csr)
{
  uint64_t* cnt = (uint64_t*)calloc((uint64_t)n + 1, sizeof(uint64_t));
  for (uint64_t e = 0; e < m_raw; ++e)
    if (src[e] != dst[e]) cnt[src[e] + 1] += 1;
  for (uint32_t i = 0; i < n; ++i) cnt[i + 1] += cnt[i];
  uint64_t* pos = (uint64_t*)malloc(sizeof(uint64_t) * ((uint64_t)n + 1));
  memcpy(pos, cnt, sizeof(uint64_t) * ((uint64_t)n + 1));
  for (uint64_t e = 0; e < m_raw; ++e)
    if (src[e] != dst[e]) csr[pos[src[e]]++] = dst[e];
  /* sort + unique each row in place, then compact */
  uint64_t* rowlen = (uint64_t*)malloc(sizeof(uint64_t) * ((uint64_t)n + 1));
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t u = 0; u < (int64_t)n; ++u) {
    uint32_t* row = csr + cnt[u];
    uint64_t  len = cnt[u + 1] - cnt[u];
    if (len > 1) qsort(row, len, sizeof(uint32_t), cmp_u32);
    uint64_t w = 0;
    for (uint64_t k = 0; k < len; ++k)
      if (w == 0 || row[w - 1] != row[k]) row[w++] = row[k];
    rowlen[u] = w;
  }
  uint64_t m = 0;
  head[0]    = 0;
  for (uint32_t u = 0; u < n; ++u) {
    uint64_t const beg = cnt[u];
    if (m != beg) memmove(csr + m, csr + beg, sizeof(uint32_t) * rowlen[u]);
    m += rowlen[u];
    head[u + 1] = m;
  }
  free(cnt);
  free(pos);
  free(rowlen);
  return m;
}

/* backward_complement_graph: kaspan/scc/backward_complement.hpp:22-68.   */
/* Counting-sort transpose; rows of the result come out ascending.        */
void
orc_transpose(uint32_t n, uint64_t const* fwh, uint32_t const* fwc, uint64_t* bwh, uint32_t* bwc)
{
  uint64_t const m = fwh[n];
  memset(bwh, 0, sizeof(uint64_t) * ((uint64_t)n + 1));
  for (uint64_t e = 0; e < m; ++e) bwh[fwc[e] + 1] += 1;
  for (uint32_t i = 0; i < n; ++i) bwh[i + 1] += bwh[i];
  uint64_t* pos = (uint64_t*)malloc(sizeof(uint64_t) * ((uint64_t)n + 1));
  memcpy(pos, bwh, sizeof(uint64_t) * ((uint64_t)n + 1));
  for (uint32_t u = 0; u < n; ++u)
    for (uint64_t e = fwh[u]; e < fwh[u + 1]; ++e) bwc[pos[fwc[e]]++] = u;
  free(pos);
}

/* ------------------------------------------------------------------ */
/* Planted-SCC generator, restating the strategy of                     */
/* kaspan/test/fuzzy.hpp:81-218 with this file's SplitMix64 stream in   */
/* place of std::mt19937 (so graphs differ from the reference's, the    */
/* construction does not):                                              */
/*  - vertex 0 starts a component; each later vertex starts a new one   */
/*    with p = 1/4, else joins a uniformly drawn existing one;          */
/*  - each component of size > 1 gets a random Hamiltonian cycle;       */
/*  - then, sweeping components in id order, random edges from the      */
/*    current component to itself or an earlier one are added until the */
/*    mean out-degree reaches d (clamped as the reference clamps it).   */
/* Planted id = component representative = its minimum vertex.         */
/* Writes fwh/fwc (rows ascending) and scc_id; returns m.  cap bounds   */
/* the edges written.                                                    */
/* ------------------------------------------------------------------ */
typedef struct
{
  uint64_t key, ctr;
} orc_rng;
static inline uint64_t
rng_next(orc_rng* r)
{
  return orc_draw(r->key, r->ctr++);
}
static inline uint64_t
rng_below(orc_rng* r, uint64_t bound) /* uniform in [0, bound) */
{
  return (uint64_t)(((__uint128_t)rng_next(r) * bound) >> 64);
}
static inline double
rng_unit(orc_rng* r)
{
  return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0);
}

typedef struct
{
  uint64_t* slot;
  uint64_t  mask;
} edge_set;
static int
edge_set_insert(edge_set* s, uint32_t u, uint32_t v)
{
  uint64_t const k = ((uint64_t)u << 32 | v) + 1;
  uint64_t       h = fmix64(k) & s->mask;
  for (;;) {
    if (s->slot[h] == 0) {
      s->slot[h] = k;
      return 1;
    }
    if (s->slot[h] == k) return 0;
    h = (h + 1) & s->mask;
  }
}

uint64_t
orc_fuzzy(uint64_t seed, uint32_t n, double d, uint32_t* scc_id, uint64_t* fwh, uint32_t* fwc, uint64_t cap)
{
  orc_rng rng = { orc_seed_key(seed), 0 };
  if (n < 2) d = -1.0;
  else {
    double const min_d = log(fmax(1.0, log((double)n)));
    double const max_d = (double)(n - 1) / 2.0;
    if (d == -1.0) d = min_d + (max_d - min_d) * rng_unit(&rng);
    else if (d < min_d) d = min_d;
    else if (d > max_d) d = max_d;
  }
  uint32_t* comp_of  = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t* reps     = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t* rep_idx  = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  uint32_t  nreps    = 0;
  for (uint32_t v = 0; v < n; ++v) {
    if (v == 0 || rng_below(&rng, 4) == 0) {
      rep_idx[v]    = nreps;
      reps[nreps++] = v;
      scc_id[v]     = v;
    } else {
      scc_id[v] = reps[rng_below(&rng, nreps)];
    }
  }
  /* members of each component, components in id order */
  uint32_t* cstart = (uint32_t*)calloc(nreps + 1, sizeof(uint32_t));
  uint32_t* member = (uint32_t*)malloc(sizeof(uint32_t) * (n + 1));
  for (uint32_t v = 0; v < n; ++v) cstart[rep_idx[scc_id[v]] + 1] += 1;
  for (uint32_t c = 0; c < nreps; ++c) cstart[c + 1] += cstart[c];
  {
    uint32_t* fill = (uint32_t*)malloc(sizeof(uint32_t) * (nreps + 1));
    memcpy(fill, cstart, sizeof(uint32_t) * (nreps + 1));
    for (uint32_t v = 0; v < n; ++v) member[fill[rep_idx[scc_id[v]]]++] = v;
    free(fill);
  }
  (void)comp_of;

  uint64_t cap_pow = 16;
  while (cap_pow < 2 * cap + 16) cap_pow <<= 1;
  edge_set  es    = { (uint64_t*)calloc(cap_pow, sizeof(uint64_t)), cap_pow - 1 };
  uint32_t* eu    = (uint32_t*)malloc(sizeof(uint32_t) * (cap + 1));
  uint32_t* ev    = (uint32_t*)malloc(sizeof(uint32_t) * (cap + 1));
  uint64_t  m     = 0;
#define TRY_ADD(U, V)                                                \
  do {                                                               \
    uint32_t const uu_ = (U), vv_ = (V);                             \
    if (uu_ != vv_ && m < cap && edge_set_insert(&es, uu_, vv_)) {   \
      eu[m] = uu_;                                                   \
      ev[m] = vv_;                                                   \
      ++m;                                                           \
    }                                                                \
  } while (0)

  for (uint32_t c = 0; c < nreps; ++c) {
    uint32_t* comp = member + cstart[c];
    uint32_t  sz   = cstart[c + 1] - cstart[c];
    if (sz > 1) {
      for (uint32_t i = sz - 1; i > 0; --i) { /* Fisher-Yates */
        uint32_t const j = (uint32_t)rng_below(&rng, (uint64_t)i + 1);
        uint32_t const t = comp[i];
        comp[i]          = comp[j];
        comp[j]          = t;
      }
      TRY_ADD(comp[0], comp[sz - 1]);
      for (uint32_t i = 1; i < sz; ++i) TRY_ADD(comp[i], comp[i - 1]);
    }
  }
  if (n > 0) {
    uint64_t guard = 0;
    while ((double)m / n < d && m < cap && guard++ < 1000000) {
      for (uint32_t c = 0; c < nreps; ++c) {
        uint32_t const  szu   = cstart[c + 1] - cstart[c];
        uint32_t const* compu = member + cstart[c];
        for (uint32_t i = 0; i < szu; ++i) {
          if ((double)m / n >= d) break;
          uint32_t const  cv    = (uint32_t)rng_below(&rng, (uint64_t)c + 1);
          uint32_t const  szv   = cstart[cv + 1] - cstart[cv];
          uint32_t const* compv = member + cstart[cv];
          uint32_t const  u     = compu[rng_below(&rng, szu)];
          uint32_t const  v     = compv[rng_below(&rng, szv)];
          TRY_ADD(u, v);
        }
      }
    }
  }
#undef TRY_ADD
  uint64_t const mm = orc_build_csr(n, m, eu, ev, fwh, fwc);
  free(es.slot);
  free(eu);
  free(ev);
  free(reps);
  free(rep_idx);
  free(cstart);
  free(member);
  free(comp_of);
  return mm;
}
