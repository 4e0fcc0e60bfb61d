/*
 * CPU CHECKER - test infrastructure only.  Compiles the reference's own
 * header-only SCC code (rawbby/KaSpan, kaspan/include) as a single rank
 * against the stand-ins in oracle/ref_shim, and exports its entry points
 * with a C ABI so tests and the bench's reference arm can call them.
 * Nothing in the product library links this; the product never calls it.
 *
 * Graph layout at this boundary: n vertices, u64 offsets (the reference
 * built with KASPAN_INDEX64), u32 neighbour ids, forward CSR plus its
 * transpose.  Vertex state is the reference's own bitset layout: u64 words,
 * bit k of word k/64 set = vertex k undecided.
 */
#include <kaspan/graph/base.hpp>
#include <kaspan/graph/bidi_graph_part.hpp>
#include <kaspan/graph/single_part.hpp>
#include <kaspan/memory/bits.hpp>
#include <kaspan/memory/hash_map.hpp>
#include <kaspan/memory/hash_set.hpp>
#include <kaspan/scc/cache_multi_pivot_search_pull.hpp>
#include <kaspan/scc/cache_pivot_search.hpp>
#include <kaspan/scc/frontier.hpp>
#include <kaspan/scc/pivot.hpp>
#include <kaspan/scc/scc.hpp>
#include <kaspan/scc/tarjan.hpp>
#include <kaspan/scc/trim_1_exhaustive.hpp>
#include <kaspan/scc/trim_1_local.hpp>
#include <kaspan/scc/adapter/manifest.hpp>
#include <kaspan/scc/variant/scc_hpc_like.hpp>
#include <kaspan/scc/variant/scc_hpc_trim_ex.hpp>
#include <kaspan/scc/variant/scc_ispan_like.hpp>
#include <kaspan/scc/variant/scc_trim_ex.hpp>
#include <kaspan/scc/variant/scc_trim_ex_light_residual.hpp>
#include <kaspan/scc/variant/scc_trim_ex_residual.hpp>
#include <kaspan/test/normalise_scc.hpp>

#include <algorithm>
#include <chrono>
#include <cstdint>

static_assert(sizeof(kaspan::index_t) == 8, "build the checker with -DKASPAN_INDEX64");
static_assert(sizeof(kaspan::vertex_t) == 4, "u32 vertex ids expected");

using namespace kaspan;

namespace {

void
ensure_init()
{
  static bool done = false;
  if (done) return;
  // KASPAN_DEFAULT_INIT() without the MPI_Init/MPI_Finalize scope guard,
  // which only makes sense inside main().
  mpi_basic::world_rank = 0;
  mpi_basic::world_size = 1;
  mpi_basic::world_root = true;
  init_mpi_edge_t();
  init_mpi_labeled_edge_t();
  init_mpi_degree_t();
  init_mpi_degree_max_op();
  done = true;
}

auto
make_view(uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc)
{
  return bidi_graph_part_view<single_part_view>{ single_part_view{ n }, m, m, fwh, fwc, bwh, bwc };
}

int64_t
now_ns()
{
  return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

} // namespace

extern "C" {

/* kaspan::scc (kaspan/scc/scc.hpp:21-87) or one of its six variants
 * (kaspan/scc/variant/*.hpp).  variant: 0 scc, 1 hpc_like, 2 hpc_trim_ex,
 * 3 ispan_like, 4 trim_ex, 5 trim_ex_light_residual, 6 trim_ex_residual.
 * Returns the wall time of the call in ns, or -1 for an unknown variant. */
int64_t
kref_scc(int variant, uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc, uint32_t* scc_id)
{
  ensure_init();
  auto       g  = make_view(n, m, fwh, fwc, bwh, bwc);
  auto const t0 = now_ns();
  switch (variant) {
    case 0: scc(g, scc_id); break;
    case 1: scc_hpc_like(g, scc_id); break;
    case 2: scc_hpc_trim_ex(g, scc_id); break;
    case 3: scc_ispan_like(g, scc_id); break;
    case 4: scc_trim_ex(g, scc_id); break;
    case 5: scc_trim_ex_light_residual(g, scc_id); break;
    case 6: scc_trim_ex_residual(g, scc_id); break;
    default: return -1;
  }
  return now_ns() - t0;
}

/* kaspan::tarjan (kaspan/scc/tarjan.hpp:124-136) over the forward CSR; each
 * SCC is named by its minimum member, as test_tarjan_vs_kaspan.cpp:37-45
 * does.  Returns ns. */
int64_t
kref_tarjan(uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint32_t* scc_id)
{
  ensure_init();
  auto const gv = graph_view{ n, m, fwh, fwc };
  auto const t0 = now_ns();
  tarjan(gv, [&](auto const* beg, auto const* end) {
    auto const id = *std::min_element(beg, end);
    for (auto const* it = beg; it != end; ++it) scc_id[*it] = id;
  });
  return now_ns() - t0;
}

/* kaspan::normalise_scc_id (kaspan/test/normalise_scc.hpp:10-25). */
void
kref_normalise(uint32_t n, uint32_t* scc_id)
{
  normalise_scc_id<vertex_t>(n, scc_id);
}

/* trim_1_first (kaspan/scc/trim_1_local.hpp:12-46).  undecided must hold
 * ceil(n/64) words, all bits of [0,n) set on entry. Returns the pivot. */
uint32_t
kref_trim_1_first(uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc, uint64_t* undecided, uint32_t* scc_id)
{
  ensure_init();
  auto g = make_view(n, m, fwh, fwc, bwh, bwc);
  return trim_1_first(g, undecided, [&](auto k, auto id) { scc_id[k] = id; });
}

/* cache_forward_backward_search (kaspan/scc/cache_pivot_search.hpp:16-104). */
void
kref_fw_bw(uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc, uint64_t* undecided, uint32_t* scc_id, uint32_t pivot)
{
  ensure_init();
  auto g          = make_view(n, m, fwh, fwc, bwh, bwc);
  auto front      = frontier{ n };
  auto active     = make_array<vertex_t>(n);
  auto is_reached = make_bits(n);
  auto cache      = hash_set<vertex_t>{ 2 * m };
  cache_forward_backward_search(g, front, active.data(), is_reached.data(), undecided, pivot, [&](auto k, auto id) { scc_id[k] = id; }, cache);
}

/* trim_1_normal (kaspan/scc/trim_1_local.hpp:48-73). */
void
kref_trim_1_normal(uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc, uint64_t* undecided, uint32_t* scc_id)
{
  ensure_init();
  auto g = make_view(n, m, fwh, fwc, bwh, bwc);
  trim_1_normal(g, undecided, [&](auto k, auto id) { scc_id[k] = id; });
}

/* One call of cache_label_search_pull (kaspan/scc/cache_multi_pivot_search_pull.hpp:40-244)
 * with map = rotr(., rotation), unmap = rotl(., rotation): the body of
 * cache_rot_label_search_pull (:246-266) with the rotation passed in
 * instead of read from its process-global counter. */
void
kref_label_search_pull(uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc, uint64_t* undecided, uint32_t* scc_id, int rotation)
{
  ensure_init();
  auto g           = make_view(n, m, fwh, fwc, bwh, bwc);
  auto front       = frontier{ n };
  auto label       = make_array<vertex_t>(n);
  auto active      = make_array<vertex_t>(n);
  auto in_active   = make_bits(n);
  auto has_changed = make_bits_clean(n);
  auto cache       = hash_map<vertex_t>{ 2 * m };
  auto const map   = [rotation](vertex_t l) { return std::rotr(l, rotation); };
  auto const unmap = [rotation](vertex_t l) { return std::rotl(l, rotation); };
  cache_label_search_pull(g, front, label.data(), active.data(), in_active.data(), has_changed.data(), undecided, [&](auto k, auto id) { scc_id[k] = id; }, map, unmap, cache);
}

/* trim_1_exhaustive_first (kaspan/scc/trim_1_exhaustive.hpp:71-131); also
 * returns the live degree arrays it leaves behind. */
void
kref_trim_1_exhaustive_first(uint32_t n, uint64_t m, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc, uint64_t* undecided, uint32_t* scc_id, uint32_t* outdegree, uint32_t* indegree)
{
  ensure_init();
  auto g     = make_view(n, m, fwh, fwc, bwh, bwc);
  auto front = frontier{ n };
  trim_1_exhaustive_first(g, undecided, outdegree, indegree, front.view<vertex_t>(), [&](auto k, auto id) { scc_id[k] = id; });
}

/* select_pivot_from_degree (kaspan/scc/pivot.hpp:53-74). */
uint32_t
kref_select_pivot_from_degree(uint32_t n, uint64_t* undecided, uint32_t const* outdegree, uint32_t const* indegree)
{
  ensure_init();
  return select_pivot_from_degree(single_part_view{ n }, undecided, outdegree, indegree);
}

/* The reference's manifest reader and loader (kaspan/scc/adapter/
 * manifest.hpp:132-245): *n_out / *m_out from the manifest; with arrays
 * given (n + 1 heads, m ids each), the graph as load_graph_from_manifest
 * builds it.  Returns 0, or -1 when the files cannot be read. */
int
kref_manifest_load(char const* path, uint64_t* n_out, uint64_t* m_out, uint64_t* fwh, uint32_t* fwc, uint64_t* bwh, uint32_t* bwc)
{
  ensure_init();
  try {
    auto const mf = manifest::load(path);
    *n_out        = mf.graph_node_count;
    *m_out        = mf.graph_edge_count;
    if (!fwh) return 0;
    auto const g = load_graph_from_manifest(mf);
    for (uint64_t i = 0; i <= mf.graph_node_count; ++i) fwh[i] = g.fw.head[i], bwh[i] = g.bw.head[i];
    for (uint64_t i = 0; i < mf.graph_edge_count; ++i) fwc[i] = g.fw.csr[i], bwc[i] = g.bw.csr[i];
    return 0;
  } catch (...) {
    return -1;
  }
}

} // extern "C"
