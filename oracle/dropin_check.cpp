/*
 * CPU CHECKER - test infrastructure only.  Exercises the C++ drop-in
 * include/kaspan_b200/scc.hpp the way a reference caller would: it builds
 * the reference's own bidi_graph_part_view<single_part_view>
 * (kaspan/graph/bidi_graph_part.hpp:12-28) over host CSR/CSC arrays, calls
 * kaspan::scc (kaspan/scc/scc.hpp:21-87) + normalise_scc_id
 * (kaspan/test/normalise_scc.hpp:10-25) and kaspan_b200::scc on the same
 * view, and compares the two id arrays bit for bit.
 *
 * Built twice by oracle/Makefile (reference headers + the ref_shim
 * stand-ins): with -DKASPAN_INDEX64 (u64 offsets, passed through) and
 * without it (the reference's default u32 index_t, which the drop-in widens
 * on the host).  Runs on a GPU; exit status 0 when every graph agrees.
 */
#include <kaspan/graph/base.hpp>
#include <kaspan/graph/bidi_graph_part.hpp>
#include <kaspan/graph/single_part.hpp>
#include <kaspan/scc/scc.hpp>
#include <kaspan/test/normalise_scc.hpp>

#include <kaspan_b200/scc.hpp>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

using namespace kaspan;

namespace {

struct host_graph
{
  std::string           name;
  vertex_t              n = 0;
  std::vector<index_t>  fwh, bwh;
  std::vector<vertex_t> fwc, bwc;
};

uint64_t
splitmix(uint64_t& s)
{
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// CSR of an edge list (rows ascending by source, entries in input order)
void
to_csr(vertex_t n, std::vector<vertex_t> const& from, std::vector<vertex_t> const& to, std::vector<index_t>& head, std::vector<vertex_t>& csr)
{
  head.assign(static_cast<size_t>(n) + 1, 0);
  for (auto u : from) ++head[u + 1];
  for (vertex_t u = 0; u < n; ++u) head[u + 1] += head[u];
  csr.assign(from.size() ? from.size() : 1, 0);
  std::vector<index_t> pos(head.begin(), head.end() - 1);
  for (size_t i = 0; i < from.size(); ++i) csr[pos[from[i]]++] = to[i];
}

host_graph
make(std::string name, vertex_t n, std::vector<vertex_t> const& src, std::vector<vertex_t> const& dst)
{
  host_graph g;
  g.name = std::move(name);
  g.n    = n;
  to_csr(n, src, dst, g.fwh, g.fwc);
  to_csr(n, dst, src, g.bwh, g.bwc);
  return g;
}

std::vector<host_graph>
graphs()
{
  std::vector<host_graph> out;
  // extern/ispan_test/test_ispan_tiny.cpp:21-90: 7 vertices, 11 edges
  out.push_back(make("kat", 7, { 0, 1, 1, 1, 2, 3, 3, 4, 4, 5, 6 }, { 2, 0, 2, 3, 0, 2, 4, 1, 3, 6, 5 }));
  out.push_back(make("single", 1, {}, {}));
  uint64_t s = 42;
  for (auto [n, m] : { std::pair<vertex_t, size_t>{ 3000, 3300 }, { 3000, 12000 }, { 1u << 16, 1u << 19 } }) {
    std::vector<vertex_t> a, b;
    for (size_t i = 0; i < m; ++i) {
      vertex_t const u = static_cast<vertex_t>(splitmix(s) % n), v = static_cast<vertex_t>(splitmix(s) % n);
      a.push_back(u), b.push_back(v); // duplicates and self-loops kept: the boundary allows them
    }
    out.push_back(make("gnm_" + std::to_string(n) + "_" + std::to_string(m), n, a, b));
  }
  // cycles of growing length joined one way, plus a tail
  {
    std::vector<vertex_t> a, b;
    vertex_t              base = 0;
    for (vertex_t len = 1; len <= 64; ++len) {
      for (vertex_t i = 0; i < len; ++i) a.push_back(base + i), b.push_back(base + (i + 1) % len);
      if (base) a.push_back(base - 1), b.push_back(base);
      base += len;
    }
    out.push_back(make("cycles", base, a, b));
  }
  return out;
}

} // namespace

int
main()
{
  // KASPAN_DEFAULT_INIT() at one rank, without its MPI_Init/Finalize guard
  mpi_basic::world_rank = 0;
  mpi_basic::world_size = 1;
  mpi_basic::world_root = true;
  init_mpi_edge_t();
  init_mpi_labeled_edge_t();
  init_mpi_degree_t();
  init_mpi_degree_max_op();
  int bad = 0;
  for (auto& g : graphs()) {
    index_t const m    = g.fwh[g.n];
    auto          view = bidi_graph_part_view<single_part_view>{ single_part_view{ g.n }, m, m, g.fwh.data(), g.fwc.data(), g.bwh.data(), g.bwc.data() };
    std::vector<vertex_t> want(g.n), got(g.n, 0xDEADBEEFu);
    kaspan::scc(view, want.data());
    normalise_scc_id<vertex_t>(g.n, want.data());
    try {
      kaspan_b200::scc(view, got.data());
    } catch (kaspan_b200::error const& e) {
      std::printf("%s: kaspan_b200::scc threw: %s\n", g.name.c_str(), e.what());
      ++bad;
      continue;
    }
    bool const same = want == got;
    std::printf("%s: n=%u m=%llu index_t=%zu bytes: %s\n", g.name.c_str(), g.n, static_cast<unsigned long long>(m), sizeof(index_t), same ? "equal" : "DIFFERENT");
    bad += same ? 0 : 1;
  }
  std::printf(bad ? "dropin check FAILED\n" : "dropin check ok\n");
  return bad ? 1 : 0;
}
