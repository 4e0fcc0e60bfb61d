// Header-only C++ drop-in over the kspn C ABI for single-rank callers of
// rawbby/KaSpan's
//
//     template<part_view_c Part = single_part_view>
//     void kaspan::scc(bidi_graph_part_view<Part> graph, vertex_t* scc_id);   // kaspan/scc/scc.hpp:21-25
//
// Usage: keep building the reference's bidi_graph_part_view (or any struct
// with the same members: part.n(), part.world_size(), local_fw_m,
// fw.head/fw.csr, bw.head/bw.csr) and call kaspan_b200::scc(graph, scc_id).
//
// Same argument meaning as the reference: graph is a non-owning view of the
// forward CSR and its transpose with u32 vertex ids; scc_id[n] is caller
// owned and fully overwritten.  Differences a caller may notice:
//   * ids are the MINIMUM member of each component (the reference writes
//     some member; normalise_scc_id, kaspan/test/normalise_scc.hpp:10-25,
//     maps both to the same array);
//   * failures throw kaspan_b200::error (the reference's ASSERT aborts,
//     kaspan/debug/assert.hpp:120-148);
//   * one rank only: a view whose part.world_size() != 1 is rejected.
// index_t of 32 bits (the reference's default without KASPAN_INDEX64) is
// widened to the u64 offsets of the C ABI on the host.
#pragma once

#include "../kspn.h"

#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace kaspan_b200 {

class error : public std::runtime_error
{
public:
  error(int status, std::string const& what)
    : std::runtime_error(std::string(kspn_strerror(status)) + ": " + what)
    , status(status)
  {
  }
  int status;
};

// One context per thread, created on first use on the thread's current
// CUDA device (cudaGetDevice at that first call; a later device change on
// the thread is not followed).  Contexts are not shared between threads.
inline kspn_context*
thread_context()
{
  struct holder
  {
    kspn_context* ctx = nullptr;
    ~holder() { kspn_context_destroy(ctx); }
  };
  thread_local holder h;
  if (!h.ctx) {
    int const rc = kspn_context_create(KSPN_DEVICE_CURRENT, &h.ctx);
    if (rc != KSPN_OK) throw error(rc, "kspn_context_create");
  }
  return h.ctx;
}

template<typename View>
void
scc(View graph, std::uint32_t* scc_id, kspn_options const* options = nullptr, kspn_stats* stats = nullptr)
{
  using head_t = std::remove_cv_t<std::remove_pointer_t<decltype(graph.fw.head)>>;
  using csr_t  = std::remove_cv_t<std::remove_pointer_t<decltype(graph.fw.csr)>>;
  static_assert(sizeof(csr_t) == 4, "kspn takes u32 vertex ids (the reference's default vertex_t)");
  static_assert(sizeof(head_t) == 4 || sizeof(head_t) == 8, "index_t must be 32 or 64 bits");
  if (graph.part.world_size() != 1) throw error(KSPN_ERR_INVALID_ARGUMENT, "kaspan_b200::scc decomposes one rank's whole graph");

  auto const          n = static_cast<std::uint32_t>(graph.part.n());
  auto const          m = static_cast<std::uint64_t>(graph.local_fw_m);
  std::uint64_t const* fwh;
  std::uint64_t const* bwh;
  std::vector<std::uint64_t> wide_fw, wide_bw;
  if constexpr (sizeof(head_t) == 8) {
    fwh = reinterpret_cast<std::uint64_t const*>(graph.fw.head);
    bwh = reinterpret_cast<std::uint64_t const*>(graph.bw.head);
  } else {
    wide_fw.assign(graph.fw.head, graph.fw.head + n + 1);
    wide_bw.assign(graph.bw.head, graph.bw.head + n + 1);
    fwh = wide_fw.data();
    bwh = wide_bw.data();
  }
  kspn_context* ctx = thread_context();
  int const     rc  = kspn_scc(ctx, n, m, fwh, reinterpret_cast<std::uint32_t const*>(graph.fw.csr), bwh, reinterpret_cast<std::uint32_t const*>(graph.bw.csr), scc_id, options, stats);
  if (rc != KSPN_OK) throw error(rc, kspn_last_error(ctx));
}

} // namespace kaspan_b200
