/*
 * Stand-in for the reference's cache-line allocator header
 * (kaspan/memory/line.hpp), used ONLY to compile the reference's own SCC
 * code into the CPU checker under oracle/_ref.  Test infrastructure.
 *
 * Why it exists: the reference rounds an allocation up to whole cache
 * lines with a mask of its 32-bit line size, and `~mask` widens with zeros,
 * so every request of 4 GiB or more loses its upper 32 bits.  kaspan::scc
 * at one rank allocates its FW-BW hash set (kaspan/scc/scc.hpp:53, 6 bytes
 * per edge rounded up to a power of two of cache lines) at exactly 4 GiB for
 * an R-MAT scale-24 graph, receives a 0-byte block and overwrites the heap.
 * (With MPI and several ranks each rank's share stays below 4 GiB.)  This
 * header offers the same names and meaning -- cache-line size, alignment
 * helpers, line-aligned allocation and release -- with every size computed
 * in 64 bits; it is found before the reference's own header because
 * ref_shim/ comes first on the include path.  Nothing else changes.
 */
#pragma once

#include <kaspan/util/arithmetic.hpp>

#include <bit>
#include <cstdint>
#include <cstdlib>
#include <new>
#include <type_traits>
#include <unistd.h>

namespace kaspan {

namespace shim_detail {
inline std::uint64_t
line_bytes()
{
  static std::uint64_t const v = [] {
    long const s = sysconf(_SC_LEVEL1_DCACHE_LINESIZE);
    return s > 0 && std::has_single_bit(static_cast<unsigned long>(s)) ? static_cast<std::uint64_t>(s) : std::uint64_t{ 64 };
  }();
  return v;
}
} // namespace shim_detail

template<unsigned_c Size = u32>
auto
linesize() -> Size
{
  return static_cast<Size>(shim_detail::line_bytes());
}

template<unsigned_c Size>
auto
line_align_down(Size size) -> Size
{
  return static_cast<Size>(static_cast<std::uint64_t>(size) & ~(shim_detail::line_bytes() - 1));
}

template<unsigned_c Size>
auto
line_align_up(Size size) -> Size
{
  std::uint64_t const mask = shim_detail::line_bytes() - 1;
  return static_cast<Size>((static_cast<std::uint64_t>(size) + mask) & ~mask);
}

template<unsigned_c Size>
auto
is_line_aligned(Size size) -> bool
{
  return (static_cast<std::uint64_t>(size) & (shim_detail::line_bytes() - 1)) == 0;
}

inline auto line_align_down(void const* p) { return reinterpret_cast<void const*>(line_align_down(reinterpret_cast<std::uint64_t>(p))); }
inline auto line_align_up(void const* p) { return reinterpret_cast<void const*>(line_align_up(reinterpret_cast<std::uint64_t>(p))); }
inline auto is_line_aligned(void const* p) { return is_line_aligned(reinterpret_cast<std::uint64_t>(p)); }
inline auto line_align_down(void* p) { return reinterpret_cast<void*>(line_align_down(reinterpret_cast<std::uint64_t>(p))); }
inline auto line_align_up(void* p) { return reinterpret_cast<void*>(line_align_up(reinterpret_cast<std::uint64_t>(p))); }

// `size` elements of T (bytes for T = void), line-aligned; nullptr for 0.
template<typename T = void>
[[nodiscard]] auto
line_alloc(integral_c auto size) noexcept(false) -> T*
{
  using elem_t              = std::conditional_t<std::is_same_v<T, void>, byte, T>;
  std::uint64_t const bytes = static_cast<std::uint64_t>(size) * sizeof(elem_t);
  if (bytes == 0) return nullptr;
  std::uint64_t const line = shim_detail::line_bytes();
  void* const         p    = std::aligned_alloc(line, (bytes + line - 1) & ~(line - 1));
  if (!p) throw std::bad_alloc{};
  return static_cast<T*>(p);
}

inline void
line_free(void* p)
{
  std::free(p);
}

} // namespace kaspan
