/* Stand-in for KaMPIng's datatype header: the reference only specialises
 * this trait (kaspan/graph/base.hpp), it never calls into KaMPIng.
 * Test infrastructure for the CPU checker under oracle/_ref. */
#pragma once
namespace kamping {
template<class T>
struct mpi_type_traits;
}
