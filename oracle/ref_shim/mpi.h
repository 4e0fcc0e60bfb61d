/*
 * Single-rank stand-in for <mpi.h>, used ONLY to compile the reference's
 * own header-only SCC code (kaspan/include) into the CPU checker under
 * oracle/_ref.  Test infrastructure, never part of the product library.
 *
 * Semantics: one process, rank 0 of a world of size 1.  Every collective is
 * a copy of the local contribution (count x extent bytes); reductions of one
 * contributor are the identity, so user ops are never invoked.  Datatypes
 * are small integers into a table of sizes; derived struct types get an
 * entry sized by their blocks so extents stay right for edge_t / degree_t.
 */
#pragma once
#include <cstddef>
#include <cstdint>
#include <cstring>

typedef long long MPI_Count;
typedef long long MPI_Aint;
typedef int       MPI_Datatype;
typedef int       MPI_Op;
typedef int       MPI_Comm;
typedef void(MPI_User_function)(void*, void*, int*, MPI_Datatype*);

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1

#define MPI_DATATYPE_NULL 0
#define MPI_BYTE 1
#define MPI_INT8_T 2
#define MPI_INT16_T 3
#define MPI_INT32_T 4
#define MPI_INT64_T 5
#define MPI_UINT8_T 6
#define MPI_UINT16_T 7
#define MPI_UINT32_T 8
#define MPI_UINT64_T 9
#define MPI_FLOAT 10
#define MPI_DOUBLE 11
#define MPI_COUNT 12
#define KSPN_SHIM_FIRST_DERIVED 16
#define KSPN_SHIM_MAX_TYPES 64

#define MPI_OP_NULL 0
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_LOR 4
#define MPI_LAND 5

#define MPI_IN_PLACE (reinterpret_cast<void*>(static_cast<std::intptr_t>(-1)))

namespace kspn_shim {
inline MPI_Aint type_sizes[KSPN_SHIM_MAX_TYPES] = { 0, 1, 1, 2, 4, 8, 1, 2, 4, 8, 4, 8, 8 };
inline int      next_type                       = KSPN_SHIM_FIRST_DERIVED;
inline int      next_op                         = 16;
inline MPI_Aint size_of(MPI_Datatype t) { return (t >= 0 && t < KSPN_SHIM_MAX_TYPES) ? type_sizes[t] : 0; }
inline void     copy(void const* src, void* dst, MPI_Count count, MPI_Datatype t)
{
  if (src == MPI_IN_PLACE || src == dst || count <= 0) return;
  std::memmove(dst, src, static_cast<std::size_t>(count * size_of(t)));
}
} // namespace kspn_shim

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Get_address(void const* p, MPI_Aint* a) { *a = reinterpret_cast<MPI_Aint>(p); return MPI_SUCCESS; }

inline int MPI_Type_create_struct(int count, int const* blocklengths, MPI_Aint const* displs, MPI_Datatype const* types, MPI_Datatype* out)
{
  MPI_Aint extent = 0;
  for (int i = 0; i < count; ++i) {
    MPI_Aint const end = displs[i] + blocklengths[i] * kspn_shim::size_of(types[i]);
    if (end > extent) extent = end;
  }
  if (kspn_shim::next_type >= KSPN_SHIM_MAX_TYPES) return 1;
  kspn_shim::type_sizes[kspn_shim::next_type] = extent;
  *out = kspn_shim::next_type++;
  return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype* t) { *t = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
inline int MPI_Type_get_extent(MPI_Datatype t, MPI_Aint* lb, MPI_Aint* extent) { *lb = 0; *extent = kspn_shim::size_of(t); return MPI_SUCCESS; }
inline int MPI_Type_size(MPI_Datatype t, int* s) { *s = static_cast<int>(kspn_shim::size_of(t)); return MPI_SUCCESS; }
inline int MPI_Op_create(MPI_User_function*, int, MPI_Op* op) { *op = kspn_shim::next_op++; return MPI_SUCCESS; }
inline int MPI_Op_free(MPI_Op* op) { *op = MPI_OP_NULL; return MPI_SUCCESS; }

inline int MPI_Allreduce_c(void const* send, void* recv, MPI_Count count, MPI_Datatype t, MPI_Op, MPI_Comm)
{
  kspn_shim::copy(send, recv, count, t);
  return MPI_SUCCESS;
}
inline int MPI_Allgather_c(void const* send, MPI_Count sc, MPI_Datatype st, void* recv, MPI_Count, MPI_Datatype, MPI_Comm)
{
  kspn_shim::copy(send, recv, sc, st);
  return MPI_SUCCESS;
}
inline int MPI_Allgatherv_c(void const* send, MPI_Count sc, MPI_Datatype st, void* recv, MPI_Count const*, MPI_Aint const* displs, MPI_Datatype rt, MPI_Comm)
{
  kspn_shim::copy(send, static_cast<char*>(recv) + displs[0] * kspn_shim::size_of(rt), sc, st);
  return MPI_SUCCESS;
}
inline int MPI_Alltoall_c(void const* send, MPI_Count sc, MPI_Datatype st, void* recv, MPI_Count, MPI_Datatype, MPI_Comm)
{
  kspn_shim::copy(send, recv, sc, st);
  return MPI_SUCCESS;
}
inline int MPI_Alltoallv_c(void const* send, MPI_Count const* sc, MPI_Aint const* sd, MPI_Datatype st, void* recv, MPI_Count const*, MPI_Aint const* rd, MPI_Datatype rt, MPI_Comm)
{
  kspn_shim::copy(static_cast<char const*>(send) + sd[0] * kspn_shim::size_of(st), static_cast<char*>(recv) + rd[0] * kspn_shim::size_of(rt), sc[0], st);
  return MPI_SUCCESS;
}
inline int MPI_Gather_c(void const* send, MPI_Count sc, MPI_Datatype st, void* recv, MPI_Count, MPI_Datatype, int, MPI_Comm)
{
  kspn_shim::copy(send, recv, sc, st);
  return MPI_SUCCESS;
}
inline int MPI_Gatherv_c(void const* send, MPI_Count sc, MPI_Datatype st, void* recv, MPI_Count const*, MPI_Aint const* displs, MPI_Datatype rt, int, MPI_Comm)
{
  if (recv) kspn_shim::copy(send, static_cast<char*>(recv) + displs[0] * kspn_shim::size_of(rt), sc, st);
  return MPI_SUCCESS;
}
