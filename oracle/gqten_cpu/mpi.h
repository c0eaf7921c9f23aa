/*
 * Single-rank MPI stand-in used ONLY to compile the reference's unchanged
 * tnbp apps and headers into the CPU oracle (oracle/_ref).  Test
 * infrastructure: nothing in the product links it.
 *
 * The reference includes "mpi.h" unconditionally
 * (include/tnbp/framework/mpiutility.h:9) and its apps call MPI_Init /
 * MPI_Allreduce / MPI_Finalize directly (apps/estimator/main.cc:18,228,241;
 * apps/kicked_ising_lattice/main.cc:23).  With one rank:
 *   - size = 1, rank = 0;
 *   - Allreduce(SUM) is a copy of the send buffer into the receive buffer;
 *   - Bcast is a no-op;
 *   - Send/Recv can only be reached when a boundary message crosses ranks,
 *     which never happens with one rank (bp.h:229-257, measure.h:247-253);
 *     they abort loudly if reached.
 */
#ifndef TNBP_ORACLE_SINGLE_RANK_MPI_H
#define TNBP_ORACLE_SINGLE_RANK_MPI_H

#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_SUM 1

/* datatype handle == element size in bytes (enough for a copying Allreduce) */
#define MPI_CHAR ((MPI_Datatype)sizeof(char))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_INT32_T ((MPI_Datatype)sizeof(int32_t))
#define MPI_UINT32_T ((MPI_Datatype)sizeof(uint32_t))
#define MPI_FLOAT ((MPI_Datatype)sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_CXX_FLOAT_COMPLEX ((MPI_Datatype)sizeof(std::complex<float>))
#define MPI_CXX_DOUBLE_COMPLEX ((MPI_Datatype)sizeof(std::complex<double>))

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }

inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype dt,
                         MPI_Op, MPI_Comm) {
  if (send != recv && count > 0) std::memmove(recv, send, (size_t)count * (size_t)dt);
  return MPI_SUCCESS;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
  std::fprintf(stderr, "single-rank MPI stand-in: MPI_Send reached\n");
  std::abort();
}
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
  std::fprintf(stderr, "single-rank MPI stand-in: MPI_Recv reached\n");
  std::abort();
}

#endif
