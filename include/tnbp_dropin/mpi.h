/* One-process MPI for tnbp's apps running on tnbp_b200.
 *
 * tnbp includes "mpi.h" unconditionally (include/tnbp/framework/mpiutility.h)
 * and its apps call MPI_Init / MPI_Comm_size / MPI_Comm_rank / MPI_Allreduce /
 * MPI_Finalize themselves (apps/estimator/main.cc, apps/kicked_ising_lattice/
 * main.cc).  On tnbp_b200 a process owns one GPU and one whole lattice (the
 * engine does not split a lattice across ranks), so the communicator has
 * exactly one rank:
 *   - MPI_Comm_size = 1, MPI_Comm_rank = 0;
 *   - MPI_Allreduce over one rank is the identity (the receive buffer gets the
 *     send buffer); MPI_Bcast from rank 0 to itself changes nothing;
 *   - point-to-point calls can only be reached when a message crosses ranks,
 *     which one rank never does; reaching one throws std::logic_error.
 * Datatypes carry their element size, which is all the identity reduction
 * needs.
 */
#ifndef TNBP_DROPIN_MPI_H
#define TNBP_DROPIN_MPI_H

#include <complex>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <stdexcept>

typedef int MPI_Comm;
typedef int MPI_Op;
typedef std::size_t MPI_Datatype;  // element size in bytes
struct MPI_Status {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
};

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_SUM 1
#define MPI_MAX 2

#define MPI_CHAR (sizeof(char))
#define MPI_INT (sizeof(int))
#define MPI_INT32_T (sizeof(std::int32_t))
#define MPI_UINT32_T (sizeof(std::uint32_t))
#define MPI_INT64_T (sizeof(std::int64_t))
#define MPI_FLOAT (sizeof(float))
#define MPI_DOUBLE (sizeof(double))
#define MPI_CXX_FLOAT_COMPLEX (sizeof(std::complex<float>))
#define MPI_CXX_DOUBLE_COMPLEX (sizeof(std::complex<double>))

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* n) {
  *n = 1;
  return MPI_SUCCESS;
}
inline int MPI_Comm_rank(MPI_Comm, int* r) {
  *r = 0;
  return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (in != out && count > 0) std::memmove(out, in, static_cast<std::size_t>(count) * t);
  return MPI_SUCCESS;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) {
  throw std::logic_error("MPI_Send on a one-rank communicator (tnbp_b200 runs one lattice per process)");
}
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
  throw std::logic_error("MPI_Recv on a one-rank communicator (tnbp_b200 runs one lattice per process)");
}

#endif
