/*
 * Single-rank stand-in for the handful of MPI names that the reference
 * headers touch when they are compiled for the oracle (test infrastructure
 * only).  Every communicator has exactly one rank; collectives copy.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H
#include <complex>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_FLOAT 5
#define MPI_C_COMPLEX 9
#define MPI_C_DOUBLE_COMPLEX 16
#define MPI_DATATYPE_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)1)

inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int oracle_mpi_size(MPI_Datatype t) {
  return t == MPI_DOUBLE ? 8 : t == MPI_C_COMPLEX ? 8 : t == MPI_C_DOUBLE_COMPLEX ? 16 : 4;
}
inline int MPI_Scatter(const void* s, int sc, MPI_Datatype st, void* r, int,
                       MPI_Datatype, int, MPI_Comm) {
  if (r != s) std::memcpy(r, s, (size_t)sc * oracle_mpi_size(st));
  return 0;
}
inline int MPI_Scatterv(const void* s, const int* sc, const int* disp,
                        MPI_Datatype st, void* r, int, MPI_Datatype, int,
                        MPI_Comm) {
  std::memcpy(r, (const char*)s + (size_t)disp[0] * oracle_mpi_size(st),
              (size_t)sc[0] * oracle_mpi_size(st));
  return 0;
}
inline int MPI_Allreduce(const void* s, void* r, int c, MPI_Datatype t, MPI_Op,
                         MPI_Comm) {
  if (s != MPI_IN_PLACE && s != r)
    std::memcpy(r, s, (size_t)c * oracle_mpi_size(t));
  return 0;
}
// One rank: an all-to-all sends the rank's single block to itself;
// point-to-point calls only ever address rank 0 and carry nothing the
// headers read back on one rank, so they complete at once.
inline int MPI_Alltoall(const void* s, int sc, MPI_Datatype st, void* r, int,
                        MPI_Datatype, MPI_Comm) {
  if (r != s) std::memcpy(r, s, (size_t)sc * oracle_mpi_size(st));
  return 0;
}
inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm,
                     MPI_Request* q) { *q = 0; return 0; }
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm,
                     MPI_Request* q) { *q = 0; return 0; }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
#endif
