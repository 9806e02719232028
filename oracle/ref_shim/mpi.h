// Stand-in for the MPI declarations the reference's hot-path sources name, for
// compiling them on one process without MPI (test infrastructure of the
// oracle only). Collectives act on this process's buffers alone.
#pragma once
#include <cstring>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_DOUBLE 8
#define MPI_FLOAT 4
#define MPI_INT 104
#define MPI_LONG 108
#define MPI_UNSIGNED_LONG 208
#define MPI_LONG_LONG 308
#define MPI_CHAR 1
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5
#define MPI_IN_PLACE ((void*)1)
inline int mpi_type_size(MPI_Datatype t) { return t % 100; }
inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (in != MPI_IN_PLACE) std::memcpy(out, in, (size_t)n * mpi_type_size(t));
  return 0;
}
inline int MPI_Reduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (in != MPI_IN_PLACE) std::memcpy(out, in, (size_t)n * mpi_type_size(t));
  return 0;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Abort(MPI_Comm, int) { return 0; }
