/* Single-rank MPI stand-in used only to compile the reference's headers into
 * the oracle library (oracle/_ref).  Rank 0 of a world of size 1: collectives
 * copy the send buffer to the receive buffer, point-to-point calls and
 * barriers do nothing, MPI_Wtime is a steady clock.  Test infrastructure only. */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H
#include <chrono>
#include <cstddef>
#include <cstdio>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Errhandler;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_ERROR_STRING 64
#define MPI_ERRORS_RETURN 1
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#define MPI_BYTE 1
#define MPI_CHAR 2
#define MPI_INT 3
#define MPI_LONG 4
#define MPI_FLOAT 5
#define MPI_DOUBLE 6

static inline size_t oracle_mpi_size(MPI_Datatype t) {
  switch (t) {
    case MPI_BYTE: case MPI_CHAR: return 1;
    case MPI_INT: case MPI_FLOAT: return 4;
    case MPI_LONG: case MPI_DOUBLE: return 8;
  }
  return 1;
}
static inline void oracle_mpi_copy(void* dst, const void* src, size_t bytes) {
  if (dst && src && dst != src && bytes) std::memmove(dst, src, bytes);
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int* flag) { *flag = 0; return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Finalized(int* flag) { *flag = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm*) { return MPI_SUCCESS; }
static inline int MPI_Comm_set_errhandler(MPI_Comm, int) { return MPI_SUCCESS; }
static inline int MPI_Error_string(int code, char* s, int* len) {
  *len = std::snprintf(s, MPI_MAX_ERROR_STRING, "mpi error %d", code);
  return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline double MPI_Wtime() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  oracle_mpi_copy(r, s, n * oracle_mpi_size(t));
  return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
  oracle_mpi_copy(r, s, sn * oracle_mpi_size(st));
  return MPI_SUCCESS;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Scatter(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) {
  oracle_mpi_copy(r, s, sn * oracle_mpi_size(st));
  return MPI_SUCCESS;
}
static inline int MPI_Scatterv(const void* s, const int* counts, const int* displs, MPI_Datatype st, void* r, int,
                               MPI_Datatype, int, MPI_Comm) {
  if (s) oracle_mpi_copy(r, (const char*)s + displs[0] * oracle_mpi_size(st), counts[0] * oracle_mpi_size(st));
  return MPI_SUCCESS;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return MPI_SUCCESS; }
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request* q) { *q = 0; return MPI_SUCCESS; }
static inline int MPI_Testall(int, MPI_Request*, int* flag, MPI_Status*) { *flag = 1; return MPI_SUCCESS; }
#endif
