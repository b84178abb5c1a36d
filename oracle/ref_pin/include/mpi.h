/* Single-rank stand-in for the MPI calls the reference's PM / COLA / 2LPT
 * sources make (py/comm.cpp, py/comm.h, py/particle.cpp, py/pm.cpp).
 * TEST INFRASTRUCTURE: used only to compile the reference's own loops into
 * oracle/_ref for pinning the oracle; never part of the product.
 * One rank: rank 0 of 1, collectives copy the send buffer. */
#ifndef FS2REF_MPI_H
#define FS2REF_MPI_H 1

#include <stddef.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Win;
typedef int MPI_Info;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_INFO_NULL 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1

#define MPI_INT 1
#define MPI_LONG 2
#define MPI_LONG_LONG 3
#define MPI_FLOAT 4
#define MPI_DOUBLE 5
#define MPI_UNSIGNED_LONG 6
#define MPI_BYTE 7

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t fs2ref_mpi_size(MPI_Datatype t) {
  switch(t) {
  case MPI_INT: return sizeof(int);
  case MPI_LONG: return sizeof(long);
  case MPI_LONG_LONG: return sizeof(long long);
  case MPI_FLOAT: return sizeof(float);
  case MPI_DOUBLE: return sizeof(double);
  case MPI_UNSIGNED_LONG: return sizeof(unsigned long);
  default: return 1;
  }
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Init_thread(int*, char***, int required, int* provided) {
  *provided = required; return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int) { abort(); return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) {
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t,
                                MPI_Op, MPI_Comm) {
  memmove(r, s, (size_t) n*fs2ref_mpi_size(t)); return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t,
                             MPI_Op, int, MPI_Comm) {
  memmove(r, s, (size_t) n*fs2ref_mpi_size(t)); return MPI_SUCCESS;
}
static inline int MPI_Scan(const void* s, void* r, int n, MPI_Datatype t,
                           MPI_Op, MPI_Comm) {
  memmove(r, s, (size_t) n*fs2ref_mpi_size(t)); return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r,
                                int, MPI_Datatype, MPI_Comm) {
  memmove(r, s, (size_t) n*fs2ref_mpi_size(t)); return MPI_SUCCESS;
}

#endif
