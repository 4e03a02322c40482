/*
 * Single-process MPI interface for the GPU drop-in build.  The drop-in runs
 * one domain per GPU in one process, so the reference's Communicator calls
 * (src/communicator.cc) reduce to copies within this process: collectives
 * copy the send buffer to the receive buffer, Sendrecv to self copies bytes,
 * Wtime is a monotonic clock.
 */
#ifndef MDACP_B200_DROPIN_MPI_H
#define MDACP_B200_DROPIN_MPI_H
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;  /* the value is the element size in bytes */
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)sizeof(unsigned long))
#define MPI_SUM ((MPI_Op)0)
#define MPI_MAX ((MPI_Op)1)
#define MPI_LOR ((MPI_Op)2)

static inline void mdg_mpi_copy(const void *src, void *dst, long bytes) {
  if (bytes > 0 && src && dst && src != dst) memmove(dst, src, (size_t)bytes);
}
static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Sendrecv(const void *sb, int sc, MPI_Datatype st, int, int, void *rb, int,
                               MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  mdg_mpi_copy(sb, rb, (long)sc * st);
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *sb, void *rb, int c, MPI_Datatype t, MPI_Op, MPI_Comm) {
  mdg_mpi_copy(sb, rb, (long)c * t);
  return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void *sb, int sc, MPI_Datatype st, void *rb, int, MPI_Datatype,
                                MPI_Comm) {
  mdg_mpi_copy(sb, rb, (long)sc * st);
  return MPI_SUCCESS;
}
static inline int MPI_Gather(const void *sb, int sc, MPI_Datatype st, void *rb, int, MPI_Datatype, int,
                             MPI_Comm) {
  mdg_mpi_copy(sb, rb, (long)sc * st);
  return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
#endif
