/* Single-rank stand-in for the MPI subset the reference uses, so the
 * reference's own ParisPencil.cpp / main.cpp / FishFry.hpp build and run on one
 * GPU without an MPI library.  Test infrastructure only (oracle/_ref).
 *   - one rank: rank 0 of size 1 on every communicator;
 *   - MPI_Alltoall / MPI_Reduce with one rank are copies; the reference passes
 *     device pointers (CUDA-aware MPI), so the copies use cudaMemcpyDefault;
 *   - MPI_Wtime is a monotonic clock in seconds. */
#ifndef FISHFRY_ORACLE_MPI_STUB_H
#define FISHFRY_ORACLE_MPI_STUB_H

#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;

#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-1)
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL 0
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int mpistub_size(MPI_Datatype t) { return t == MPI_INT ? (int)sizeof(int) : (int)sizeof(double); }

static inline int mpistub_copy(void *dst, const void *src, size_t bytes) {
  if (dst == src || bytes == 0) return 0;
  cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyDefault);
  if (e != cudaSuccess) {
    fprintf(stderr, "mpi stub copy failed: %s\n", cudaGetErrorString(e));
    exit(1);
  }
  return 0;
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *c) { *c = 0; return 0; }
static inline int MPI_Comm_split_type(MPI_Comm, int, int, MPI_Info, MPI_Comm *c) { *c = 0; return 0; }
static inline int MPI_Comm_free(MPI_Comm *) { return 0; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Alltoall(const void *s, int sc, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  return mpistub_copy(r, s, (size_t)sc * mpistub_size(st));
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  return mpistub_copy(r, s, (size_t)n * mpistub_size(t));
}

#endif
