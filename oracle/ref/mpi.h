/*
 * mpi.h -- single-rank stand-in for the MPI interface, written for this
 * project so that the reference solver (rismical-dev/3D-RISM-CUDA-MPI,
 * src-cuda-mpi/) can be compiled and run at one rank without an MPI
 * installation.  TEST INFRASTRUCTURE: it only serves oracle/ref/build_ref.sh,
 * whose output (oracle/_ref/) is used to pin the CPU oracle.
 *
 * At one rank every collective degenerates to a local copy: Bcast is a no-op,
 * Allreduce/Reduce copy the send buffer, Alltoall copies `count` elements
 * (device pointers allowed: cudaMemcpyDefault), and MPI-IO maps onto stdio.
 */
#ifndef R3D_SINGLE_RANK_MPI_H
#define R3D_SINGLE_RANK_MPI_H
#include <stdio.h>
#include <string.h>
#include <time.h>
#include <cuda_runtime.h>

typedef int MPI_Comm;
typedef int MPI_Datatype; /* value = element size in bytes */
typedef int MPI_Op;
typedef int MPI_Info;
typedef FILE *MPI_File;
typedef struct { int unused; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_INTEGER ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_DOUBLE_PRECISION ((MPI_Datatype)sizeof(double))
#define MPI_DOUBLE_COMPLEX ((MPI_Datatype)(2 * sizeof(double)))
#define MPI_SUM 0
#define MPI_INFO_NULL 0
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_SEEK_SET SEEK_SET
#define MPI_THREAD_FUNNELED 1

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Init_thread(int *, char ***, int, int *p) { if (p) *p = 1; return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_split(MPI_Comm, int, int, MPI_Comm *c) { *c = 0; return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t,
                                MPI_Op, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * t);
  return 0;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t,
                             MPI_Op, int, MPI_Comm) {
  if (s != r) memmove(r, s, (size_t)n * t);
  return 0;
}
static inline int MPI_Alltoall(const void *s, int n, MPI_Datatype t, void *r,
                               int, MPI_Datatype, MPI_Comm) {
  cudaMemcpy(r, s, (size_t)n * t, cudaMemcpyDefault);
  return 0;
}
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static inline int MPI_File_open(MPI_Comm, const char *path, int, MPI_Info,
                                MPI_File *f) {
  *f = fopen(path, "wb");
  return *f ? 0 : 1;
}
static inline int MPI_File_write(MPI_File f, const void *b, int n,
                                 MPI_Datatype t, MPI_Status *) {
  fwrite(b, (size_t)t, (size_t)n, f);
  return 0;
}
static inline int MPI_File_write_all(MPI_File f, const void *b, int n,
                                     MPI_Datatype t, MPI_Status *) {
  fwrite(b, (size_t)t, (size_t)n, f);
  return 0;
}
static inline int MPI_File_seek(MPI_File f, long off, int whence) {
  return fseek(f, off, whence);
}
static inline int MPI_File_close(MPI_File *f) {
  fclose(*f);
  return 0;
}
#endif
