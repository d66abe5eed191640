/*
 * Single-rank MPI stand-in used ONLY to compile the reference Tapas headers
 * into the test oracle (oracle/_ref).  It is test scaffolding, not product
 * code: nothing under tapas-reduce_b200/ includes it.
 *
 * Semantics: one process, rank 0 of size 1.  A datatype handle is its size in
 * bytes, so every collective is a plain copy from the send buffer to the
 * receive buffer (the only data movement a 1-rank collective performs).
 * Point-to-point calls never execute on one rank in the reference driver
 * (CheckResult skips them when src == dst) and are no-ops here.
 */
#ifndef ORACLE_MPI_SHIM_H_
#define ORACLE_MPI_SHIM_H_

#include <string.h>
#include <stdio.h>
#include <time.h>

typedef int MPI_Comm;
typedef long MPI_Datatype; /* byte size of one element */
typedef int MPI_Op;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_IN_PLACE ((void *)1)

#define MPI_BYTE ((MPI_Datatype)1)
#define MPI_CHAR ((MPI_Datatype)sizeof(char))
#define MPI_UNSIGNED_CHAR ((MPI_Datatype)sizeof(unsigned char))
#define MPI_WCHAR ((MPI_Datatype)sizeof(wchar_t))
#define MPI_SHORT ((MPI_Datatype)sizeof(short))
#define MPI_UNSIGNED_SHORT ((MPI_Datatype)sizeof(unsigned short))
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_UNSIGNED ((MPI_Datatype)sizeof(unsigned))
#define MPI_LONG ((MPI_Datatype)sizeof(long))
#define MPI_UNSIGNED_LONG ((MPI_Datatype)sizeof(unsigned long))
#define MPI_LONG_LONG ((MPI_Datatype)sizeof(long long))
#define MPI_UNSIGNED_LONG_LONG ((MPI_Datatype)sizeof(unsigned long long))
#define MPI_FLOAT ((MPI_Datatype)sizeof(float))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_LONG_DOUBLE ((MPI_Datatype)sizeof(long double))

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Get_processor_name(char *name, int *len) {
  snprintf(name, MPI_MAX_PROCESSOR_NAME, "localhost");
  *len = (int)strlen(name);
  return MPI_SUCCESS;
}
static inline int MPI_Error_string(int, char *s, int *len) {
  snprintf(s, 32, "mpi shim error");
  *len = (int)strlen(s);
  return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *t) {
  *t = (MPI_Datatype)count * old;
  return MPI_SUCCESS;
}
static inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
static inline int MPI_Type_extent(MPI_Datatype t, MPI_Aint *e) { *e = t; return MPI_SUCCESS; }

static inline void oracle_mpi_copy_(const void *s, void *r, long bytes) {
  if (s != MPI_IN_PLACE && s != r && bytes > 0) memmove(r, s, (size_t)bytes);
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  oracle_mpi_copy_(s, r, (long)n * t); return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  oracle_mpi_copy_(s, r, (long)n * t); return MPI_SUCCESS;
}
static inline int MPI_Scan(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  oracle_mpi_copy_(s, r, (long)n * t); return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, int, MPI_Comm) {
  oracle_mpi_copy_(s, r, (long)sn * st); return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  oracle_mpi_copy_(s, r, (long)sn * st); return MPI_SUCCESS;
}
static inline int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *, const int *rd,
                                 MPI_Datatype rt, MPI_Comm) {
  oracle_mpi_copy_(s, (char *)r + (long)rd[0] * rt, (long)sn * st); return MPI_SUCCESS;
}
static inline int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int, MPI_Datatype, MPI_Comm) {
  oracle_mpi_copy_(s, r, (long)sn * st); return MPI_SUCCESS;
}
static inline int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r,
                                const int *, const int *rd, MPI_Datatype rt, MPI_Comm) {
  oracle_mpi_copy_((const char *)s + (long)sd[0] * st, (char *)r + (long)rd[0] * rt, (long)sc[0] * st);
  return MPI_SUCCESS;
}
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return MPI_SUCCESS; }

#endif /* ORACLE_MPI_SHIM_H_ */
