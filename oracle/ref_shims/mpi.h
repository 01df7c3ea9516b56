/* Single-rank stand-in for the MPI calls that the reference's BSP build path
 * makes (include/bsp/broadcast_bsp_framework.cpp:36-210, src/bsp_index.hpp:
 * 442-445, 554; src/diskann.cpp:101-122).  World size is 1 and every
 * collective is a copy from the send buffer to the receive buffer, which is
 * exactly what `mpirun -np 1` does.  Used only to compile the reference's own
 * sources as a test oracle; never linked into the product library. */
#pragma once
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_UINT64_T 8
#define MPI_LONG_LONG 8
#define MPI_DOUBLE 8
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_SUCCESS 0

/* element size of each datatype, encoded as the datatype value itself */
static inline size_t dd_shim_type_size(MPI_Datatype t) { return (size_t)t; }

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
static inline double MPI_Wtime() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch()).count();
}
static inline int MPI_Alltoall(const void* s, int sc, MPI_Datatype st, void* r,
                               int, MPI_Datatype, MPI_Comm) {
  std::memmove(r, s, (size_t)sc * dd_shim_type_size(st));
  return MPI_SUCCESS;
}
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd,
                                MPI_Datatype st, void* r, const int*,
                                const int* rd, MPI_Datatype, MPI_Comm) {
  size_t es = dd_shim_type_size(st);
  std::memmove((char*)r + (size_t)rd[0] * es, (const char*)s + (size_t)sd[0] * es,
               (size_t)sc[0] * es);
  return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* s, void* r, int c, MPI_Datatype t,
                                MPI_Op, MPI_Comm) {
  std::memmove(r, s, (size_t)c * dd_shim_type_size(t));
  return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int c, MPI_Datatype t,
                             MPI_Op, int, MPI_Comm) {
  std::memmove(r, s, (size_t)c * dd_shim_type_size(t));
  return MPI_SUCCESS;
}
static inline int MPI_Gather(const void* s, int sc, MPI_Datatype st, void* r,
                             int, MPI_Datatype, int, MPI_Comm) {
  std::memmove(r, s, (size_t)sc * dd_shim_type_size(st));
  return MPI_SUCCESS;
}
