/*
 * One-rank stand-in for <mpi.h>, used only to compile the reference's own
 * header-only iSVD stages into the CPU checker (oracle/_ref).  It is test
 * infrastructure, never part of the product.
 *
 * With a single rank every collective degenerates into a copy (or nothing):
 * an all-reduce of one contribution is that contribution, a broadcast from
 * rank 0 to rank 0 moves nothing, a gather of one block is that block.
 * Datatype handles encode their element size in bytes so the copies know
 * how much to move.
 */
#ifndef MCNLA_ORACLE_MPI_STUB_H_
#define MCNLA_ORACLE_MPI_STUB_H_

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_SUCCESS 0
#define MPI_SUM ((MPI_Op)1)
#define MPI_MAX ((MPI_Op)2)
#define MPI_MIN ((MPI_Op)3)
#define MPI_IN_PLACE ((void*)1)

/* datatype handle == element size in bytes */
#define MPI_BYTE       ((MPI_Datatype)1)
#define MPI_CHAR       ((MPI_Datatype)1)
#define MPI_CHARACTER  ((MPI_Datatype)1)
#define MPI_INTEGER1   ((MPI_Datatype)1)
#define MPI_INTEGER2   ((MPI_Datatype)2)
#define MPI_INTEGER4   ((MPI_Datatype)4)
#define MPI_INTEGER8   ((MPI_Datatype)8)
#define MPI_INTEGER    ((MPI_Datatype)4)
#define MPI_INT        ((MPI_Datatype)4)
#define MPI_REAL4      ((MPI_Datatype)4)
#define MPI_REAL8      ((MPI_Datatype)8)
#define MPI_REAL       ((MPI_Datatype)4)
#define MPI_DOUBLE     ((MPI_Datatype)8)
#define MPI_COMPLEX8   ((MPI_Datatype)8)
#define MPI_COMPLEX16  ((MPI_Datatype)16)
#define MPI_COMPLEX    ((MPI_Datatype)8)

static inline void mpi_stub_copy_(const void* s, void* r, int n, MPI_Datatype t) {
  if (s != MPI_IN_PLACE && s != r && n > 0) memmove(r, s, (size_t)n * (size_t)t);
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  mpi_stub_copy_(s, r, n, t); return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  mpi_stub_copy_(s, r, n, t); return MPI_SUCCESS;
}
static inline int MPI_Reduce_scatter_block(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  mpi_stub_copy_(s, r, n, t); return MPI_SUCCESS;
}
static inline int MPI_Scatter(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
  mpi_stub_copy_(s, r, n, t); return MPI_SUCCESS;
}
static inline int MPI_Scatterv(const void* s, const int* cnt, const int* disp, MPI_Datatype t, void* r, int,
                               MPI_Datatype, int, MPI_Comm) {
  mpi_stub_copy_((const char*)s + (size_t)disp[0] * (size_t)t, r, cnt[0], t); return MPI_SUCCESS;
}
static inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
  mpi_stub_copy_(s, r, n, t); return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* disp,
                              MPI_Datatype, int, MPI_Comm) {
  mpi_stub_copy_(s, (char*)r + (size_t)disp[0] * (size_t)t, n, t); return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
  mpi_stub_copy_(s, r, n, t); return MPI_SUCCESS;
}
static inline int MPI_Alltoall(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
  mpi_stub_copy_(s, r, n, t); return MPI_SUCCESS;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return MPI_SUCCESS; }

#endif  /* MCNLA_ORACLE_MPI_STUB_H_ */
