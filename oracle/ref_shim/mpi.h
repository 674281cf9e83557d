/*
 * Single-rank MPI stand-in used ONLY to compile the reference solver's own
 * headers into the CPU oracle library (oracle/_ref).  It is test
 * infrastructure, never linked into the product.
 *
 * With Comm_size == 1 the reference never posts a send/recv or an allreduce
 * (every call site is guarded by `mpi->size > 1` or `rank > 0`,
 * src/cfd.h:256-274, src/mv.h:26, src/alm.h:373), so every function here is
 * a no-op that returns success.
 */
#pragma once

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int dummy; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_LONG 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_UNSIGNED_CHAR 5
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) { return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Allreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
static inline int MPI_Iallreduce(const void *, void *, int, MPI_Datatype, MPI_Op, MPI_Comm, MPI_Request *) { return 0; }
