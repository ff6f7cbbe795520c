/* Single-rank stand-in for the MPI interface that the reference's
 * codes/parallel/src/BasicParallel.cpp binds.  Test infrastructure only:
 * it lets the reference CPU solver build as an oracle with HX_PARALLEL
 * defined (without it the reference's residual norms are NaN, see
 * codes/parallel/src/BasicParallel.cpp:177-193).  Rank 0 of 1; reductions
 * copy; point-to-point calls are no-ops. */
#pragma once
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_INTEGER 4
#define MPI_DOUBLE 8
#define MPI_LONG_LONG_INT 9
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_MIN 2
#define MPI_REQUEST_NULL 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_BOTTOM ((void *)0)

static inline int ofg_mpi_type_size(MPI_Datatype t) { return t == MPI_LONG_LONG_INT ? 8 : t; }
static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
static inline int MPI_Get_processor_name(char *n, int *len) { strcpy(n, "oracle"); *len = 6; return 0; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline int MPI_Wait(MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void *s, void *t, int n, MPI_Datatype dt, MPI_Op, MPI_Comm)
{
    if (s != t) memmove(t, s, (size_t)n * ofg_mpi_type_size(dt));
    return 0;
}
