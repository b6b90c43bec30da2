/* Single-rank stand-in for the MPI calls made by the reference's hot-path
 * sources (test infrastructure only).  Every collective is called with
 * MPI_IN_PLACE on one rank, so it is a no-op. */
#ifndef SBSLPM_ORACLE_SHIM_MPI_H
#define SBSLPM_ORACLE_SHIM_MPI_H

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Win;
#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_SUM 0
#define MPI_IN_PLACE ((void*)1)
#define MPI_SUCCESS 0

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* p) { *p = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Allreduce(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return 0; }
static inline int MPI_Win_fence(int, MPI_Win) { return 0; }
static inline int MPI_Accumulate(const void*, int, MPI_Datatype, int, long, int, MPI_Datatype, MPI_Op,
                                 MPI_Win) { return 0; }
static inline int MPI_Get(void*, int, MPI_Datatype, int, long, int, MPI_Datatype, MPI_Win) { return 0; }

#endif
