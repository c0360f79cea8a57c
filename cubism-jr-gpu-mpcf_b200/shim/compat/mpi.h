/* mpi.h -- single-rank stand-in for builds without an MPI library.
 * Covers what the hot path's callers use on one rank: the Cartesian
 * communicator set-up of GridMPI (source/GridMPI.h:57-106) and the dt
 * MIN all-reduce of LSRK3_IntegratorMPI (LSRK3_IntegratorMPI.cpp:40).  With
 * one rank every reduction is the identity and every neighbour is self.
 * Only on the include path when no real mpi.h is available. */
#pragma once
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_IN_PLACE ((void*)1)
#define MPI_DOUBLE 8
#define MPI_FLOAT 4
#define MPI_INT 4
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_ANY_TAG (-1)

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize() { return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* n) { *n = 1; return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Cart_create(MPI_Comm, int, const int*, const int*, int, MPI_Comm* c) { *c = 0; return 0; }
static inline int MPI_Cart_coords(MPI_Comm, int, int n, int* coords) { for (int i = 0; i < n; ++i) coords[i] = 0; return 0; }
static inline int MPI_Cart_rank(MPI_Comm, const int*, int* r) { *r = 0; return 0; }
static inline int MPI_Allreduce(const void* s, void* r, int count, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    if (s != MPI_IN_PLACE) memcpy(r, s, (size_t)count * (size_t)t);
    return 0;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }

#ifdef __cplusplus
/* the datatype names of the MPI-2 C++ bindings, which the reference's case
 * set-up passes to MPI_Bcast (Sim_SICCloudMPI.cpp:162-169) */
namespace MPI
{
static const MPI_Datatype CHAR = 1, INT = 4, FLOAT = 4, DOUBLE = 8;
}
#endif
