/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference
 * solver as the CPU oracle (test infrastructure, never shipped).
 *
 * With one rank the reference's 3D Cartesian communicator has dims 1x1x1,
 * so every MPI_Cart_shift neighbour is MPI_PROC_NULL and every
 * MPI_Sendrecv is a no-op; Allreduce/Reduce are identities
 * (reference call sites: calculation_2D.cpp:401,449-456,615-775,1106;
 * air.cpp:2536-2699; airpore.cpp:919-932).
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SUM 1
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0

static inline int oracle_mpi_type_size(MPI_Datatype t) { return t == MPI_DOUBLE ? 8 : 4; }

inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

inline int MPI_Cart_create(MPI_Comm, int, int *, int *, int, MPI_Comm *cart)
{
    *cart = 1;
    return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm, int, int, int *src, int *dst)
{
    *src = MPI_PROC_NULL;
    *dst = MPI_PROC_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int *coords)
{
    for (int d = 0; d < maxdims; ++d) coords[d] = 0;
    return MPI_SUCCESS;
}

/* Both partners are MPI_PROC_NULL on one rank: nothing is sent or received. */
inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int,
                        void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *)
{
    return MPI_SUCCESS;
}

inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    std::memmove(out, in, (size_t)n * oracle_mpi_type_size(t));
    return MPI_SUCCESS;
}

inline int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    std::memmove(out, in, (size_t)n * oracle_mpi_type_size(t));
    return MPI_SUCCESS;
}

#endif
