/* Oracle-only single-rank stand-in for <mpi.h> (test infrastructure): the
 * calls the reference's grid, boundary and reduction code makes, with the
 * semantics they have on one rank -- a 1x1x1 Cartesian communicator whose
 * neighbour in a periodic dimension is the rank itself (MPI_PROC_NULL across a
 * non-periodic border), a send-receive with oneself that leaves the buffer as
 * it is, and in-place all-reductions that change nothing. */
#pragma once

#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_PROC_NULL (-2)
#define MPI_SUCCESS 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_CXX_BOOL 3
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)

namespace hcl_mpi_stub {
// periodicity of the one Cartesian communicator (set by MPI_Cart_create)
inline int& periods(int d)
{
    static int p[3] = {0, 0, 0};
    return p[d];
}
} // namespace hcl_mpi_stub

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size)
{
    *size = 1;
    return MPI_SUCCESS;
}
inline int MPI_Comm_rank(MPI_Comm, int* rank)
{
    *rank = 0;
    return MPI_SUCCESS;
}
inline int MPI_Comm_free(MPI_Comm* c)
{
    *c = MPI_COMM_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Dims_create(int, int ndims, int* dims)
{
    for (int d = 0; d < ndims; ++d) {
        if (dims[d] == 0) {
            dims[d] = 1;
        }
    }
    return MPI_SUCCESS;
}
inline int MPI_Cart_create(MPI_Comm, int ndims, const int*, const int* periodic, int, MPI_Comm* out)
{
    for (int d = 0; d < ndims && d < 3; ++d) {
        hcl_mpi_stub::periods(d) = periodic[d];
    }
    *out = 2;
    return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int* coords)
{
    for (int d = 0; d < maxdims; ++d) {
        coords[d] = 0;
    }
    return MPI_SUCCESS;
}
inline int MPI_Cart_sub(MPI_Comm, const int*, MPI_Comm* out)
{
    *out = 3;
    return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm, int dir, int, int* src, int* dst)
{
    const int nb = hcl_mpi_stub::periods(dir) ? 0 : MPI_PROC_NULL;
    *src = nb;
    *dst = nb;
    return MPI_SUCCESS;
}
inline int MPI_Sendrecv_replace(void*, int, MPI_Datatype, int, int, int, int, MPI_Comm, MPI_Status*)
{
    return MPI_SUCCESS; // exchanging a buffer with oneself leaves it unchanged
}
inline int MPI_Allreduce(const void* in, void* out, int count, MPI_Datatype type, MPI_Op, MPI_Comm)
{
    if (in != MPI_IN_PLACE) {
        const int sz = type == MPI_DOUBLE ? 8 : (type == MPI_INT ? 4 : 1);
        std::memcpy(out, in, (size_t)count * sz);
    }
    return MPI_SUCCESS;
}
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
