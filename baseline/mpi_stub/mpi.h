/* mpi.h -- single-process stand-in for the few MPI calls the reference's sweep
 * driver makes (src/app/sweep.cu: MPI_Comm_rank/size, MPI_Gather, MPI_Gatherv,
 * MPI_Reduce).  With one rank every collective is a copy from the send buffer to
 * the receive buffer, so runSweep runs its own code path unchanged on one GPU.
 * Used only to build the reference's GPU code for comparison (baseline/Makefile). */
#ifndef SBR_BASELINE_MPI_STUB_H
#define SBR_BASELINE_MPI_STUB_H

#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_SUM 1
#define MPI_MAX 2

static inline size_t sbr_mpi_stub_size(MPI_Datatype t) {
    return t == MPI_DOUBLE ? sizeof(double) : t == MPI_FLOAT ? sizeof(float) : sizeof(int);
}

static inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }

static inline int MPI_Gather(const void* send, int count, MPI_Datatype type, void* recv, int, MPI_Datatype,
                             int, MPI_Comm) {
    if (count > 0 && recv != send) memcpy(recv, send, (size_t)count * sbr_mpi_stub_size(type));
    return MPI_SUCCESS;
}

static inline int MPI_Gatherv(const void* send, int count, MPI_Datatype type, void* recv, const int*,
                              const int* displs, MPI_Datatype, int, MPI_Comm) {
    if (count > 0) {
        char* dst = (char*)recv + (size_t)displs[0] * sbr_mpi_stub_size(type);
        if (dst != send) memcpy(dst, send, (size_t)count * sbr_mpi_stub_size(type));
    }
    return MPI_SUCCESS;
}

static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
    if (count > 0 && recv != send) memcpy(recv, send, (size_t)count * sbr_mpi_stub_size(type));
    return MPI_SUCCESS;
}

#endif
