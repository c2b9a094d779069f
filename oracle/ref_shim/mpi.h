/*
 * mpi.h — single-rank stand-in for MPI, used only to compile the reference
 * program (anpicon/EDUS main_MPI.cpp) as a CPU checker under oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY. With one rank every collective the reference
 * issues is local: MPI_Reduce copies the send buffer into the receive buffer
 * (a sum / max / min over one rank is the value itself), MPI_Bcast from rank 0
 * to rank 0 leaves the buffer as it is, and MPI_Barrier returns at once. The
 * reference only sends or receives when num_procs > 1 (for example
 * headers/MPIcommunication.h:4, headers/Observables_MPI.h:80-104), so the
 * point-to-point calls are unreachable; they abort if ever reached.
 */
#ifndef EDUS_REF_SHIM_MPI_H
#define EDUS_REF_SHIM_MPI_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <complex>
#include <omp.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_SUCCESS 0

/* Datatype handles carry the element size in bytes. */
#define MPI_INT ((MPI_Datatype)sizeof(int))
#define MPI_DOUBLE ((MPI_Datatype)sizeof(double))
#define MPI_C_DOUBLE_COMPLEX ((MPI_Datatype)(2 * sizeof(double)))

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

#define MPI_STATUS_IGNORE ((MPI_Status*)0)

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Init_thread(int*, char***, int required, int* provided) {
    *provided = required;
    return MPI_SUCCESS;
}
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) {
    *r = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm, int* n) {
    *n = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }

static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
    if (send != recv && count > 0) std::memmove(recv, send, (size_t)count * (size_t)type);
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm c) {
    return MPI_Reduce(send, recv, count, type, op, 0, c);
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }

static inline int mpi_shim_unreachable(const char* what) {
    std::fprintf(stderr, "mpi shim: %s called with one rank\n", what);
    std::abort();
    return 1;
}
static inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return mpi_shim_unreachable("MPI_Send"); }
static inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) {
    return mpi_shim_unreachable("MPI_Recv");
}

#endif
