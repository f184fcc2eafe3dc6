/*
 * Single-process stand-in for the handful of MPI calls the lpmCxx sources make
 * (test infrastructure for the oracle build only; never linked into the product).
 *
 * The reference splits targets with MPIReplicatedData(n, rank, size)
 * (src/LpmMPIReplicatedData.cpp:12-23) and then replicates slices with MPI_Bcast
 * (src/LpmDirectSum.cpp:256-291).  Here every "rank" is an independent process:
 * MPI_Comm_rank / MPI_Comm_size report LPM_STUB_RANK / LPM_STUB_SIZE from the
 * environment (default 0 / 1), MPI_Bcast is a no-op and MPI_Reduce copies.
 * That lets the CPU baseline run the reference's own target split on P host
 * cores as P processes.
 */
#ifndef LPM_ORACLE_MPI_STUB_H
#define LPM_ORACLE_MPI_STUB_H

#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_LONG 3
#define MPI_SUM 0
#define MPI_MAX 1
#define MPI_SUCCESS 0

static inline int lpm_stub_env_int(const char* name, int dflt) {
    const char* s = getenv(name);
    return s ? atoi(s) : dflt;
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Finalize() { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* size) {
    *size = lpm_stub_env_int("LPM_STUB_SIZE", 1);
    return MPI_SUCCESS;
}
static inline int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = lpm_stub_env_int("LPM_STUB_RANK", 0);
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int lpm_stub_type_size(MPI_Datatype t) {
    return t == MPI_DOUBLE ? 8 : (t == MPI_LONG ? 8 : 4);
}
static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    memcpy(recv, send, (size_t)count * lpm_stub_type_size(t));
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    memcpy(recv, send, (size_t)count * lpm_stub_type_size(t));
    return MPI_SUCCESS;
}
static inline double MPI_Wtime() {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#endif
