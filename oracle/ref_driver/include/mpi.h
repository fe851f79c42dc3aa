/* mpi.h — single-rank stand-in so the reference's own serial() driver
 * (src/driver_pm.cpp) compiles against the C++ drop-in without an MPI
 * installation.  TEST INFRASTRUCTURE ONLY.  Every call behaves as a one-rank
 * communicator, so main() takes its serial() branch. */
#ifndef HGPM_REF_DRIVER_MPI_H
#define HGPM_REF_DRIVER_MPI_H
#include <string.h>
typedef int MPI_Comm;
#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
static inline int MPI_Init(int* argc, char*** argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
#endif
