/* mpi.h — single-rank stand-in so the reference's serial sources compile
 * without an MPI installation.  TEST INFRASTRUCTURE ONLY (reference harness).
 * Only the calls the serial path's translation units reference are provided;
 * each behaves as a one-rank communicator. */
#ifndef HGPM_REF_HARNESS_MPI_H
#define HGPM_REF_HARNESS_MPI_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_LOR 2
#define MPI_SUCCESS 0
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* in, void* out, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c;
    if (in != out && t == MPI_INT) for (int i = 0; i < n; ++i) ((int*)out)[i] = ((const int*)in)[i];
    return MPI_SUCCESS;
}
#endif
