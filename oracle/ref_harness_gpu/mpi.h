/* Stand-in for <mpi.h> in the oracle's build of the reference GPU solvers.
 * Test infrastructure only.  The GPU solvers name MPI types in sim_env.h and
 * call MPI_Reduce in total_energy (never called by the driver); the
 * single-rank definitions live in ref_gpu_env.cu. */
#ifndef COFFEE_ORACLE_MPI_STUB_GPU_H
#define COFFEE_ORACLE_MPI_STUB_GPU_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int source, tag, error; } MPI_Status;
#define MPI_SUM 0
int MPI_Reduce(const void* sendbuf, void* recvbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm);
#endif
