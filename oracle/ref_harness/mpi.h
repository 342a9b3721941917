/* Type-only stand-in for <mpi.h>.
 *
 * The reference's sim_env.h (src/sim_env.h:9,43-53) names MPI_Comm,
 * MPI_Datatype and MPI_Status in member declarations.  The single-rank
 * test double in ref_env.cpp never calls MPI, so only the type names are
 * needed to compile the reference's CPU translation units against it.
 * This file is test infrastructure for the oracle only.
 */
#ifndef COFFEE_ORACLE_MPI_STUB_H
#define COFFEE_ORACLE_MPI_STUB_H
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct { int source, tag, error; } MPI_Status;
#endif
