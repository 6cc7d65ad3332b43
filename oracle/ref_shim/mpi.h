/* Test-infrastructure stub of <mpi.h> for compiling the reference's CPU
 * interpolation sources in place (oracle/_ref).  The reference includes
 * <mpi.h> from include/process.h:4 and its Data.cpp files, but the loader and
 * kernels built here never call MPI: only the type MPI_Comm and the constant
 * MPI_SUCCESS are needed. */
#ifndef ORACLE_REF_MPI_STUB_H
#define ORACLE_REF_MPI_STUB_H
typedef int MPI_Comm;
#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#endif
