/* Minimal stand-in for <mpi.h> so that the reference's single-particle
 * physics files (src_mpi/Particle/*.cpp, src_mpi/TimeStepRoutines.cpp)
 * compile without an MPI installation.  Those files only name the MPI
 * handle types through src_mpi/global.h; none of them calls MPI.
 * Test infrastructure only: used to build oracle/_ref, the checker. */
#ifndef ABYSS_ORACLE_STUB_MPI_H
#define ABYSS_ORACLE_STUB_MPI_H
typedef int MPI_Win;
typedef int MPI_Comm;
typedef int MPI_Request;
typedef int MPI_Status;
typedef int MPI_Datatype;
#endif
