// Communicator type used by the ddla handle API.
//
// The reference's handle header includes <mpi.h> (include/ddla/ddla_handle_t.h:8)
// because ddlaSet takes an MPI communicator.  This build serves the 1x1 process
// grid only, so when no MPI header has been included before this one (and
// DDLA_WITH_MPI is not defined) a single-rank stand-in supplies the handful of
// names the API mentions: a communicator is an int, MPI_COMM_WORLD has size 1.
#ifndef DDLA_MPI_H
#define DDLA_MPI_H

#if defined(DDLA_WITH_MPI) || defined(MPI_VERSION)
#include <mpi.h>
#else
typedef int MPI_Comm;
typedef int MPI_Fint;
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#endif
#ifndef MPI_COMM_NULL
#define MPI_COMM_NULL ((MPI_Comm)0x04000000)
#endif
#define DDLA_SINGLE_RANK_MPI 1
inline MPI_Comm MPI_Comm_f2c(MPI_Fint f) { return (MPI_Comm)f; }
inline MPI_Fint MPI_Comm_c2f(MPI_Comm c) { return (MPI_Fint)c; }
#endif

#endif
