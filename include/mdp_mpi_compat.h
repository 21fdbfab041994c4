/*
 * MPI handle type for the drop-in headers.  The reference's Mat and Tpltz
 * structs embed an MPI_Comm (algebra/include/mapmat/mapmat.h:62,
 * algebra/include/toeplitz/toeplitz.h:202).  When the caller has included a
 * real <mpi.h> first, its MPI_Comm is used; otherwise the MPICH ABI handle
 * (int) is declared here.  This single-GPU build is compiled with the int
 * handle: a caller whose MPI uses pointer handles (Open MPI) must rebuild the
 * library against its own mpi.h (define MDP_WITH_MPI_H).
 */
#ifndef MDP_MPI_COMPAT_H
#define MDP_MPI_COMPAT_H
#if defined(MDP_WITH_MPI_H)
#include <mpi.h>
#elif !defined(MPI_VERSION) && !defined(MPI_COMM_WORLD)
typedef int MPI_Comm;
#define MPI_COMM_WORLD ((MPI_Comm) 0x44000000)
#endif
#endif
