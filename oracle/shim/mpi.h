/*
 * Minimal MPI stand-in used ONLY to compile the reference's C sources into the
 * test oracle (oracle/_ref).  It is test infrastructure, never product code.
 *
 * The reference needs <mpi.h> unconditionally (algebra/include/mapmat/mapmat.h:24,
 * mappraiser/src/pcg_true.c:14, mappraiser/src/precond.c:13).  No MPI exists in
 * this image, so this header declares the ~20 MPI entry points the hot-path
 * files call (MPI_Allreduce, MPI_Isend/Irecv, MPI_Wtime, ...).
 *
 * Two implementations exist behind this one header:
 *   shim_mpi.c  - "world" of one or more processes created with fork(); the
 *                 collectives run through a POSIX shared-memory arena.  With one
 *                 process every collective is a copy, which is the exact
 *                 single-rank semantics of a real MPI.
 * The handle types follow the MPICH ABI (int handles).
 */
#ifndef ORACLE_SHIM_MPI_H
#define ORACLE_SHIM_MPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPI_VERSION    3
#define MPI_SUBVERSION 1

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;

typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count_bytes;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL  ((MPI_Comm) 0x04000000)
#define MPI_COMM_WORLD ((MPI_Comm) 0x44000000)
#define MPI_COMM_SELF  ((MPI_Comm) 0x44000001)

/* datatype handles carry their byte size in the low byte */
#define MPI_CHAR     ((MPI_Datatype) 0x4c000101)
#define MPI_BYTE     ((MPI_Datatype) 0x4c00010d)
#define MPI_INT      ((MPI_Datatype) 0x4c000405)
#define MPI_FLOAT    ((MPI_Datatype) 0x4c00040a)
#define MPI_LONG     ((MPI_Datatype) 0x4c000807)
#define MPI_INT64_T  ((MPI_Datatype) 0x4c000837)
#define MPI_DOUBLE   ((MPI_Datatype) 0x4c00080b)

#define MPI_SUM  ((MPI_Op) 0x58000003)
#define MPI_MAX  ((MPI_Op) 0x58000001)
#define MPI_MIN  ((MPI_Op) 0x58000002)

#define MPI_PROC_NULL (-1)
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_IN_PLACE ((void *) -1)
#define MPI_STATUS_IGNORE ((MPI_Status *) 1)
#define MPI_STATUSES_IGNORE ((MPI_Status *) 1)
#define MPI_REQUEST_NULL ((MPI_Request) 0x2c000000)

int    MPI_Init(int *argc, char ***argv);
int    MPI_Initialized(int *flag);
int    MPI_Finalize(void);
int    MPI_Abort(MPI_Comm comm, int code);
double MPI_Wtime(void);
int    MPI_Comm_rank(MPI_Comm comm, int *rank);
int    MPI_Comm_size(MPI_Comm comm, int *size);
int    MPI_Barrier(MPI_Comm comm);
int    MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op,
                     MPI_Comm comm);
int    MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, int root,
                  MPI_Comm comm);
int    MPI_Gather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                  int recvcount, MPI_Datatype recvtype, int root, MPI_Comm comm);
int    MPI_Alltoallv(const void *sendbuf, const int *sendcounts, const int *sdispls,
                     MPI_Datatype sendtype, void *recvbuf, const int *recvcounts, const int *rdispls,
                     MPI_Datatype recvtype, MPI_Comm comm);
int    MPI_Send(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm);
int    MPI_Recv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm,
                MPI_Status *status);
int    MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm comm,
                 MPI_Request *req);
int    MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm comm,
                 MPI_Request *req);
int    MPI_Wait(MPI_Request *req, MPI_Status *status);
int    MPI_Waitall(int count, MPI_Request reqs[], MPI_Status statuses[]);
int    MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                    void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                    MPI_Comm comm, MPI_Status *status);
int    MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype dt, int dest, int sendtag, int source,
                            int recvtag, MPI_Comm comm, MPI_Status *status);

/* shim control (not MPI): run `fn(rank, arg)` on `nranks` forked processes sharing one world. */
int shim_mpi_run(int nranks, void (*fn)(int rank, void *arg), void *arg);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_SHIM_MPI_H */
