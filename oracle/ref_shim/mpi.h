/* Project-written single-rank stand-in for the MPI subset the reference
 * channel-dns sources call (test infrastructure: lets the reference's own
 * sources build here as a checker and CPU baseline).  Communicator size is
 * always 1: collectives copy the local contribution, barriers and
 * broadcasts return at once, MPI_Abort exits the process. */
#ifndef CDNS_MPI_SHIM_H
#define CDNS_MPI_SHIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Errhandler;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_ERRORS_RETURN ((MPI_Errhandler)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_MAX_ERROR_STRING 256
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_UNSIGNED ((MPI_Datatype)104)
#define MPI_INT64_T ((MPI_Datatype)1008)
#define MPI_UINT64_T ((MPI_Datatype)1108)

#define MPI_SUM ((MPI_Op)1)
#define MPI_MIN ((MPI_Op)2)
#define MPI_MAX ((MPI_Op)3)

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_set_errhandler(MPI_Comm comm, MPI_Errhandler handler);
int MPI_Error_string(int code, char *text, int *length);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Alltoallv(const void *sendbuf, const int *sendcounts, const int *sdispls,
                  MPI_Datatype sendtype, void *recvbuf, const int *recvcounts, const int *rdispls,
                  MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buffer, int count, MPI_Datatype type, int root, MPI_Comm comm);
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm);

#ifdef __cplusplus
}
#endif
#endif
