// Single-rank implementation of the MPI subset declared in mpi.h.
#include "mpi.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace {
size_t type_size(MPI_Datatype t) {
    switch (t) {
    case MPI_DOUBLE: return sizeof(double);
    case MPI_INT: return sizeof(int);
    case MPI_UNSIGNED: return sizeof(unsigned);
    case MPI_INT64_T: return sizeof(int64_t);
    case MPI_UINT64_T: return sizeof(uint64_t);
    default: return 0;
    }
}
int copy(const void *src, void *dst, int count, MPI_Datatype type) {
    const size_t s = type_size(type);
    if (!s || count < 0) return MPI_ERR_OTHER;
    if (count && src != dst) std::memmove(dst, src, s * static_cast<size_t>(count));
    return MPI_SUCCESS;
}
}  // namespace

extern "C" {
int MPI_Init_thread(int *, char ***, int required, int *provided) {
    if (provided) *provided = required;
    return MPI_SUCCESS;
}
int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm, int code) { std::exit(code); }
int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }
int MPI_Error_string(int code, char *text, int *length) {
    *length = std::snprintf(text, MPI_MAX_ERROR_STRING, "single-rank MPI shim error %d", code);
    return MPI_SUCCESS;
}
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int,
                 void *recvbuf, int recvcount, MPI_Datatype, int source, int, MPI_Comm,
                 MPI_Status *) {
    if (dest != 0 || source != 0 || recvcount < sendcount) return MPI_ERR_OTHER;
    return copy(sendbuf, recvbuf, sendcount, sendtype);
}
int MPI_Alltoallv(const void *sendbuf, const int *sendcounts, const int *sdispls,
                  MPI_Datatype sendtype, void *recvbuf, const int *recvcounts, const int *rdispls,
                  MPI_Datatype, MPI_Comm) {
    if (recvcounts[0] != sendcounts[0]) return MPI_ERR_OTHER;
    const size_t s = type_size(sendtype);
    return copy(static_cast<const char *>(sendbuf) + s * sdispls[0],
                static_cast<char *>(recvbuf) + s * rdispls[0], sendcounts[0], sendtype);
}
int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Reduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op, int,
               MPI_Comm) {
    return copy(sendbuf, recvbuf, count, type);
}
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype type, MPI_Op,
                  MPI_Comm) {
    return copy(sendbuf, recvbuf, count, type);
}
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf, int,
                  MPI_Datatype, MPI_Comm) {
    return copy(sendbuf, recvbuf, sendcount, sendtype);
}
}
