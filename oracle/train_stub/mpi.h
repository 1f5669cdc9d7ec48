// Single-process stand-in for the MPI calls of the reference's training
// library (src/libnnptrain, application/nnp-train.cpp), written for this
// project and used ONLY to compile the reference's nnp-train into the test
// oracle (oracle/_ref/nnp-train).  With one process every collective is a
// copy from the send buffer to the receive buffer (or nothing with
// MPI_IN_PLACE); point-to-point calls are never reached on one process and
// throw if they are.
#ifndef N2P2B200_MPI_STUB_H
#define N2P2B200_MPI_STUB_H

#include <cstddef>
#include <cstring>
#include <stdexcept>
#include <string>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
struct MPI_Status
{
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
};

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_IN_PLACE ((void*)1)

// Datatypes encode their size in bytes.
#define MPI_CHAR 1
#define MPI_UNSIGNED_CHAR 1
#define MPI_PACKED 1
#define MPI_SHORT 2
#define MPI_UNSIGNED_SHORT 2
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 4
#define MPI_LONG 8
#define MPI_UNSIGNED_LONG 8
#define MPI_LONG_LONG 8
#define MPI_UNSIGNED_LONG_LONG 8
#define MPI_INT64_T 8
#define MPI_DOUBLE 8

#define MPI_SUM 0
#define MPI_MIN 1
#define MPI_MAX 2

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }
inline int MPI_Comm_free(MPI_Comm*) { return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Get_processor_name(char* name, int* len)
{
    std::strcpy(name, "localhost");
    *len = 9;
    return MPI_SUCCESS;
}

namespace n2p2b200_mpi_stub {
inline void copy(const void* send, void* recv, int count, MPI_Datatype t)
{
    if (send != MPI_IN_PLACE && send != recv && count > 0) std::memmove(recv, send, (std::size_t)count * t);
}
[[noreturn]] inline void unreachable(const char* what)
{
    throw std::runtime_error(std::string("MPI stub: ") + what + " needs more than one process");
}
} // namespace n2p2b200_mpi_stub

inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm)
{
    n2p2b200_mpi_stub::copy(s, r, n, t);
    return MPI_SUCCESS;
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm)
{
    n2p2b200_mpi_stub::copy(s, r, n, t);
    return MPI_SUCCESS;
}
inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm)
{
    n2p2b200_mpi_stub::copy(s, r, sn, st);
    return MPI_SUCCESS;
}
inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm)
{
    n2p2b200_mpi_stub::copy(s, r, sn, st);
    return MPI_SUCCESS;
}
inline int MPI_Gatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs, MPI_Datatype rt,
                       int, MPI_Comm)
{
    if (s != MPI_IN_PLACE) n2p2b200_mpi_stub::copy(s, (char*)r + (std::size_t)displs[0] * rt, sn, st);
    return MPI_SUCCESS;
}
inline int MPI_Allgatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs,
                          MPI_Datatype rt, MPI_Comm)
{
    if (s != MPI_IN_PLACE) n2p2b200_mpi_stub::copy(s, (char*)r + (std::size_t)displs[0] * rt, sn, st);
    return MPI_SUCCESS;
}
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { n2p2b200_mpi_stub::unreachable("MPI_Send"); }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*)
{
    n2p2b200_mpi_stub::unreachable("MPI_Recv");
}
inline int MPI_Pack_size(int n, MPI_Datatype t, MPI_Comm, int* size)
{
    *size = n * t;
    return MPI_SUCCESS;
}
inline int MPI_Pack(const void* in, int n, MPI_Datatype t, void* out, int, int* pos, MPI_Comm)
{
    std::memcpy((char*)out + *pos, in, (std::size_t)n * t);
    *pos += n * t;
    return MPI_SUCCESS;
}
inline int MPI_Unpack(const void* in, int, int* pos, void* out, int n, MPI_Datatype t, MPI_Comm)
{
    std::memcpy(out, (const char*)in + *pos, (std::size_t)n * t);
    *pos += n * t;
    return MPI_SUCCESS;
}

#endif
