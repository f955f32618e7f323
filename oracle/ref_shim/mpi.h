/*
 * Single-rank MPI stand-in used only to compile the reference LYNX CPU sources
 * into the test oracle (oracle/_ref).  It is test infrastructure: no product
 * code includes it.  Every communicator has exactly one rank, so collectives
 * reduce to copies from the send buffer to the receive buffer.
 */
#pragma once
#include <cstring>
#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;

#define MPI_COMM_NULL (-1)
#define MPI_COMM_WORLD 0
#define MPI_COMM_SELF 1
#define MPI_INFO_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_COMM_TYPE_SHARED 1
#define MPI_SUCCESS 0

#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_C_DOUBLE_COMPLEX 3
#define MPI_CHAR 4
#define MPI_BYTE 5
#define MPI_LONG 6
#define MPI_UNSIGNED 7
#define MPI_LONG_LONG 8
#define MPI_CXX_BOOL 9
#define MPI_C_BOOL 9

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LOR 4
#define MPI_LAND 5

#define MPI_IN_PLACE ((void*)1)

inline std::size_t lynx_mpi_stub_size(MPI_Datatype t) {
    switch (t) {
        case MPI_INT: return sizeof(int);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_C_DOUBLE_COMPLEX: return 2 * sizeof(double);
        case MPI_CHAR: case MPI_BYTE: return 1;
        case MPI_LONG: return sizeof(long);
        case MPI_UNSIGNED: return sizeof(unsigned);
        case MPI_LONG_LONG: return sizeof(long long);
        case MPI_CXX_BOOL: return sizeof(bool);
        default: return 1;
    }
}

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Initialized(int* f) { *f = 1; return 0; }
inline int MPI_Finalized(int* f) { *f = 0; return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Abort(MPI_Comm, int) { return 0; }
inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* n) { *n = c; return 0; }
inline int MPI_Comm_split(MPI_Comm, int color, int, MPI_Comm* n) {
    *n = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : 2;
    return 0;
}
inline int MPI_Comm_split_type(MPI_Comm, int, int, MPI_Info, MPI_Comm* n) { *n = 2; return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) std::memcpy(r, s, n * lynx_mpi_stub_size(t));
    return 0;
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) std::memcpy(r, s, n * lynx_mpi_stub_size(t));
    return 0;
}
inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) std::memcpy(r, s, n * lynx_mpi_stub_size(t));
    return 0;
}
inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* displs,
                          MPI_Datatype, MPI_Comm) {
    if (s != MPI_IN_PLACE)
        std::memmove(static_cast<char*>(r) + (displs ? displs[0] : 0) * lynx_mpi_stub_size(t), s,
                     n * lynx_mpi_stub_size(t));
    return 0;
}
inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
    if (s != MPI_IN_PLACE && s != r) std::memcpy(r, s, n * lynx_mpi_stub_size(t));
    return 0;
}
inline double MPI_Wtime() { return 0.0; }
// Point-to-point on one rank: a send to oneself is received at once.
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
inline int MPI_Sendrecv(const void* s, int n, MPI_Datatype t, int, int, void* r, int, MPI_Datatype, int, int,
                        MPI_Comm, MPI_Status*) {
    if (s != r) std::memmove(r, s, n * lynx_mpi_stub_size(t));
    return 0;
}
