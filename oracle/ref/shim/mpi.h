/*
 * Single-rank MPI stand-in used ONLY to compile the reference's own flow
 * sources into the CPU oracle (oracle/_ref).  Test infrastructure, not product.
 *
 * With one rank every point-to-point message in the reference is a send to
 * itself: `shift()` (include/Math/lattice.h:360-594 of the reference) posts
 * MPI_Isend of the wrapped face and then MPI_Irecv from the same rank, so
 * Irecv copies the bytes the matching Isend recorded.  Allreduce over one
 * rank is the identity (the reference passes aliased buffers,
 * src/Observables/superobs.cpp:24-28).  MPI-IO maps onto stdio
 * (src/InputOutput/inputconf.cpp:114-155 reads with MPI_File_read_at).
 */
#pragma once
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef FILE* MPI_File;
struct MPI_Status { int source, tag, error; };

#define MPI_COMM_WORLD 0
#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_SUM 1
#define MPI_INFO_NULL 0
#define MPI_MODE_CREATE 1
#define MPI_MODE_RDWR 2
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

namespace ymshim {
/* the one outstanding self-send: shift() posts exactly one Isend before its Irecv */
struct PendingSend { const void* buf; size_t bytes; };
inline PendingSend& pending() { static PendingSend p = {nullptr, 0}; return p; }
inline size_t type_bytes(MPI_Datatype t) { return (size_t)t; }
}

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int code) { std::exit(code ? code : 1); }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }

inline int MPI_Cart_create(MPI_Comm c, int, const int*, const int*, int, MPI_Comm* out) {
    *out = c; return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int ndims, int* coords) {
    for (int i = 0; i < ndims; ++i) coords[i] = 0;
    return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm, int, int, int* src, int* dst) {
    *src = 0; *dst = 0; return MPI_SUCCESS;
}
inline int MPI_Cart_rank(MPI_Comm, const int*, int* rank) { *rank = 0; return MPI_SUCCESS; }

inline int MPI_Isend(const void* buf, int count, MPI_Datatype t, int, int, MPI_Comm, MPI_Request* req) {
    ymshim::pending().buf = buf;
    ymshim::pending().bytes = (size_t)count * ymshim::type_bytes(t);
    *req = 1;
    return MPI_SUCCESS;
}
inline int MPI_Irecv(void* buf, int count, MPI_Datatype t, int, int, MPI_Comm, MPI_Request* req) {
    size_t want = (size_t)count * ymshim::type_bytes(t);
    ymshim::PendingSend& p = ymshim::pending();
    if (!p.buf || p.bytes != want) {
        std::fprintf(stderr, "mpi shim: receive without matching self-send\n");
        std::exit(3);
    }
    std::memcpy(buf, p.buf, want);
    p.buf = nullptr;
    *req = 2;
    return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
inline int MPI_Sendrecv(const void* sb, int sc, MPI_Datatype st, int, int, void* rb, int, MPI_Datatype,
                        int, int, MPI_Comm, MPI_Status*) {
    std::memmove(rb, sb, (size_t)sc * ymshim::type_bytes(st));
    return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void* sb, void* rb, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
    if (sb != rb) std::memmove(rb, sb, (size_t)count * ymshim::type_bytes(t));
    return MPI_SUCCESS;
}

inline int MPI_File_open(MPI_Comm, const char* name, int, MPI_Info, MPI_File* f) {
    *f = std::fopen(name, "rb");
    if (!*f) {
        std::fprintf(stderr, "mpi shim: cannot open %s\n", name);
        std::exit(4);
    }
    return MPI_SUCCESS;
}
inline int MPI_File_read_at(MPI_File f, MPI_Offset off, void* buf, int count, MPI_Datatype t, MPI_Status*) {
    size_t n = (size_t)count * ymshim::type_bytes(t);
    if (std::fseek(f, (long)off, SEEK_SET) != 0 || std::fread(buf, 1, n, f) != n) {
        std::fprintf(stderr, "mpi shim: short read at offset %lld\n", (long long)off);
        std::exit(5);
    }
    return MPI_SUCCESS;
}
inline int MPI_File_write_at(MPI_File, MPI_Offset, const void*, int, MPI_Datatype, MPI_Status*) {
    return MPI_SUCCESS;
}
inline int MPI_File_close(MPI_File* f) {
    if (*f) std::fclose(*f);
    *f = nullptr;
    return MPI_SUCCESS;
}
