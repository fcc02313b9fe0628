// Test-infrastructure shim: a single-rank MPI covering the calls the
// GR-ray-tracer reference headers make.  Every collective on one rank is a copy
// from the send buffer to the receive buffer.  Nothing in the product links it.
#pragma once

#include <cstddef>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_DATATYPE_NULL (-1)
#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_UINT64_T 4
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

namespace mpi_shim {
inline std::vector<std::size_t>& derived_sizes() {
    static std::vector<std::size_t> sizes;
    return sizes;
}
inline std::size_t type_size(MPI_Datatype t) {
    switch (t) {
        case MPI_BYTE: return 1;
        case MPI_INT: return sizeof(int);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_UINT64_T: return 8;
        default: break;
    }
    const int index = t - 100;
    if (index >= 0 && static_cast<std::size_t>(index) < derived_sizes().size()) {
        return derived_sizes()[static_cast<std::size_t>(index)];
    }
    return 0;
}
inline void copy(const void* src, void* dst, int count, MPI_Datatype t) {
    if (src == dst || count <= 0) return;
    std::memmove(dst, src, static_cast<std::size_t>(count) * type_size(t));
}
}  // namespace mpi_shim

inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    mpi_shim::copy(s, r, n, t);
    return MPI_SUCCESS;
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    mpi_shim::copy(s, r, n, t);
    return MPI_SUCCESS;
}
inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    mpi_shim::copy(s, r, sn, st);
    return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    mpi_shim::copy(s, r, sn, st);
    return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st,
                         void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm) {
    const std::size_t size = mpi_shim::type_size(st);
    mpi_shim::copy(static_cast<const char*>(s) + static_cast<std::size_t>(sd[0]) * size,
                   static_cast<char*>(r) + static_cast<std::size_t>(rd[0]) * size, sc[0], st);
    return MPI_SUCCESS;
}
inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* out) {
    mpi_shim::derived_sizes().push_back(static_cast<std::size_t>(count) * mpi_shim::type_size(old));
    *out = 100 + static_cast<int>(mpi_shim::derived_sizes().size()) - 1;
    return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype* t) { *t = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
