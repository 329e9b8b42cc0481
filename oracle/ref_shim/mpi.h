/*
 * Single-rank stand-in for <mpi.h>.
 *
 * Test infrastructure only: it lets the reference implementation's own C++ sources (graph/, metrics/paths/,
 * external/mpi-wrapper, external/cpp-utility) compile and run unmodified on one process, so that their results
 * can pin the CPU restatement of the oracle. It is never linked into the product library.
 *
 * Semantics: MPI_COMM_WORLD has exactly one rank (0). Every collective degenerates into a copy of the local
 * contribution (reductions over one rank are the identity), RMA windows are plain local memory, non-blocking calls
 * complete immediately, and point-to-point messages to self go through a FIFO. Datatypes are integer handles into a
 * table of extents, which is all a one-rank copy needs to know about them.
 *
 * At one rank the reference's RMAWindow never calls MPI_Get/MPI_Put for its own memory
 * (external/mpi-wrapper/rma/RMAWindow.h:210-212, :510-512); they are implemented anyway for completeness.
 */
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <mutex>
#include <vector>

using MPI_Aint = std::ptrdiff_t;
using MPI_Datatype = int;
using MPI_Comm = int;
using MPI_Group = int;
using MPI_Op = int;
using MPI_Win = int;
using MPI_Request = int;
using MPI_Info = int;
using MPI_Errhandler = int;

struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    std::size_t count_bytes_;
};

constexpr int MPI_SUCCESS = 0;
constexpr int MPI_ERR_OTHER = 16;
constexpr int MPI_UNDEFINED = -32766;
constexpr int MPI_PROC_NULL = -2;
constexpr int MPI_ANY_SOURCE = -1;
constexpr int MPI_ANY_TAG = -1;

constexpr MPI_Comm MPI_COMM_NULL = 0;
constexpr MPI_Comm MPI_COMM_WORLD = 1;
constexpr MPI_Comm MPI_COMM_SELF = 2;
constexpr MPI_Group MPI_GROUP_NULL = 0;
constexpr MPI_Group MPI_GROUP_EMPTY = 1;
constexpr MPI_Win MPI_WIN_NULL = 0;
constexpr MPI_Info MPI_INFO_NULL = 0;
constexpr MPI_Errhandler MPI_ERRORS_RETURN = 1;
constexpr MPI_Request MPI_REQUEST_NULL = 0;

constexpr int MPI_THREAD_SINGLE = 0;
constexpr int MPI_THREAD_FUNNELED = 1;
constexpr int MPI_THREAD_SERIALIZED = 2;
constexpr int MPI_THREAD_MULTIPLE = 3;

constexpr int MPI_LOCK_EXCLUSIVE = 234;
constexpr int MPI_LOCK_SHARED = 235;

#define MPI_STATUS_IGNORE (static_cast<MPI_Status*>(nullptr))
#define MPI_STATUSES_IGNORE (static_cast<MPI_Status*>(nullptr))
#define MPI_IN_PLACE (reinterpret_cast<void*>(static_cast<std::intptr_t>(-1)))

/* Reduction operators: only their identity matters at one rank. */
constexpr MPI_Op MPI_SUM = 1, MPI_MAX = 2, MPI_MIN = 3, MPI_PROD = 4, MPI_LAND = 5, MPI_LOR = 6, MPI_BAND = 7, MPI_BOR = 8, MPI_BXOR = 9,
                 MPI_MAXLOC = 10, MPI_MINLOC = 11, MPI_LXOR = 12;

/* Predefined datatypes: handle == index into the extent table below. */
enum : int {
    MPI_DATATYPE_NULL = 0,
    MPI_BYTE,
    MPI_CHAR,
    MPI_SIGNED_CHAR,
    MPI_UNSIGNED_CHAR,
    MPI_SHORT,
    MPI_UNSIGNED_SHORT,
    MPI_INT,
    MPI_UNSIGNED,
    MPI_LONG,
    MPI_UNSIGNED_LONG,
    MPI_LONG_LONG,
    MPI_UNSIGNED_LONG_LONG,
    MPI_FLOAT,
    MPI_DOUBLE,
    MPI_LONG_DOUBLE,
    MPI_C_BOOL,
    MPI_INT8_T,
    MPI_INT16_T,
    MPI_INT32_T,
    MPI_INT64_T,
    MPI_UINT8_T,
    MPI_UINT16_T,
    MPI_UINT32_T,
    MPI_UINT64_T,
    MPI_2INT,
    MPI_SHORT_INT,
    MPI_LONG_INT,
    MPI_FLOAT_INT,
    MPI_DOUBLE_INT,
    MPI_LONG_DOUBLE_INT,
    MPI_UINT, /* not a real MPI name; kept so that stray uses compile */
    mpi_shim_predefined_count_
};
#define MPI_LONG_LONG_INT MPI_LONG_LONG

namespace mpi_shim {

struct TypeInfo {
    MPI_Aint lb;
    MPI_Aint extent;
};

inline std::vector<TypeInfo>& types() {
    static std::vector<TypeInfo> table = [] {
        struct LongDoubleInt {
            long double a;
            int b;
        };
        struct DoubleInt {
            double a;
            int b;
        };
        struct FloatInt {
            float a;
            int b;
        };
        struct LongInt {
            long a;
            int b;
        };
        struct ShortInt {
            short a;
            int b;
        };
        auto t = std::vector<TypeInfo>(mpi_shim_predefined_count_);
        const MPI_Aint sizes[] = { 0,
                                   1,
                                   sizeof(char),
                                   sizeof(signed char),
                                   sizeof(unsigned char),
                                   sizeof(short),
                                   sizeof(unsigned short),
                                   sizeof(int),
                                   sizeof(unsigned),
                                   sizeof(long),
                                   sizeof(unsigned long),
                                   sizeof(long long),
                                   sizeof(unsigned long long),
                                   sizeof(float),
                                   sizeof(double),
                                   sizeof(long double),
                                   sizeof(bool),
                                   1,
                                   2,
                                   4,
                                   8,
                                   1,
                                   2,
                                   4,
                                   8,
                                   2 * sizeof(int),
                                   sizeof(ShortInt),
                                   sizeof(LongInt),
                                   sizeof(FloatInt),
                                   sizeof(DoubleInt),
                                   sizeof(LongDoubleInt),
                                   sizeof(unsigned) };
        for (int i = 0; i < mpi_shim_predefined_count_; ++i) {
            t[static_cast<std::size_t>(i)] = { 0, sizes[i] };
        }
        return t;
    }();
    return table;
}

inline std::mutex& lock() {
    static std::mutex m;
    return m;
}

inline MPI_Aint extent(MPI_Datatype t) {
    std::lock_guard g{ lock() };
    return types().at(static_cast<std::size_t>(t)).extent;
}

inline MPI_Datatype add_type(MPI_Aint lb, MPI_Aint ext) {
    std::lock_guard g{ lock() };
    types().push_back({ lb, ext });
    return static_cast<MPI_Datatype>(types().size() - 1);
}

inline void copy(const void* src, void* dst, int count, MPI_Datatype type) {
    if (src == MPI_IN_PLACE || src == dst || count <= 0) {
        return;
    }
    std::memmove(dst, src, static_cast<std::size_t>(count) * static_cast<std::size_t>(extent(type)));
}

struct Message {
    int tag;
    std::vector<unsigned char> bytes;
};

inline std::deque<Message>& mailbox() {
    static std::deque<Message> box;
    return box;
}

struct Window {
    void* base;
    MPI_Aint size;
    int disp_unit;
};

inline std::vector<Window>& windows() {
    static std::vector<Window> w(1, Window{ nullptr, 0, 1 });
    return w;
}

inline unsigned char* window_address(MPI_Win win, MPI_Aint disp) {
    auto& w = windows().at(static_cast<std::size_t>(win));
    return static_cast<unsigned char*>(w.base) + disp * w.disp_unit;
}

} // namespace mpi_shim

/* ---------------------------------------------------------------- environment */
inline int MPI_Init_thread(int*, char***, int required, int* provided) {
    *provided = required;
    return MPI_SUCCESS;
}
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }
inline int MPI_Win_set_errhandler(MPI_Win, MPI_Errhandler) { return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int* size) {
    *size = 1;
    return MPI_SUCCESS;
}
inline int MPI_Comm_rank(MPI_Comm, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
inline int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) {
    *out = comm;
    return MPI_SUCCESS;
}
inline int MPI_Comm_split(MPI_Comm comm, int color, int, MPI_Comm* out) {
    *out = color == MPI_UNDEFINED ? MPI_COMM_NULL : comm;
    return MPI_SUCCESS;
}
inline int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm* out) {
    *out = group == MPI_GROUP_EMPTY ? MPI_COMM_NULL : comm;
    return MPI_SUCCESS;
}
inline int MPI_Comm_free(MPI_Comm* comm) {
    *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Comm_group(MPI_Comm, MPI_Group* group) {
    *group = 2;
    return MPI_SUCCESS;
}
inline int MPI_Group_size(MPI_Group group, int* size) {
    *size = group == MPI_GROUP_EMPTY ? 0 : 1;
    return MPI_SUCCESS;
}
inline int MPI_Group_rank(MPI_Group group, int* rank) {
    *rank = group == MPI_GROUP_EMPTY ? MPI_UNDEFINED : 0;
    return MPI_SUCCESS;
}
inline int MPI_Group_incl(MPI_Group group, int n, const int*, MPI_Group* out) {
    *out = n == 0 ? MPI_GROUP_EMPTY : group;
    return MPI_SUCCESS;
}
inline int MPI_Group_excl(MPI_Group group, int n, const int*, MPI_Group* out) {
    *out = n == 0 ? group : MPI_GROUP_EMPTY;
    return MPI_SUCCESS;
}
inline int MPI_Group_free(MPI_Group* group) {
    *group = MPI_GROUP_NULL;
    return MPI_SUCCESS;
}

/* Cartesian topologies over one rank: every dimension has extent 1, all coordinates are 0. */
inline int MPI_Dims_create(int, int ndims, int* dims) {
    for (int i = 0; i < ndims; ++i) {
        if (dims[i] == 0) {
            dims[i] = 1;
        }
    }
    return MPI_SUCCESS;
}
inline int MPI_Cart_create(MPI_Comm comm, int, const int*, const int*, int, MPI_Comm* out) {
    *out = comm;
    return MPI_SUCCESS;
}
inline int MPI_Cartdim_get(MPI_Comm, int* ndims) {
    *ndims = 1;
    return MPI_SUCCESS;
}
inline int MPI_Cart_get(MPI_Comm, int maxdims, int* dims, int* periods, int* coords) {
    for (int i = 0; i < maxdims; ++i) {
        dims[i] = 1;
        periods[i] = 0;
        coords[i] = 0;
    }
    return MPI_SUCCESS;
}
inline int MPI_Cart_rank(MPI_Comm, const int*, int* rank) {
    *rank = 0;
    return MPI_SUCCESS;
}
inline int MPI_Cart_coords(MPI_Comm, int, int maxdims, int* coords) {
    for (int i = 0; i < maxdims; ++i) {
        coords[i] = 0;
    }
    return MPI_SUCCESS;
}
inline int MPI_Cart_shift(MPI_Comm, int, int, int* source, int* dest) {
    *source = MPI_PROC_NULL;
    *dest = MPI_PROC_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Cart_sub(MPI_Comm comm, const int*, MPI_Comm* out) {
    *out = comm;
    return MPI_SUCCESS;
}

/* ---------------------------------------------------------------- datatypes */
inline int MPI_Get_address(const void* location, MPI_Aint* address) {
    *address = reinterpret_cast<MPI_Aint>(location);
    return MPI_SUCCESS;
}
inline int MPI_Type_contiguous(int count, MPI_Datatype old_type, MPI_Datatype* out) {
    *out = mpi_shim::add_type(0, count * mpi_shim::extent(old_type));
    return MPI_SUCCESS;
}
inline int MPI_Type_create_struct(int count, const int* block_lengths, const MPI_Aint* displacements, const MPI_Datatype* types, MPI_Datatype* out) {
    MPI_Aint end = 0;
    for (int i = 0; i < count; ++i) {
        const auto member_end = displacements[i] + block_lengths[i] * mpi_shim::extent(types[i]);
        end = member_end > end ? member_end : end;
    }
    *out = mpi_shim::add_type(0, end);
    return MPI_SUCCESS;
}
inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint lb, MPI_Aint extent, MPI_Datatype* out) {
    *out = mpi_shim::add_type(lb, extent);
    return MPI_SUCCESS;
}
inline int MPI_Type_get_extent(MPI_Datatype type, MPI_Aint* lb, MPI_Aint* extent) {
    *lb = 0;
    *extent = mpi_shim::extent(type);
    return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype*) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype* type) {
    *type = MPI_DATATYPE_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Get_count(const MPI_Status* status, MPI_Datatype type, int* count) {
    const auto ext = mpi_shim::extent(type);
    *count = ext == 0 ? 0 : static_cast<int>(static_cast<MPI_Aint>(status->count_bytes_) / ext);
    return MPI_SUCCESS;
}

/* ---------------------------------------------------------------- memory */
inline int MPI_Alloc_mem(MPI_Aint size, MPI_Info, void* base_ptr) {
    void* p = std::malloc(size > 0 ? static_cast<std::size_t>(size) : 1);
    std::memcpy(base_ptr, &p, sizeof(void*));
    return p == nullptr ? MPI_ERR_OTHER : MPI_SUCCESS;
}
inline int MPI_Free_mem(void* base) {
    std::free(base);
    return MPI_SUCCESS;
}

/* ---------------------------------------------------------------- synchronisation and requests */
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Ibarrier(MPI_Comm, MPI_Request* request) {
    *request = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Wait(MPI_Request* request, MPI_Status*) {
    *request = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Waitall(int count, MPI_Request* requests, MPI_Status*) {
    for (int i = 0; i < count; ++i) {
        requests[i] = MPI_REQUEST_NULL;
    }
    return MPI_SUCCESS;
}
inline int MPI_Test(MPI_Request* request, int* flag, MPI_Status*) {
    *request = MPI_REQUEST_NULL;
    *flag = 1;
    return MPI_SUCCESS;
}

/* ---------------------------------------------------------------- collectives (one rank: copies) */
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, int, MPI_Comm) {
    mpi_shim::copy(send, recv, count, type);
    return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    mpi_shim::copy(send, recv, count, type);
    return MPI_SUCCESS;
}
inline int MPI_Scan(const void* send, void* recv, int count, MPI_Datatype type, MPI_Op, MPI_Comm) {
    mpi_shim::copy(send, recv, count, type);
    return MPI_SUCCESS;
}
inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) {
    /* The receive buffer of rank 0 is undefined for an exclusive scan. */
    return MPI_SUCCESS;
}
inline int MPI_Gather(const void* send, int send_count, MPI_Datatype send_type, void* recv, int, MPI_Datatype, int, MPI_Comm) {
    mpi_shim::copy(send, recv, send_count, send_type);
    return MPI_SUCCESS;
}
inline int MPI_Gatherv(const void* send, int send_count, MPI_Datatype send_type, void* recv, const int*, const int* displs, MPI_Datatype recv_type, int,
                       MPI_Comm) {
    if (recv != nullptr) {
        mpi_shim::copy(send, static_cast<unsigned char*>(recv) + displs[0] * mpi_shim::extent(recv_type), send_count, send_type);
    }
    return MPI_SUCCESS;
}
inline int MPI_Allgather(const void* send, int send_count, MPI_Datatype send_type, void* recv, int, MPI_Datatype, MPI_Comm) {
    mpi_shim::copy(send, recv, send_count, send_type);
    return MPI_SUCCESS;
}
inline int MPI_Allgatherv(const void* send, int send_count, MPI_Datatype send_type, void* recv, const int*, const int* displs, MPI_Datatype recv_type,
                          MPI_Comm) {
    mpi_shim::copy(send, static_cast<unsigned char*>(recv) + displs[0] * mpi_shim::extent(recv_type), send_count, send_type);
    return MPI_SUCCESS;
}
inline int MPI_Scatter(const void* send, int, MPI_Datatype, void* recv, int recv_count, MPI_Datatype recv_type, int, MPI_Comm) {
    mpi_shim::copy(send, recv, recv_count, recv_type);
    return MPI_SUCCESS;
}
inline int MPI_Scatterv(const void* send, const int*, const int* displs, MPI_Datatype send_type, void* recv, int recv_count, MPI_Datatype recv_type, int,
                        MPI_Comm) {
    if (recv != MPI_IN_PLACE) {
        mpi_shim::copy(static_cast<const unsigned char*>(send) + displs[0] * mpi_shim::extent(send_type), recv, recv_count, recv_type);
    }
    return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void* send, int send_count, MPI_Datatype send_type, void* recv, int, MPI_Datatype, MPI_Comm) {
    mpi_shim::copy(send, recv, send_count, send_type);
    return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void* send, const int* send_counts, const int* send_displs, MPI_Datatype send_type, void* recv, const int*,
                         const int* recv_displs, MPI_Datatype recv_type, MPI_Comm) {
    mpi_shim::copy(static_cast<const unsigned char*>(send) + send_displs[0] * mpi_shim::extent(send_type),
                   static_cast<unsigned char*>(recv) + recv_displs[0] * mpi_shim::extent(recv_type), send_counts[0], send_type);
    return MPI_SUCCESS;
}

#define MPI_SHIM_NONBLOCKING(name, blocking, params, args)                                                                                                    \
    inline int name params {                                                                                                                                  \
        *request = MPI_REQUEST_NULL;                                                                                                                          \
        return blocking args;                                                                                                                                 \
    }
MPI_SHIM_NONBLOCKING(MPI_Ibcast, MPI_Bcast, (void* b, int c, MPI_Datatype t, int r, MPI_Comm m, MPI_Request* request), (b, c, t, r, m))
MPI_SHIM_NONBLOCKING(MPI_Ireduce, MPI_Reduce, (const void* s, void* r, int c, MPI_Datatype t, MPI_Op o, int root, MPI_Comm m, MPI_Request* request),
                     (s, r, c, t, o, root, m))
MPI_SHIM_NONBLOCKING(MPI_Iallreduce, MPI_Allreduce, (const void* s, void* r, int c, MPI_Datatype t, MPI_Op o, MPI_Comm m, MPI_Request* request),
                     (s, r, c, t, o, m))
MPI_SHIM_NONBLOCKING(MPI_Iscan, MPI_Scan, (const void* s, void* r, int c, MPI_Datatype t, MPI_Op o, MPI_Comm m, MPI_Request* request), (s, r, c, t, o, m))
MPI_SHIM_NONBLOCKING(MPI_Iexscan, MPI_Exscan, (const void* s, void* r, int c, MPI_Datatype t, MPI_Op o, MPI_Comm m, MPI_Request* request),
                     (s, r, c, t, o, m))
MPI_SHIM_NONBLOCKING(MPI_Igather, MPI_Gather,
                     (const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, int root, MPI_Comm m, MPI_Request* request),
                     (s, sc, st, r, rc, rt, root, m))
MPI_SHIM_NONBLOCKING(MPI_Igatherv, MPI_Gatherv,
                     (const void* s, int sc, MPI_Datatype st, void* r, const int* rc, const int* d, MPI_Datatype rt, int root, MPI_Comm m,
                      MPI_Request* request),
                     (s, sc, st, r, rc, d, rt, root, m))
MPI_SHIM_NONBLOCKING(MPI_Iallgather, MPI_Allgather,
                     (const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, MPI_Comm m, MPI_Request* request), (s, sc, st, r, rc, rt, m))
MPI_SHIM_NONBLOCKING(MPI_Iallgatherv, MPI_Allgatherv,
                     (const void* s, int sc, MPI_Datatype st, void* r, const int* rc, const int* d, MPI_Datatype rt, MPI_Comm m, MPI_Request* request),
                     (s, sc, st, r, rc, d, rt, m))
MPI_SHIM_NONBLOCKING(MPI_Iscatter, MPI_Scatter,
                     (const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, int root, MPI_Comm m, MPI_Request* request),
                     (s, sc, st, r, rc, rt, root, m))
MPI_SHIM_NONBLOCKING(MPI_Iscatterv, MPI_Scatterv,
                     (const void* s, const int* sc, const int* d, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, int root, MPI_Comm m,
                      MPI_Request* request),
                     (s, sc, d, st, r, rc, rt, root, m))
MPI_SHIM_NONBLOCKING(MPI_Ialltoall, MPI_Alltoall,
                     (const void* s, int sc, MPI_Datatype st, void* r, int rc, MPI_Datatype rt, MPI_Comm m, MPI_Request* request), (s, sc, st, r, rc, rt, m))
MPI_SHIM_NONBLOCKING(MPI_Ialltoallv, MPI_Alltoallv,
                     (const void* s, const int* sc, const int* sd, MPI_Datatype st, void* r, const int* rc, const int* rd, MPI_Datatype rt, MPI_Comm m,
                      MPI_Request* request),
                     (s, sc, sd, st, r, rc, rd, rt, m))
#undef MPI_SHIM_NONBLOCKING

/* ---------------------------------------------------------------- point to point (self messages only) */
inline int MPI_Send(const void* buffer, int count, MPI_Datatype type, int, int tag, MPI_Comm) {
    const auto bytes = static_cast<std::size_t>(count) * static_cast<std::size_t>(mpi_shim::extent(type));
    auto message = mpi_shim::Message{ tag, std::vector<unsigned char>(bytes) };
    if (bytes > 0) {
        std::memcpy(message.bytes.data(), buffer, bytes);
    }
    mpi_shim::mailbox().push_back(std::move(message));
    return MPI_SUCCESS;
}
inline int MPI_Isend(const void* buffer, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm, MPI_Request* request) {
    *request = MPI_REQUEST_NULL;
    return MPI_Send(buffer, count, type, dest, tag, comm);
}
inline int MPI_Recv(void* buffer, int count, MPI_Datatype type, int, int tag, MPI_Comm, MPI_Status* status) {
    auto& box = mpi_shim::mailbox();
    for (auto it = box.begin(); it != box.end(); ++it) {
        if (tag == MPI_ANY_TAG || it->tag == tag) {
            const auto capacity = static_cast<std::size_t>(count) * static_cast<std::size_t>(mpi_shim::extent(type));
            const auto bytes = it->bytes.size() < capacity ? it->bytes.size() : capacity;
            if (bytes > 0) {
                std::memcpy(buffer, it->bytes.data(), bytes);
            }
            if (status != nullptr) {
                *status = MPI_Status{ 0, it->tag, MPI_SUCCESS, bytes };
            }
            box.erase(it);
            return MPI_SUCCESS;
        }
    }
    return MPI_ERR_OTHER; /* a one-rank receive without a matching self-send would block forever */
}
inline int MPI_Irecv(void* buffer, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm, MPI_Request* request) {
    *request = MPI_REQUEST_NULL;
    return MPI_Recv(buffer, count, type, source, tag, comm, MPI_STATUS_IGNORE);
}
inline int MPI_Iprobe(int, int tag, MPI_Comm, int* flag, MPI_Status* status) {
    *flag = 0;
    for (const auto& message : mpi_shim::mailbox()) {
        if (tag == MPI_ANY_TAG || message.tag == tag) {
            *flag = 1;
            if (status != nullptr) {
                *status = MPI_Status{ 0, message.tag, MPI_SUCCESS, message.bytes.size() };
            }
            break;
        }
    }
    return MPI_SUCCESS;
}
inline int MPI_Probe(int source, int tag, MPI_Comm comm, MPI_Status* status) {
    int flag = 0;
    MPI_Iprobe(source, tag, comm, &flag, status);
    return flag ? MPI_SUCCESS : MPI_ERR_OTHER;
}
inline int MPI_Sendrecv(const void* send, int send_count, MPI_Datatype send_type, int, int, void* recv, int, MPI_Datatype, int, int, MPI_Comm,
                        MPI_Status* status) {
    mpi_shim::copy(send, recv, send_count, send_type);
    if (status != nullptr) {
        *status = MPI_Status{ 0, 0, MPI_SUCCESS, static_cast<std::size_t>(send_count * mpi_shim::extent(send_type)) };
    }
    return MPI_SUCCESS;
}
inline int MPI_Sendrecv_replace(void*, int, MPI_Datatype, int, int, int, int, MPI_Comm, MPI_Status*) { return MPI_SUCCESS; }

/* ---------------------------------------------------------------- one-sided (local memory) */
inline int MPI_Win_create(void* base, MPI_Aint size, int disp_unit, MPI_Info, MPI_Comm, MPI_Win* win) {
    mpi_shim::windows().push_back({ base, size, disp_unit });
    *win = static_cast<MPI_Win>(mpi_shim::windows().size() - 1);
    return MPI_SUCCESS;
}
inline int MPI_Win_free(MPI_Win* win) {
    *win = MPI_WIN_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Win_lock(int, int, int, MPI_Win) { return MPI_SUCCESS; }
inline int MPI_Win_unlock(int, MPI_Win) { return MPI_SUCCESS; }
inline int MPI_Win_lock_all(int, MPI_Win) { return MPI_SUCCESS; }
inline int MPI_Win_unlock_all(MPI_Win) { return MPI_SUCCESS; }
inline int MPI_Win_flush_all(MPI_Win) { return MPI_SUCCESS; }
inline int MPI_Win_fence(int, MPI_Win) { return MPI_SUCCESS; }
inline int MPI_Get(void* origin, int origin_count, MPI_Datatype origin_type, int, MPI_Aint target_disp, int, MPI_Datatype, MPI_Win win) {
    mpi_shim::copy(mpi_shim::window_address(win, target_disp), origin, origin_count, origin_type);
    return MPI_SUCCESS;
}
inline int MPI_Rget(void* origin, int origin_count, MPI_Datatype origin_type, int rank, MPI_Aint target_disp, int target_count, MPI_Datatype target_type,
                    MPI_Win win, MPI_Request* request) {
    *request = MPI_REQUEST_NULL;
    return MPI_Get(origin, origin_count, origin_type, rank, target_disp, target_count, target_type, win);
}
inline int MPI_Put(const void* origin, int origin_count, MPI_Datatype origin_type, int, MPI_Aint target_disp, int, MPI_Datatype, MPI_Win win) {
    mpi_shim::copy(origin, mpi_shim::window_address(win, target_disp), origin_count, origin_type);
    return MPI_SUCCESS;
}
inline int MPI_Accumulate(const void*, int, MPI_Datatype, int, MPI_Aint, int, MPI_Datatype, MPI_Op, MPI_Win) {
    /* Not on the shortest-path hot path; a one-rank accumulate would need the operator's arithmetic. */
    return MPI_ERR_OTHER;
}
