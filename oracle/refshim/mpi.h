/*
 * Single-rank stand-in for <mpi.h>, used ONLY to compile the unmodified
 * reference sources into the test oracle (oracle/_ref).  Test infrastructure,
 * never shipped.
 *
 * Semantics (one process, one rank):
 *  - MPI_Cart_shift returns rank 0 in periodic dimensions and MPI_PROC_NULL
 *    otherwise, mirroring a 1x1x1 Cartesian communicator
 *    (reference: field_structures.h:1062-1115).
 *  - MPI_Isend/MPI_Irecv to/from self are matched by tag when MPI_Waitall runs;
 *    the halo exchanges use unique tags per face (field_structures.h:907-922,
 *    967-982, 1029-1044), so tag matching reproduces the self-exchange.
 *  - Reductions and broadcasts copy input to output.
 */
#ifndef ORACLE_REFSHIM_MPI_H
#define ORACLE_REFSHIM_MPI_H

#include <chrono>
#include <cstddef>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
struct MPI_Status { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; };

#define MPI_COMM_NULL (-1)
#define MPI_COMM_WORLD 0
#define MPI_PROC_NULL (-2)
#define MPI_INFO_NULL 0
#define MPI_SUCCESS 0
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_REQUEST_NULL (-1)

#define MPI_DOUBLE 8
#define MPI_INT 4
#define MPI_BYTE 1
#define MPI_LONG_LONG 16
#define MPI_UNSIGNED_LONG_LONG 17
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

namespace refshim {
struct Pending { bool is_send; void *buf; int bytes; int peer; int tag; bool live; };
inline std::vector<Pending> &table() { static std::vector<Pending> t; return t; }
inline int periods[3] = {0, 0, 0};
inline int type_bytes(MPI_Datatype t) {
    switch (t) { case MPI_DOUBLE: return 8; case MPI_INT: return 4; case MPI_BYTE: return 1;
                 case MPI_LONG_LONG: case MPI_UNSIGNED_LONG_LONG: return 8; default: return 8; }
}
inline int post(bool is_send, const void *buf, int count, MPI_Datatype t, int peer, int tag) {
    table().push_back(Pending{is_send, const_cast<void *>(buf), count * type_bytes(t), peer, tag, true});
    return (int)table().size() - 1;
}
inline void complete_all() {
    auto &t = table();
    for (auto &r : t) {
        if (!r.live || r.is_send) continue;
        if (r.peer == MPI_PROC_NULL) { r.live = false; continue; }
        for (auto &s : t) {
            if (s.live && s.is_send && s.tag == r.tag && s.peer != MPI_PROC_NULL) {
                std::memcpy(r.buf, s.buf, (size_t)r.bytes);
                s.live = false;
                break;
            }
        }
        r.live = false;
    }
    t.clear();
}
}  // namespace refshim

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return 0; }
inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *o) { *o = c; return 0; }
inline int MPI_Dims_create(int, int nd, int *dims) { for (int i = 0; i < nd; ++i) dims[i] = 1; return 0; }
inline int MPI_Cart_create(MPI_Comm, int nd, const int *, const int *per, int, MPI_Comm *c) {
    for (int i = 0; i < nd && i < 3; ++i) refshim::periods[i] = per[i];
    *c = 0; return 0;
}
inline int MPI_Cart_coords(MPI_Comm, int, int nd, int *co) { for (int i = 0; i < nd; ++i) co[i] = 0; return 0; }
inline int MPI_Cart_shift(MPI_Comm, int dim, int, int *src, int *dst) {
    int p = refshim::periods[dim] ? 0 : MPI_PROC_NULL; *src = p; *dst = p; return 0;
}
inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm, MPI_Request *rq) {
    *rq = refshim::post(true, b, n, t, d, tag); return 0;
}
inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm, MPI_Request *rq) {
    *rq = refshim::post(false, b, n, t, s, tag); return 0;
}
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { refshim::complete_all(); return 0; }
inline int MPI_Wait(MPI_Request *, MPI_Status *) { refshim::complete_all(); return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    std::memmove(out, in, (size_t)n * refshim::type_bytes(t)); return 0;
}
inline int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    std::memmove(out, in, (size_t)n * refshim::type_bytes(t)); return 0;
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
inline double MPI_Wtime() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}
#endif
