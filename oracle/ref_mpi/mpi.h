/*
 * In-process stand-in for <mpi.h>, used only to compile and run the
 * reference's own CPU sources in the test-only checkers under oracle/_ref:
 *   - the kernel templates, Euclidean primitives and structured generator
 *     (libcupcfd_ref.so), which only register MPI datatypes;
 *   - the reference's mesh construction path (MeshConfig ->
 *     PartitionerNaive -> CupCfdSoAMesh::addData / finalize), its
 *     distributed adjacency list and exchange patterns, which call the
 *     collectives, point-to-point and one-sided operations below.
 *
 * TEST INFRASTRUCTURE ONLY: nothing in the shipped library includes this.
 *
 * Ranks are threads of one process. cupcfd_oracle_mpi::run_ranks(P, body)
 * runs body(rank) on P threads that form MPI_COMM_WORLD; outside it the
 * world is the calling thread alone (rank 0 of 1). The reference's mesh path
 * needs more than one rank: DistributedAdjacencyList::finalize broadcasts
 * each rank's ghost-node list, and its BroadcastMPI wrapper returns
 * E_NO_DATA for an empty list, which every rank of a one-rank world has
 * (DistributedAdjacencyList.cpp:427, BroadcastMPI.ipp:28-30); the
 * reference's own mesh tests run on 4 ranks.
 *
 * Semantics follow MPI for the calls the reference makes:
 *   - collectives: each rank deposits its buffers, the ranks meet at a
 *     barrier, each copies what it receives from the others' buffers, and a
 *     second barrier ends the call; reductions run over ranks in rank order;
 *   - point to point: a send is buffered at once, a receive is matched by
 *     (source, tag) in posting order when MPI_Waitall runs;
 *   - one-sided: MPI_Win_create is collective and records every rank's
 *     window; a put writes into the target's window memory; fences are
 *     barriers; post/start/complete/wait are counted per window and rank.
 * Every wait gives up after WAIT_SECONDS and aborts the process with a
 * message, so a mismatched call sequence ends a test instead of hanging it.
 * Datatype extents are tracked so buffers move by the right byte counts;
 * derived types carry the extent MPI_Type_create_struct / _resized give.
 */
#ifndef CUPCFD_ORACLE_MPI_STUB_H
#define CUPCFD_ORACLE_MPI_STUB_H

#include <stddef.h>
#include <string.h>

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Win;
typedef int MPI_Group;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_DATATYPE_NULL 0
#define MPI_INT 1
#define MPI_DOUBLE 2
#define MPI_FLOAT 3
#define MPI_LONG 4
#define MPI_CXX_BOOL 5
#define MPI_CHAR 6
#define MPI_UNSIGNED 7
#define MPI_BYTE 8
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_PROD 4
#define MPI_INFO_NULL 0
#define MPI_WIN_NULL 0
#define MPI_GROUP_EMPTY 0
#define MPI_GROUP_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_MODE_NOPUT 1
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

#ifdef __cplusplus
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

namespace cupcfd_oracle_mpi {

constexpr int WAIT_SECONDS = 120;

struct World {
    std::mutex mu;
    std::condition_variable cv;
    int size = 1;
    // barrier
    int arrived = 0;
    long generation = 0;
    // per-rank deposits of the collective in progress
    struct Slot {
        const void *s = nullptr;
        const int *counts = nullptr, *displs = nullptr;
        int n = 0;
        void *extra = nullptr;
    };
    std::vector<Slot> slots = std::vector<Slot>(1);
    // derived datatype extents (handle - 100)
    std::vector<long> derived;
    // point to point: buffered messages per (source, dest, tag)
    std::map<std::tuple<int, int, int>, std::deque<std::vector<char>>> mail;
    struct Recv { int src, tag; void *buf; long bytes; };
    std::map<int, Recv> recvs;  // request -> posted receive
    int nextRequest = 1;
    // groups (handle - 1 -> ranks), windows (handle - 1 -> per-rank base and unit)
    std::vector<std::vector<int>> groups;
    struct Win { std::vector<char *> base; std::vector<long> unit; std::vector<long> posted, completed;
                 std::vector<std::vector<long>> started; std::vector<int> postGroup, startGroup; };
    std::vector<Win> wins;
    std::vector<int> winCount = std::vector<int>(1, 0);  // windows created so far, per rank
};
inline World &world() { static World w; return w; }
inline int &my_rank() { static thread_local int r = 0; return r; }

[[noreturn]] inline void fail(const char *what) {
    std::fprintf(stderr, "oracle mpi stand-in: %s (rank %d)\n", what, my_rank());
    std::abort();
}

// waits on the world's condition variable for pred, at most WAIT_SECONDS
template <class P>
inline void wait_for(std::unique_lock<std::mutex> &lk, P pred, const char *what) {
    if (!world().cv.wait_for(lk, std::chrono::seconds(WAIT_SECONDS), pred)) fail(what);
}

inline void barrier_locked(std::unique_lock<std::mutex> &lk) {
    World &w = world();
    long gen = w.generation;
    if (++w.arrived == w.size) {
        w.arrived = 0;
        w.generation++;
        w.cv.notify_all();
    } else {
        wait_for(lk, [&] { return w.generation != gen; }, "barrier timed out");
    }
}
inline void barrier() {
    std::unique_lock<std::mutex> lk(world().mu);
    barrier_locked(lk);
}

inline long extent(MPI_Datatype t) {
    switch (t) {
        case MPI_INT: case MPI_FLOAT: case MPI_UNSIGNED: return 4;
        case MPI_DOUBLE: case MPI_LONG: return 8;
        case MPI_CXX_BOOL: case MPI_CHAR: case MPI_BYTE: return 1;
        default: break;
    }
    std::lock_guard<std::mutex> lk(world().mu);
    if (t >= 100 && t - 100 < (int) world().derived.size()) return world().derived[(size_t) t - 100];
    fail("unknown datatype");
}
inline MPI_Datatype new_type(long ext) {
    std::lock_guard<std::mutex> lk(world().mu);
    world().derived.push_back(ext);
    return 100 + (int) world().derived.size() - 1;
}
inline void copy(const void *src, long bytes, void *dst, long room) {
    if (bytes > room) fail("receive buffer too small");
    if (bytes > 0 && src != dst) memmove(dst, src, (size_t) bytes);
}

// Deposit this rank's buffers, meet, run `take` (reads the other ranks'
// deposits), meet again so no deposit goes away while another rank reads it.
inline void collective(const World::Slot &mine, const std::function<void(const std::vector<World::Slot> &)> &take) {
    World &w = world();
    {
        std::unique_lock<std::mutex> lk(w.mu);
        w.slots[(size_t) my_rank()] = mine;
        barrier_locked(lk);
    }
    take(w.slots);
    barrier();
}

template <class T>
inline void reduce_into(T *acc, const T *x, int n, MPI_Op op, bool first) {
    for (int i = 0; i < n; i++) {
        if (first) { acc[i] = x[i]; continue; }
        switch (op) {
            case MPI_SUM: acc[i] = acc[i] + x[i]; break;
            case MPI_PROD: acc[i] = acc[i] * x[i]; break;
            case MPI_MAX: acc[i] = x[i] > acc[i] ? x[i] : acc[i]; break;
            case MPI_MIN: acc[i] = x[i] < acc[i] ? x[i] : acc[i]; break;
            default: fail("unknown reduction");
        }
    }
}
inline void reduce_all(const std::vector<World::Slot> &sl, void *r, int n, MPI_Datatype t, MPI_Op op) {
    std::vector<char> acc((size_t) n * (size_t) extent(t));
    for (size_t j = 0; j < sl.size(); j++) {
        const bool first = j == 0;
        switch (t) {
            case MPI_INT: reduce_into((int *) acc.data(), (const int *) sl[j].s, n, op, first); break;
            case MPI_UNSIGNED: reduce_into((unsigned *) acc.data(), (const unsigned *) sl[j].s, n, op, first); break;
            case MPI_LONG: reduce_into((long *) acc.data(), (const long *) sl[j].s, n, op, first); break;
            case MPI_FLOAT: reduce_into((float *) acc.data(), (const float *) sl[j].s, n, op, first); break;
            case MPI_DOUBLE: reduce_into((double *) acc.data(), (const double *) sl[j].s, n, op, first); break;
            case MPI_CXX_BOOL: reduce_into((bool *) acc.data(), (const bool *) sl[j].s, n, op, first); break;
            default: fail("reduction over an unsupported datatype");
        }
    }
    memcpy(r, acc.data(), acc.size());
}

// Runs body(rank) on `ranks` threads forming MPI_COMM_WORLD; returns when
// all have finished. Not re-entrant.
inline void run_ranks(int ranks, const std::function<void(int)> &body) {
    World &w = world();
    {
        std::lock_guard<std::mutex> lk(w.mu);
        w.size = ranks;
        w.arrived = 0;
        w.slots.assign((size_t) ranks, World::Slot());
        w.winCount.assign((size_t) ranks, 0);
        w.wins.clear();
        w.mail.clear();
        w.recvs.clear();
    }
    std::vector<std::thread> th;
    for (int r = 0; r < ranks; r++)
        th.emplace_back([r, &body] {
            my_rank() = r;
            body(r);
        });
    for (std::thread &t : th) t.join();
    std::lock_guard<std::mutex> lk(w.mu);
    w.size = 1;
    w.slots.assign(1, World::Slot());
    w.winCount.assign(1, 0);
    w.wins.clear();
}

}  // namespace cupcfd_oracle_mpi


inline int MPI_Type_create_struct(int n, const int *len, const MPI_Aint *disp, const MPI_Datatype *types,
                                  MPI_Datatype *t) {
    long ext = 0;
    for (int i = 0; i < n; i++) {
        long e = disp[i] + (long) len[i] * cupcfd_oracle_mpi::extent(types[i]);
        if (e > ext) ext = e;
    }
    *t = cupcfd_oracle_mpi::new_type(ext);
    return MPI_SUCCESS;
}
inline int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype *t) {
    *t = cupcfd_oracle_mpi::new_type((long) n * cupcfd_oracle_mpi::extent(old));
    return MPI_SUCCESS;
}
inline int MPI_Type_create_resized(MPI_Datatype, MPI_Aint, MPI_Aint ext, MPI_Datatype *t) {
    *t = cupcfd_oracle_mpi::new_type(ext);
    return MPI_SUCCESS;
}
inline int MPI_Type_commit(MPI_Datatype *) { return MPI_SUCCESS; }
inline int MPI_Type_free(MPI_Datatype *t) { *t = MPI_DATATYPE_NULL; return MPI_SUCCESS; }
inline int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint) p; return MPI_SUCCESS; }

inline int MPI_Initialized(int *f) { *f = 1; return MPI_SUCCESS; }
inline int MPI_Abort(MPI_Comm, int) { cupcfd_oracle_mpi::fail("MPI_Abort"); }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = cupcfd_oracle_mpi::my_rank(); return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *s) {
    std::lock_guard<std::mutex> lk(cupcfd_oracle_mpi::world().mu);
    *s = cupcfd_oracle_mpi::world().size;
    return MPI_SUCCESS;
}
inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *n) { *n = c; return MPI_SUCCESS; }
inline int MPI_Comm_free(MPI_Comm *c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
inline int MPI_Info_create(MPI_Info *i) { *i = 1; return MPI_SUCCESS; }
inline int MPI_Info_free(MPI_Info *i) { *i = MPI_INFO_NULL; return MPI_SUCCESS; }
inline int MPI_Barrier(MPI_Comm) { cupcfd_oracle_mpi::barrier(); return MPI_SUCCESS; }

inline int MPI_Comm_group(MPI_Comm, MPI_Group *g) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    std::lock_guard<std::mutex> lk(w.mu);
    std::vector<int> all((size_t) w.size);
    for (int i = 0; i < w.size; i++) all[(size_t) i] = i;
    w.groups.push_back(all);
    *g = (int) w.groups.size();
    return MPI_SUCCESS;
}
inline int MPI_Group_incl(MPI_Group, int n, const int *ranks, MPI_Group *g) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    std::lock_guard<std::mutex> lk(w.mu);
    w.groups.push_back(std::vector<int>(ranks, ranks + n));
    *g = (int) w.groups.size();
    return MPI_SUCCESS;
}
inline int MPI_Group_free(MPI_Group *g) { *g = MPI_GROUP_NULL; return MPI_SUCCESS; }

// ---- collectives
inline int MPI_Bcast(void *buf, int n, MPI_Datatype t, int root, MPI_Comm) {
    const long b = (long) n * cupcfd_oracle_mpi::extent(t);
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = buf;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        if (cupcfd_oracle_mpi::my_rank() != root) cupcfd_oracle_mpi::copy(sl[(size_t) root].s, b, buf, b);
    });
    return MPI_SUCCESS;
}
inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm) {
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        cupcfd_oracle_mpi::reduce_all(sl, r, n, t, op);
    });
    return MPI_SUCCESS;
}
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm) {
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        if (cupcfd_oracle_mpi::my_rank() == root) cupcfd_oracle_mpi::reduce_all(sl, r, n, t, op);
    });
    return MPI_SUCCESS;
}
inline int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm) {
    const long sb = (long) sn * cupcfd_oracle_mpi::extent(st), rb = (long) rn * cupcfd_oracle_mpi::extent(rt);
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        for (size_t j = 0; j < sl.size(); j++) cupcfd_oracle_mpi::copy(sl[j].s, sb, (char *) r + (long) j * rb, rb);
    });
    return MPI_SUCCESS;
}
inline int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm) {
    const long sb = (long) sn * cupcfd_oracle_mpi::extent(st), rb = (long) rn * cupcfd_oracle_mpi::extent(rt);
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        if (cupcfd_oracle_mpi::my_rank() != root) return;
        for (size_t j = 0; j < sl.size(); j++) cupcfd_oracle_mpi::copy(sl[j].s, sb, (char *) r + (long) j * rb, rb);
    });
    return MPI_SUCCESS;
}
inline int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd,
                          MPI_Datatype rt, MPI_Comm) {
    const long se = cupcfd_oracle_mpi::extent(st), re = cupcfd_oracle_mpi::extent(rt);
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    mine.n = sn;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        for (size_t j = 0; j < sl.size(); j++)
            cupcfd_oracle_mpi::copy(sl[j].s, sl[j].n * se, (char *) r + rd[j] * re, rc[j] * re);
    });
    return MPI_SUCCESS;
}
inline int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd,
                       MPI_Datatype rt, int root, MPI_Comm) {
    const long se = cupcfd_oracle_mpi::extent(st), re = cupcfd_oracle_mpi::extent(rt);
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    mine.n = sn;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        if (cupcfd_oracle_mpi::my_rank() != root) return;
        for (size_t j = 0; j < sl.size(); j++)
            cupcfd_oracle_mpi::copy(sl[j].s, sl[j].n * se, (char *) r + rd[j] * re, rc[j] * re);
    });
    return MPI_SUCCESS;
}
inline int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm) {
    const long sb = (long) sn * cupcfd_oracle_mpi::extent(st), rb = (long) rn * cupcfd_oracle_mpi::extent(rt);
    const int me = cupcfd_oracle_mpi::my_rank();
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        for (size_t j = 0; j < sl.size(); j++)
            cupcfd_oracle_mpi::copy((const char *) sl[j].s + me * sb, sb, (char *) r + (long) j * rb, rb);
    });
    return MPI_SUCCESS;
}
inline int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, const int *rc,
                         const int *rd, MPI_Datatype rt, MPI_Comm) {
    const long se = cupcfd_oracle_mpi::extent(st), re = cupcfd_oracle_mpi::extent(rt);
    const int me = cupcfd_oracle_mpi::my_rank();
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    mine.counts = sc;
    mine.displs = sd;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        for (size_t j = 0; j < sl.size(); j++)
            cupcfd_oracle_mpi::copy((const char *) sl[j].s + sl[j].displs[me] * se, sl[j].counts[me] * se,
                                    (char *) r + rd[j] * re, rc[j] * re);
    });
    return MPI_SUCCESS;
}
inline int MPI_Scatter(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm) {
    const long sb = (long) sn * cupcfd_oracle_mpi::extent(st), rb = (long) rn * cupcfd_oracle_mpi::extent(rt);
    const int me = cupcfd_oracle_mpi::my_rank();
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        cupcfd_oracle_mpi::copy((const char *) sl[(size_t) root].s + me * sb, sb, r, rb);
    });
    return MPI_SUCCESS;
}
inline int MPI_Scatterv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, int rn,
                        MPI_Datatype rt, int root, MPI_Comm) {
    const long se = cupcfd_oracle_mpi::extent(st), rb = (long) rn * cupcfd_oracle_mpi::extent(rt);
    const int me = cupcfd_oracle_mpi::my_rank();
    cupcfd_oracle_mpi::World::Slot mine;
    mine.s = s;
    mine.counts = sc;
    mine.displs = sd;
    cupcfd_oracle_mpi::collective(mine, [&](const std::vector<cupcfd_oracle_mpi::World::Slot> &sl) {
        const cupcfd_oracle_mpi::World::Slot &rs = sl[(size_t) root];
        cupcfd_oracle_mpi::copy((const char *) rs.s + rs.displs[me] * se, rs.counts[me] * se, r, rb);
    });
    return MPI_SUCCESS;
}

// ---- point to point (buffered sends; receives matched at MPI_Waitall)
inline int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm, MPI_Request *req) {
    const long bytes = (long) n * cupcfd_oracle_mpi::extent(t);
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    std::lock_guard<std::mutex> lk(w.mu);
    if (dest < 0 || dest >= w.size) cupcfd_oracle_mpi::fail("send to a rank outside the world");
    w.mail[std::make_tuple(cupcfd_oracle_mpi::my_rank(), dest, tag)].emplace_back((const char *) b, (const char *) b + bytes);
    *req = w.nextRequest++;
    w.cv.notify_all();
    return MPI_SUCCESS;
}
inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Request *req) {
    const long bytes = (long) n * cupcfd_oracle_mpi::extent(t);
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    std::lock_guard<std::mutex> lk(w.mu);
    if (src < 0 || src >= w.size) cupcfd_oracle_mpi::fail("receive from a rank outside the world");
    *req = w.nextRequest++;
    w.recvs[*req] = cupcfd_oracle_mpi::World::Recv{src, tag, b, bytes};
    return MPI_SUCCESS;
}
inline int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    const int me = cupcfd_oracle_mpi::my_rank();
    std::unique_lock<std::mutex> lk(w.mu);
    for (int k = 0; k < n; k++) {
        auto it = w.recvs.find(reqs[k]);
        if (it != w.recvs.end()) {
            const cupcfd_oracle_mpi::World::Recv rv = it->second;
            const auto key = std::make_tuple(rv.src, me, rv.tag);
            cupcfd_oracle_mpi::wait_for(lk, [&] { return !w.mail[key].empty(); }, "receive timed out");
            std::vector<char> msg = std::move(w.mail[key].front());
            w.mail[key].pop_front();
            cupcfd_oracle_mpi::copy(msg.data(), (long) msg.size(), rv.buf, rv.bytes);
            w.recvs.erase(reqs[k]);
        }
        reqs[k] = MPI_REQUEST_NULL;
    }
    return MPI_SUCCESS;
}

// ---- one-sided
inline int MPI_Win_create(void *base, MPI_Aint, int unit, MPI_Info, MPI_Comm, MPI_Win *win) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    const int me = cupcfd_oracle_mpi::my_rank();
    std::unique_lock<std::mutex> lk(w.mu);
    const int id = w.winCount[(size_t) me]++;  // collective: every rank creates its windows in the same order
    if ((int) w.wins.size() <= id) {
        cupcfd_oracle_mpi::World::Win nw;
        const size_t P = (size_t) w.size;
        nw.base.assign(P, nullptr);
        nw.unit.assign(P, 0);
        nw.posted.assign(P, 0);
        nw.completed.assign(P, 0);
        nw.started.assign(P, std::vector<long>(P, 0));
        nw.postGroup.assign(P, 0);
        nw.startGroup.assign(P, 0);
        w.wins.push_back(nw);
    }
    w.wins[(size_t) id].base[(size_t) me] = (char *) base;
    w.wins[(size_t) id].unit[(size_t) me] = unit;
    *win = id + 1;
    cupcfd_oracle_mpi::barrier_locked(lk);
    return MPI_SUCCESS;
}
inline int MPI_Win_free(MPI_Win *win) {
    cupcfd_oracle_mpi::barrier();
    *win = MPI_WIN_NULL;
    return MPI_SUCCESS;
}
inline int MPI_Win_fence(int, MPI_Win) {
    cupcfd_oracle_mpi::barrier();
    return MPI_SUCCESS;
}
inline int MPI_Put(const void *o, int on, MPI_Datatype ot, int rank, MPI_Aint disp, int tn, MPI_Datatype tt, MPI_Win win) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    char *dst;
    {
        std::lock_guard<std::mutex> lk(w.mu);
        if (win < 1 || win > (int) w.wins.size() || rank < 0 || rank >= w.size) cupcfd_oracle_mpi::fail("bad put");
        const cupcfd_oracle_mpi::World::Win &wn = w.wins[(size_t) win - 1];
        dst = wn.base[(size_t) rank] + disp * wn.unit[(size_t) rank];
    }
    const long ob = (long) on * cupcfd_oracle_mpi::extent(ot), tb = (long) tn * cupcfd_oracle_mpi::extent(tt);
    cupcfd_oracle_mpi::copy(o, ob, dst, tb);
    return MPI_SUCCESS;
}
// active-target epochs: a target posts to its origins, an origin starts once
// every target of its group has posted, completes by counting itself in at
// each target, and a target's wait ends when all its origins have completed
inline int MPI_Win_post(MPI_Group g, int, MPI_Win win) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    const int me = cupcfd_oracle_mpi::my_rank();
    std::lock_guard<std::mutex> lk(w.mu);
    cupcfd_oracle_mpi::World::Win &wn = w.wins[(size_t) win - 1];
    wn.postGroup[(size_t) me] = g;
    wn.posted[(size_t) me]++;
    w.cv.notify_all();
    return MPI_SUCCESS;
}
inline int MPI_Win_start(MPI_Group g, int, MPI_Win win) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    const int me = cupcfd_oracle_mpi::my_rank();
    std::unique_lock<std::mutex> lk(w.mu);
    cupcfd_oracle_mpi::World::Win &wn = w.wins[(size_t) win - 1];
    wn.startGroup[(size_t) me] = g;
    const std::vector<int> targets = g > 0 ? w.groups[(size_t) g - 1] : std::vector<int>();
    for (int t : targets) {
        const long epoch = ++wn.started[(size_t) me][(size_t) t];
        cupcfd_oracle_mpi::wait_for(lk, [&] { return w.wins[(size_t) win - 1].posted[(size_t) t] >= epoch; },
                                    "start timed out waiting for a post");
    }
    return MPI_SUCCESS;
}
inline int MPI_Win_complete(MPI_Win win) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    const int me = cupcfd_oracle_mpi::my_rank();
    std::lock_guard<std::mutex> lk(w.mu);
    cupcfd_oracle_mpi::World::Win &wn = w.wins[(size_t) win - 1];
    const int g = wn.startGroup[(size_t) me];
    if (g > 0)
        for (int t : w.groups[(size_t) g - 1]) wn.completed[(size_t) t]++;
    w.cv.notify_all();
    return MPI_SUCCESS;
}
inline int MPI_Win_wait(MPI_Win win) {
    cupcfd_oracle_mpi::World &w = cupcfd_oracle_mpi::world();
    const int me = cupcfd_oracle_mpi::my_rank();
    std::unique_lock<std::mutex> lk(w.mu);
    cupcfd_oracle_mpi::World::Win &wn = w.wins[(size_t) win - 1];
    const int g = wn.postGroup[(size_t) me];
    const long need = g > 0 ? (long) w.groups[(size_t) g - 1].size() : 0;
    cupcfd_oracle_mpi::wait_for(lk, [&] { return w.wins[(size_t) win - 1].completed[(size_t) me] >= need; },
                                "wait timed out for the origins' completes");
    w.wins[(size_t) win - 1].completed[(size_t) me] -= need;
    return MPI_SUCCESS;
}
#endif  /* __cplusplus */

#endif
