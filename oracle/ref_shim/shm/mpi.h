/*
 * Multi-process MPI subset over process-shared memory (TEST / BASELINE
 * INFRASTRUCTURE ONLY: used to run the reference solver's own CPU path as N
 * ranks on one host, where no MPI library exists; never linked into the
 * product).
 *
 * It implements exactly the calls the reference makes (src/solver.h:543-587,
 * 1000-1031; src/cfd.h:253-301 and its four copies; src/eq.h:47-91,
 * 190-235, 569, 682, 781; src/mv.h:27, 51, 96-136, 223-263; src/alm.h:
 * 280-412; src/cfd.h:1137) with MPI's semantics for the way the reference
 * uses them:
 *
 *   - point-to-point messages only between neighbouring ranks (the x-slab
 *     halo exchange): one mailbox per ordered pair (src, src +- 1).  Isend
 *     waits until the mailbox is empty, copies the message in and returns
 *     completed (eager send); Irecv records the request and Wait copies the
 *     message out and empties the mailbox.  Each exchange posts one message
 *     per neighbour and waits for all of them before the next, so a single
 *     slot per pair keeps MPI's per-pair FIFO order and cannot deadlock: a
 *     sender blocked on a full slot waits only for a receiver that is
 *     already inside the Wait of the previous exchange.
 *   - Allreduce / Iallreduce (SUM, MAX; double, int, long; up to 8 values):
 *     every rank writes its values into its slot of one of two alternating
 *     buffers, all meet at a barrier, and every rank reduces the slots in
 *     rank order (so every rank gets the same, deterministic result).  Two
 *     buffers suffice: a rank can only write the same buffer again after the
 *     next barrier, which every rank reaches only after reading this one.
 *     Iallreduce completes at the call (all ranks post them in one order).
 *   - Barrier: a sense-reversing counter barrier.
 *
 * Waits spin on atomics and yield the core after a while; each gives up
 * after DALM_SHM_WAIT_LIMIT seconds (default 1800) and aborts the process,
 * so a rank that died cannot leave the others spinning for ever (the
 * launcher then stops the job).
 *
 * The launcher creates the shared region with shm_world_create() before it
 * forks the ranks and sets each child's rank with shm_world_join().
 */
#pragma once

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <new>

#include <sched.h>
#include <sys/mman.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int dummy; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_INT 1
#define MPI_LONG 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_UNSIGNED_CHAR 5
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_REQUEST_NULL 0

namespace shm_mpi {

constexpr int MAX_RANKS = 256;
constexpr int MAX_RED = 8;
constexpr int MAX_PENDING = 64;

struct alignas(64) Mailbox {
    std::atomic<int> full;
    int tag;
    size_t bytes;
    char *data;  // inside the shared region
};

struct alignas(64) World {
    int size;
    size_t capacity;  // bytes per mailbox
    alignas(64) std::atomic<int> bar_count;
    alignas(64) std::atomic<int> bar_sense;
    alignas(64) unsigned char red[2][MAX_RANKS][MAX_RED * 8];
    Mailbox box[MAX_RANKS][2];  // [src][0: to src-1, 1: to src+1]
};

struct Pending {
    void *buf;
    size_t bytes;
    int source, tag, used;
};

static World *g_world = nullptr;
static int g_rank = 0;
static int g_sense = 0;
static unsigned g_red_gen = 0;
static Pending g_pending[MAX_PENDING];

inline double limit_seconds() {
    const char *e = std::getenv("DALM_SHM_WAIT_LIMIT");
    double v = e ? std::atof(e) : 0.0;
    return v > 0 ? v : 1800.0;
}

inline double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

// Spins until pred() holds; aborts after the wait limit.
template <typename Pred>
inline void wait_until(Pred pred, const char *what) {
    unsigned long n = 0;
    double t0 = -1;
    while (!pred()) {
        if (++n > 2000) sched_yield();
        if ((n & 0xffff) == 0) {
            double t = now_s();
            if (t0 < 0) t0 = t;
            else if (t - t0 > limit_seconds()) {
                std::fprintf(stderr, "[shm-mpi] rank %d: %s did not complete in %.0f s\n", g_rank,
                             what, limit_seconds());
                std::abort();
            }
        }
    }
}

inline size_t type_size(MPI_Datatype t) {
    switch (t) {
    case MPI_INT: return sizeof(int);
    case MPI_LONG: return sizeof(long);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_UNSIGNED_CHAR: return 1;
    default: std::fprintf(stderr, "[shm-mpi] unsupported datatype %d\n", t); std::abort();
    }
}

inline Mailbox &box(int src, int dst) {
    if (dst != src - 1 && dst != src + 1) {
        std::fprintf(stderr, "[shm-mpi] message %d -> %d: only neighbours are supported\n", src, dst);
        std::abort();
    }
    return g_world->box[src][dst == src + 1 ? 1 : 0];
}

// One region for the world and every mailbox, mapped shared before fork.
inline World *create(int size, size_t capacity) {
    if (size < 1 || size > MAX_RANKS) return nullptr;
    capacity = (capacity + 63) & ~(size_t)63;
    size_t head = (sizeof(World) + 63) & ~(size_t)63;
    size_t total = head + (size_t)size * 2 * capacity;
    void *p = mmap(nullptr, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE,
                   -1, 0);
    if (p == MAP_FAILED) return nullptr;
    World *w = new (p) World();
    w->size = size;
    w->capacity = capacity;
    w->bar_count.store(0);
    w->bar_sense.store(0);
    char *data = (char *)p + head;
    for (int r = 0; r < size; r++)
        for (int d = 0; d < 2; d++) {
            Mailbox &b = w->box[r][d];
            b.full.store(0);
            b.tag = -1;
            b.bytes = 0;
            b.data = data + ((size_t)r * 2 + d) * capacity;
        }
    return w;
}

inline void join(World *w, int rank) {
    g_world = w;
    g_rank = rank;
    g_sense = 0;
    g_red_gen = 0;
    std::memset(g_pending, 0, sizeof g_pending);
}

inline void barrier() {
    World *w = g_world;
    g_sense ^= 1;
    const int sense = g_sense;
    if (w->bar_count.fetch_add(1, std::memory_order_acq_rel) == w->size - 1) {
        w->bar_count.store(0, std::memory_order_relaxed);
        w->bar_sense.store(sense, std::memory_order_release);
    } else {
        wait_until([&] { return w->bar_sense.load(std::memory_order_acquire) == sense; }, "barrier");
    }
}

template <typename T>
inline void reduce_as(unsigned char (*slots)[MAX_RED * 8], int n, int count, MPI_Op op, void *out) {
    T acc[MAX_RED];
    std::memcpy(acc, slots[0], count * sizeof(T));
    for (int r = 1; r < n; r++) {
        T v[MAX_RED];
        std::memcpy(v, slots[r], count * sizeof(T));
        for (int m = 0; m < count; m++) acc[m] = (op == MPI_MAX) ? (v[m] > acc[m] ? v[m] : acc[m]) : acc[m] + v[m];
    }
    std::memcpy(out, acc, count * sizeof(T));
}

inline int allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op) {
    if (count > MAX_RED || (op != MPI_SUM && op != MPI_MAX)) {
        std::fprintf(stderr, "[shm-mpi] allreduce of %d values / op %d unsupported\n", count, op);
        std::abort();
    }
    const size_t ts = type_size(t);
    unsigned char (*slots)[MAX_RED * 8] = g_world->red[g_red_gen++ & 1u];
    std::memcpy(slots[g_rank], send == MPI_IN_PLACE ? recv : send, count * ts);
    barrier();
    switch (t) {
    case MPI_DOUBLE: reduce_as<double>(slots, g_world->size, count, op, recv); break;
    case MPI_FLOAT: reduce_as<float>(slots, g_world->size, count, op, recv); break;
    case MPI_INT: reduce_as<int>(slots, g_world->size, count, op, recv); break;
    case MPI_LONG: reduce_as<long>(slots, g_world->size, count, op, recv); break;
    default: std::abort();
    }
    return 0;
}

}  // namespace shm_mpi

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_size(MPI_Comm, int *s) {
    *s = shm_mpi::g_world ? shm_mpi::g_world->size : 1;
    return 0;
}
inline int MPI_Comm_rank(MPI_Comm, int *r) {
    *r = shm_mpi::g_rank;
    return 0;
}
inline int MPI_Barrier(MPI_Comm) {
    if (shm_mpi::g_world) shm_mpi::barrier();
    return 0;
}
inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm,
                     MPI_Request *req) {
    using namespace shm_mpi;
    size_t bytes = (size_t)count * type_size(t);
    Mailbox &b = box(g_rank, dest);
    if (bytes > g_world->capacity) {
        std::fprintf(stderr, "[shm-mpi] message of %zu bytes > mailbox %zu\n", bytes, g_world->capacity);
        std::abort();
    }
    wait_until([&] { return b.full.load(std::memory_order_acquire) == 0; }, "send");
    std::memcpy(b.data, buf, bytes);
    b.bytes = bytes;
    b.tag = tag;
    b.full.store(1, std::memory_order_release);
    *req = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm,
                     MPI_Request *req) {
    using namespace shm_mpi;
    for (int n = 0; n < MAX_PENDING; n++) {
        if (!g_pending[n].used) {
            g_pending[n] = Pending{buf, (size_t)count * type_size(t), source, tag, 1};
            *req = n + 1;
            return 0;
        }
    }
    std::fprintf(stderr, "[shm-mpi] too many pending receives\n");
    std::abort();
}
inline int MPI_Wait(MPI_Request *req, MPI_Status *) {
    using namespace shm_mpi;
    if (*req == MPI_REQUEST_NULL) return 0;
    Pending &p = g_pending[*req - 1];
    Mailbox &b = box(p.source, g_rank);
    wait_until([&] { return b.full.load(std::memory_order_acquire) == 1; }, "receive");
    if (b.tag != p.tag || b.bytes != p.bytes) {
        std::fprintf(stderr, "[shm-mpi] rank %d: message from %d has tag %d / %zu bytes, expected %d / %zu\n",
                     g_rank, p.source, b.tag, b.bytes, p.tag, p.bytes);
        std::abort();
    }
    std::memcpy(p.buf, b.data, p.bytes);
    b.full.store(0, std::memory_order_release);
    p.used = 0;
    *req = MPI_REQUEST_NULL;
    return 0;
}
inline int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *) {
    for (int i = 0; i < n; i++) MPI_Wait(&reqs[i], MPI_STATUS_IGNORE);
    return 0;
}
inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm) {
    if (!shm_mpi::g_world || shm_mpi::g_world->size == 1) {
        if (send != MPI_IN_PLACE) std::memcpy(recv, send, (size_t)count * shm_mpi::type_size(t));
        return 0;
    }
    return shm_mpi::allreduce(send, recv, count, t, op);
}
inline int MPI_Iallreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op op,
                          MPI_Comm c, MPI_Request *req) {
    *req = MPI_REQUEST_NULL;
    return MPI_Allreduce(send, recv, count, t, op, c);
}
