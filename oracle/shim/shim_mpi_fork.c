/*
 * Multi-process MPI stand-in (the subset declared in mpi.h) used ONLY to run the reference solver's
 * own domain decomposition on all host cores as the CPU baseline (oracle/ref_mpi_run.c). Test and
 * baseline infrastructure, never product code; no MPI library exists in this image.
 *
 * MPI_Init forks the process into TEAL_SHIM_RANKS ranks (default 1) that share one anonymous shared
 * mapping. Every rank owns an inbox ring in it. A send copies the message into the destination's
 * ring right away (eager, so MPI_Isend completes at once); a rank that waits for anything first
 * moves the finished messages of its own ring into a private queue (so a ring never stays full
 * while its owner waits), then matches receives there by (source, tag, communicator) in arrival
 * order, which keeps MPI's order between two ranks. Collectives are built from these messages on
 * an internal channel; reductions combine the contributions in rank order, so every rank gets the
 * same bits. All communicators span all ranks; Cartesian topologies number ranks row-major as MPI
 * does. A rank that fails or waits longer than TEAL_SHIM_TIMEOUT seconds (default 900) raises a
 * shared abort flag that ends every rank; children die with their parent (PR_SET_PDEATHSIG).
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/types.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

enum { MAX_RANKS = 1024, MAX_COMMS = 64, INTERNAL = 1 << 20 };
enum { ST_WRITING = 1, ST_READY = 2, ST_CONSUMED = 3, ST_PAD = 4 };

typedef struct {
    uint32_t state;
    int src;
    int tag;
    int comm;
    uint64_t bytes;
    uint64_t len; /* block length in the ring, header included, a multiple of 64 */
    uint64_t pad_;
} Block;

typedef struct {
    int lock;
    uint64_t head; /* consumer position (monotonic bytes) */
    uint64_t tail; /* producer position (monotonic bytes) */
    char pad_[64 - sizeof(int) - 2 * sizeof(uint64_t)];
} Ring;

typedef struct {
    int size;
    int abort;
    int barrier_count;
    int barrier_gen;
    uint64_t ring_bytes;
    char pad_[40];
    Ring rings[];
} Shared;

static Shared *shm = 0;
static size_t shm_bytes = 0;
static char *ring_data = 0;
static int my_rank = 0, world = 1, initialized = 0;
static pid_t children[MAX_RANKS];
static double timeout_s = 900.0;

static int type_bytes(MPI_Datatype type)
{
    return type & ((1 << 20) - 1);
}

static int type_kind(MPI_Datatype type)
{
    return type >> 20;
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + (1e-9 * (double)ts.tv_nsec);
}

static void fail(const char *what)
{
    fprintf(stderr, "mpi shim (rank %d): %s\n", my_rank, what);
    fflush(stderr);
    if (shm) {
        __atomic_store_n(&shm->abort, 1, __ATOMIC_RELEASE);
    }
    _exit(1);
}

/* one round of a wait loop: abort checks, a deadline, a short pause after the first spins */
typedef struct {
    double start;
    long spins;
} Waiter;

static void wait_step(Waiter *w)
{
    if (__atomic_load_n(&shm->abort, __ATOMIC_ACQUIRE)) {
        _exit(1);
    }
    if (my_rank == 0 && (w->spins & 1023) == 0) {
        int status;
        pid_t p = waitpid(-1, &status, WNOHANG);
        if (p > 0 && !(WIFEXITED(status) && WEXITSTATUS(status) == 0)) {
            fail("a rank ended abnormally");
        }
        if (p > 0) {
            for (int r = 1; r < world; r++) {
                if (children[r] == p) {
                    children[r] = 0; /* reaped early: it finished its part */
                }
            }
        }
    }
    if (w->spins == 0) {
        w->start = MPI_Wtime();
    }
    w->spins++;
    if (w->spins > 64) {
        if ((w->spins & 255) == 0 && MPI_Wtime() - w->start > timeout_s) {
            fail("wait timed out");
        }
        struct timespec ts = {0, w->spins > 4096 ? 20000 : 1000};
        nanosleep(&ts, 0);
    }
}

/* ---- environment ---------------------------------------------------------------------------- */

int MPI_Init(int *argc, char ***argv)
{
    (void)argc;
    (void)argv;
    const char *env = getenv("TEAL_SHIM_RANKS");
    world = env ? atoi(env) : 1;
    if (world < 1 || world > MAX_RANKS) {
        fail("TEAL_SHIM_RANKS out of range");
    }
    const char *t = getenv("TEAL_SHIM_TIMEOUT");
    if (t) {
        timeout_s = atof(t);
    }
    const char *mb = getenv("TEAL_SHIM_RING_MB");
    uint64_t ring = (uint64_t)(mb ? atol(mb) : 64) << 20;
    shm_bytes = sizeof(Shared) + world * sizeof(Ring) + world * ring;
    void *p = mmap(0, shm_bytes, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) {
        fail("shared mapping failed");
    }
    shm = p;
    shm->size = world;
    shm->ring_bytes = ring;
    ring_data = (char *)p + sizeof(Shared) + world * sizeof(Ring);
    fflush(0);
    pid_t parent = getpid();
    for (int r = 1; r < world; r++) {
        pid_t c = fork();
        if (c < 0) {
            fail("fork failed");
        }
        if (c == 0) {
            prctl(PR_SET_PDEATHSIG, SIGKILL);
            if (getppid() != parent) {
                _exit(1);
            }
            my_rank = r;
            break;
        }
        children[r] = c;
    }
    initialized = 1;
    return MPI_SUCCESS;
}

int MPI_Initialized(int *flag)
{
    *flag = initialized;
    return MPI_SUCCESS;
}

static void barrier(void)
{
    int gen = __atomic_load_n(&shm->barrier_gen, __ATOMIC_ACQUIRE);
    if (__atomic_add_fetch(&shm->barrier_count, 1, __ATOMIC_ACQ_REL) == world) {
        __atomic_store_n(&shm->barrier_count, 0, __ATOMIC_RELAXED);
        __atomic_store_n(&shm->barrier_gen, gen + 1, __ATOMIC_RELEASE);
        return;
    }
    Waiter w = {0, 0};
    while (__atomic_load_n(&shm->barrier_gen, __ATOMIC_ACQUIRE) == gen) {
        wait_step(&w);
    }
}

int MPI_Finalize(void)
{
    barrier();
    fflush(0);
    if (my_rank != 0) {
        _exit(0);
    }
    int bad = 0;
    for (int r = 1; r < world; r++) {
        int status;
        if (children[r] > 0 && waitpid(children[r], &status, 0) == children[r]) {
            bad |= !(WIFEXITED(status) && WEXITSTATUS(status) == 0);
        }
    }
    munmap(shm, shm_bytes);
    shm = 0;
    initialized = 0;
    if (bad) {
        fprintf(stderr, "mpi shim: a rank ended abnormally\n");
        exit(1);
    }
    return MPI_SUCCESS;
}

/* communicators: ids handed out in call order, the same on every rank */
typedef struct {
    int ndims;
    int dims[3];
    int periods[3];
} Topology;

static Topology topo[MAX_COMMS];
static int next_comm = 2; /* MPI_COMM_WORLD is 1 */

int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm)
{
    if (next_comm >= MAX_COMMS) {
        fail("too many communicators");
    }
    topo[next_comm] = topo[comm];
    *newcomm = next_comm++;
    return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm *comm)
{
    *comm = MPI_COMM_NULL;
    return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
    (void)comm;
    *rank = my_rank;
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
    (void)comm;
    *size = world;
    return MPI_SUCCESS;
}

/* ---- datatypes: a datatype is its byte size (plus a kind tag) -------------------------------- */

int MPI_Type_size(MPI_Datatype type, int *size)
{
    *size = type_bytes(type);
    return MPI_SUCCESS;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *type)
{
    *type = (7 << 20) | (count * type_bytes(old));
    return MPI_SUCCESS;
}

int MPI_Type_create_resized(MPI_Datatype old, MPI_Aint lb, MPI_Aint extent, MPI_Datatype *type)
{
    (void)old;
    (void)lb;
    *type = (8 << 20) | (int)extent;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *type)
{
    (void)type;
    return MPI_SUCCESS;
}

int MPI_Type_free(MPI_Datatype *type)
{
    (void)type;
    return MPI_SUCCESS;
}

/* ---- messages ------------------------------------------------------------------------------- */

static void ring_lock(Ring *r)
{
    Waiter w = {0, 0};
    while (__atomic_exchange_n(&r->lock, 1, __ATOMIC_ACQUIRE)) {
        wait_step(&w);
    }
}

static void ring_unlock(Ring *r)
{
    __atomic_store_n(&r->lock, 0, __ATOMIC_RELEASE);
}

typedef struct Message {
    int src, tag, comm;
    size_t bytes;
    struct Message *next;
    char data[];
} Message;

static Message *inbox_head = 0, *inbox_tail = 0;

/* move the finished messages of this rank's ring into the private queue, in ring order */
static void drain(void)
{
    Ring *r = &shm->rings[my_rank];
    char *base = ring_data + (size_t)my_rank * shm->ring_bytes;
    uint64_t cap = shm->ring_bytes;
    uint64_t head = __atomic_load_n(&r->head, __ATOMIC_ACQUIRE);
    uint64_t tail = __atomic_load_n(&r->tail, __ATOMIC_ACQUIRE);
    for (uint64_t pos = head; pos < tail;) {
        Block *b = (Block *)(base + (pos % cap));
        uint32_t st = __atomic_load_n(&b->state, __ATOMIC_ACQUIRE);
        if (st == ST_READY) {
            Message *m = malloc(sizeof(*m) + (b->bytes ? b->bytes : 1));
            if (!m) {
                fail("out of memory");
            }
            m->src = b->src, m->tag = b->tag, m->comm = b->comm, m->bytes = b->bytes, m->next = 0;
            memcpy(m->data, (char *)b + sizeof(Block), b->bytes);
            if (inbox_tail) {
                inbox_tail->next = m;
            }
            else {
                inbox_head = m;
            }
            inbox_tail = m;
            __atomic_store_n(&b->state, ST_CONSUMED, __ATOMIC_RELEASE);
        }
        pos += b->len;
    }
    /* release the leading finished blocks */
    while (head < tail) {
        Block *b = (Block *)(base + (head % cap));
        uint32_t st = __atomic_load_n(&b->state, __ATOMIC_ACQUIRE);
        if (st != ST_CONSUMED && st != ST_PAD) {
            break;
        }
        head += b->len;
    }
    __atomic_store_n(&r->head, head, __ATOMIC_RELEASE);
}

static void post(int dest, int tag, int comm, const void *buf, size_t bytes)
{
    if (dest < 0 || dest >= world) {
        fail("send to an invalid rank");
    }
    Ring *r = &shm->rings[dest];
    char *base = ring_data + (size_t)dest * shm->ring_bytes;
    uint64_t cap = shm->ring_bytes;
    uint64_t need = (sizeof(Block) + bytes + 63) & ~(uint64_t)63;
    if (need > cap / 2) {
        fail("message larger than half an inbox ring (raise TEAL_SHIM_RING_MB)");
    }
    Block *b = 0;
    Waiter w = {0, 0};
    for (;;) {
        ring_lock(r);
        uint64_t head = __atomic_load_n(&r->head, __ATOMIC_ACQUIRE);
        uint64_t tail = r->tail;
        uint64_t room = cap - (tail % cap); /* bytes up to the end of the ring */
        uint64_t total = need + (room < need ? room : 0);
        if (tail + total - head <= cap) {
            if (room < need) { /* pad to the end and wrap */
                Block *p = (Block *)(base + (tail % cap));
                p->len = room;
                p->state = ST_PAD;
                tail += room;
            }
            b = (Block *)(base + (tail % cap));
            b->state = ST_WRITING;
            b->src = my_rank, b->tag = tag, b->comm = comm, b->bytes = bytes, b->len = need;
            __atomic_store_n(&r->tail, tail + need, __ATOMIC_RELEASE);
            ring_unlock(r);
            break;
        }
        ring_unlock(r);
        drain(); /* free this rank's own ring while it waits for room in another */
        wait_step(&w);
    }
    if (bytes) {
        memcpy((char *)b + sizeof(Block), buf, bytes);
    }
    __atomic_store_n(&b->state, ST_READY, __ATOMIC_RELEASE);
}

/* the first queued message from `src` with `tag` on `comm`, unlinked, or 0 */
static Message *take(int src, int tag, int comm)
{
    for (Message **p = &inbox_head, *prev = 0; *p; prev = *p, p = &(*p)->next) {
        Message *m = *p;
        if (m->src == src && m->tag == tag && m->comm == comm) {
            *p = m->next;
            if (inbox_tail == m) {
                inbox_tail = prev;
            }
            return m;
        }
    }
    return 0;
}

/* a matching message copied into buf if one has arrived; returns 1 when done */
static int try_receive(int src, int tag, int comm, void *buf, size_t cap_bytes)
{
    Message *m = take(src, tag, comm);
    if (!m) {
        drain();
        m = take(src, tag, comm);
    }
    if (!m) {
        return 0;
    }
    if (m->bytes > cap_bytes) {
        fail("message truncated");
    }
    memcpy(buf, m->data, m->bytes);
    free(m);
    return 1;
}

static void receive(int src, int tag, int comm, void *buf, size_t cap_bytes)
{
    Waiter w = {0, 0};
    while (!try_receive(src, tag, comm, buf, cap_bytes)) {
        wait_step(&w);
    }
}

/* ---- point to point ------------------------------------------------------------------------- */

struct shim_request {
    int pending; /* a receive not yet matched */
    int src, tag, comm;
    void *buf;
    size_t bytes;
};

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request *req)
{
    struct shim_request *r = calloc(1, sizeof(*r));
    *req = r;
    if (dest != MPI_PROC_NULL) {
        post(dest, tag, comm, buf, (size_t)count * type_bytes(type)); /* eager: done on return */
    }
    return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
              MPI_Request *req)
{
    struct shim_request *r = calloc(1, sizeof(*r));
    *req = r;
    if (source != MPI_PROC_NULL) {
        if (source < 0 || source >= world) {
            fail("receive from an invalid rank");
        }
        r->pending = 1;
        r->src = source, r->tag = tag, r->comm = comm, r->buf = buf;
        r->bytes = (size_t)count * type_bytes(type);
        if (try_receive(r->src, r->tag, r->comm, r->buf, r->bytes)) {
            r->pending = 0;
        }
    }
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
    (void)statuses;
    Waiter w = {0, 0};
    for (;;) {
        int left = 0;
        for (int i = 0; i < count; i++) {
            struct shim_request *r = reqs[i];
            if (r && r->pending) {
                if (try_receive(r->src, r->tag, r->comm, r->buf, r->bytes)) {
                    r->pending = 0;
                }
                else {
                    left++;
                }
            }
        }
        if (!left) {
            break;
        }
        wait_step(&w);
    }
    for (int i = 0; i < count; i++) {
        free(reqs[i]);
        reqs[i] = 0;
    }
    return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
    if (dest != MPI_PROC_NULL) {
        post(dest, tag, comm, buf, (size_t)count * type_bytes(type));
    }
    return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status *status)
{
    (void)status;
    if (source != MPI_PROC_NULL) {
        receive(source, tag, comm, buf, (size_t)count * type_bytes(type));
    }
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag, void *rbuf,
                 int rcount, MPI_Datatype rtype, int source, int rtag, MPI_Comm comm,
                 MPI_Status *status)
{
    MPI_Send(sbuf, scount, stype, dest, stag, comm);
    return MPI_Recv(rbuf, rcount, rtype, source, rtag, comm, status);
}

int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype type, int dest, int stag, int source,
                         int rtag, MPI_Comm comm, MPI_Status *status)
{
    /* the send copies the buffer out before the receive overwrites it */
    MPI_Send(buf, count, type, dest, stag, comm);
    return MPI_Recv(buf, count, type, source, rtag, comm, status);
}

/* ---- collectives, on an internal channel of each communicator ------------------------------- */

enum { T_GATHER = 1, T_ALLTOALL = 2, T_BCAST = 3 };

/* every rank's `bytes` from `mine` into all[rank * bytes] on every rank */
static void all_gather_bytes(const void *mine, void *all, size_t bytes, MPI_Comm comm)
{
    int ch = comm + INTERNAL;
    for (int r = 0; r < world; r++) {
        if (r != my_rank) {
            post(r, T_GATHER, ch, mine, bytes);
        }
    }
    memmove((char *)all + (size_t)my_rank * bytes, mine, bytes);
    for (int r = 0; r < world; r++) {
        if (r != my_rank) {
            receive(r, T_GATHER, ch, (char *)all + (size_t)r * bytes, bytes);
        }
    }
}

#define REDUCE_AS(T)                                                                                   do {                                                                                                   T *a = (T *)acc;                                                                                   const T *b = (const T *)in;                                                                        for (int i = 0; i < count; i++) {                                                                      if (op == MPI_SUM)                                                                                     a[i] = a[i] + b[i];                                                                            else if (op == MPI_MIN)                                                                                a[i] = b[i] < a[i] ? b[i] : a[i];                                                              else                                                                                                   a[i] = b[i] > a[i] ? b[i] : a[i];                                                          }                                                                                              } while (0)

static void reduce_into(void *acc, const void *in, int count, MPI_Datatype type, MPI_Op op)
{
    switch (type_kind(type)) {
        case 1: REDUCE_AS(char); break;
        case 2: REDUCE_AS(int); break;
        case 3: REDUCE_AS(unsigned); break;
        case 4: REDUCE_AS(long); break;
        case 5: REDUCE_AS(float); break;
        case 6: REDUCE_AS(double); break;
        default: fail("reduction of a derived datatype");
    }
}

/* contributions of all ranks, [world][bytes] (freed by the caller) */
static char *gather_all(const void *mine, size_t bytes, MPI_Comm comm)
{
    char *all = malloc(world * bytes + 1);
    if (!all) {
        fail("out of memory");
    }
    all_gather_bytes(mine, all, bytes, comm);
    return all;
}

int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
    size_t bytes = (size_t)count * type_bytes(type);
    char *all = gather_all(send == MPI_IN_PLACE ? recv : send, bytes, comm);
    memcpy(recv, all, bytes);
    for (int r = 1; r < world; r++) {
        reduce_into(recv, all + r * bytes, count, type, op);
    }
    free(all);
    return MPI_SUCCESS;
}

int MPI_Exscan(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op,
               MPI_Comm comm)
{
    /* rank 0's result is undefined by the standard (left as it is); rank r combines ranks < r */
    size_t bytes = (size_t)count * type_bytes(type);
    char *all = gather_all(send == MPI_IN_PLACE ? recv : send, bytes, comm);
    if (my_rank > 0) {
        memcpy(recv, all, bytes);
        for (int r = 1; r < my_rank; r++) {
            reduce_into(recv, all + r * bytes, count, type, op);
        }
    }
    free(all);
    return MPI_SUCCESS;
}

int MPI_Scan(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    size_t bytes = (size_t)count * type_bytes(type);
    char *all = gather_all(send == MPI_IN_PLACE ? recv : send, bytes, comm);
    memcpy(recv, all, bytes);
    for (int r = 1; r <= my_rank; r++) {
        reduce_into(recv, all + r * bytes, count, type, op);
    }
    free(all);
    return MPI_SUCCESS;
}

int MPI_Allgather(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm)
{
    size_t bytes = (size_t)rcount * type_bytes(rtype);
    const void *mine = (char *)recv + (size_t)my_rank * bytes;
    if (send != MPI_IN_PLACE) {
        if ((size_t)scount * type_bytes(stype) != bytes) {
            fail("allgather with different send and receive sizes");
        }
        mine = send;
    }
    all_gather_bytes(mine, recv, bytes, comm);
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *send, const int *scounts, const int *sdispls, MPI_Datatype stype,
                  void *recv, const int *rcounts, const int *rdispls, MPI_Datatype rtype,
                  MPI_Comm comm)
{
    int ch = comm + INTERNAL;
    size_t sb = type_bytes(stype), rb = type_bytes(rtype);
    for (int r = 0; r < world; r++) {
        if (r != my_rank) {
            post(r, T_ALLTOALL, ch, (const char *)send + sdispls[r] * sb, scounts[r] * sb);
        }
    }
    if (scounts[my_rank]) {
        memmove((char *)recv + rdispls[my_rank] * rb, (const char *)send + sdispls[my_rank] * sb,
                scounts[my_rank] * sb);
    }
    for (int r = 0; r < world; r++) {
        if (r != my_rank) {
            receive(r, T_ALLTOALL, ch, (char *)recv + rdispls[r] * rb, rcounts[r] * rb);
        }
    }
    return MPI_SUCCESS;
}

int MPI_Alltoall(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
                 MPI_Datatype rtype, MPI_Comm comm)
{
    int *sc = malloc(4 * world * sizeof(int));
    int *sd = sc + world, *rc = sc + 2 * world, *rd = sc + 3 * world;
    for (int r = 0; r < world; r++) {
        sc[r] = scount, sd[r] = r * scount, rc[r] = rcount, rd[r] = r * rcount;
    }
    MPI_Alltoallv(send, sc, sd, stype, recv, rc, rd, rtype, comm);
    free(sc);
    return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    int ch = comm + INTERNAL;
    size_t bytes = (size_t)count * type_bytes(type);
    if (my_rank == root) {
        for (int r = 0; r < world; r++) {
            if (r != root) {
                post(r, T_BCAST, ch, buf, bytes);
            }
        }
    }
    else {
        receive(root, T_BCAST, ch, buf, bytes);
    }
    return MPI_SUCCESS;
}

/* ---- Cartesian topology, ranks row-major (the last dimension fastest) ----------------------- */

int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder,
                    MPI_Comm *comm)
{
    (void)reorder;
    if (ndims < 0 || ndims > 3) {
        fail("Cartesian topology of more than 3 dimensions");
    }
    int prod = 1;
    for (int i = 0; i < ndims; i++) {
        prod *= dims[i];
    }
    if (prod != world) {
        fail("Cartesian grid size differs from the number of ranks");
    }
    MPI_Comm_dup(old, comm);
    Topology *t = &topo[*comm];
    t->ndims = ndims;
    for (int i = 0; i < ndims; i++) {
        t->dims[i] = dims[i];
        t->periods[i] = periods[i];
    }
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords)
{
    const Topology *t = &topo[comm];
    for (int i = t->ndims - 1; i >= 0; i--) {
        if (i < maxdims) {
            coords[i] = rank % t->dims[i];
        }
        rank /= t->dims[i];
    }
    return MPI_SUCCESS;
}

static int cart_rank(const Topology *t, const int *coords)
{
    int rank = 0;
    for (int i = 0; i < t->ndims; i++) {
        rank = rank * t->dims[i] + coords[i];
    }
    return rank;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *source, int *dest)
{
    const Topology *t = &topo[comm];
    if (direction < 0 || direction >= t->ndims) {
        fail("invalid Cartesian shift direction");
    }
    int c[3] = {0, 0, 0};
    MPI_Cart_coords(comm, my_rank, 3, c);
    int out[2];
    for (int s = 0; s < 2; s++) {
        int cc[3] = {c[0], c[1], c[2]};
        int x = c[direction] + (s == 0 ? -disp : disp);
        int n = t->dims[direction];
        if (x < 0 || x >= n) {
            if (!t->periods[direction]) {
                out[s] = MPI_PROC_NULL;
                continue;
            }
            x = ((x % n) + n) % n;
        }
        cc[direction] = x;
        out[s] = cart_rank(t, cc);
    }
    *source = out[0];
    *dest = out[1];
    return MPI_SUCCESS;
}
