/*
 * Single-rank MPI stand-in (see mpi.h). Test infrastructure only.
 */
#define _POSIX_C_SOURCE 200809L
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static int type_bytes(MPI_Datatype type)
{
    return type & ((1 << 20) - 1);
}

/* ---- environment ---------------------------------------------------------------------------- */

static int initialized = 0;

int MPI_Init(int *argc, char ***argv)
{
    (void)argc;
    (void)argv;
    initialized = 1;
    return MPI_SUCCESS;
}

int MPI_Initialized(int *flag)
{
    *flag = initialized;
    return MPI_SUCCESS;
}

int MPI_Finalize(void)
{
    initialized = 0;
    return MPI_SUCCESS;
}

int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm)
{
    *newcomm = comm;
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
    *rank = 0;
    return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
    (void)comm;
    *size = 1;
    return MPI_SUCCESS;
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + (1e-9 * (double)ts.tv_nsec);
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

/* ---- collectives over one rank -------------------------------------------------------------- */

static void copy_in(const void *send, void *recv, size_t bytes)
{
    if (send != MPI_IN_PLACE && send != recv && bytes) {
        memmove(recv, send, bytes);
    }
}

int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
    (void)op;
    (void)comm;
    copy_in(send, recv, (size_t)count * type_bytes(type));
    return MPI_SUCCESS;
}

int MPI_Exscan(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op,
               MPI_Comm comm)
{
    /* the result on rank 0 is undefined by the standard; the reference zeroes it itself */
    (void)send;
    (void)recv;
    (void)count;
    (void)type;
    (void)op;
    (void)comm;
    return MPI_SUCCESS;
}

int MPI_Scan(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm)
{
    (void)op;
    (void)comm;
    copy_in(send, recv, (size_t)count * type_bytes(type));
    return MPI_SUCCESS;
}

int MPI_Allgather(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm)
{
    (void)rcount;
    (void)rtype;
    (void)comm;
    copy_in(send, recv, (size_t)scount * type_bytes(stype));
    return MPI_SUCCESS;
}

int MPI_Alltoall(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
                 MPI_Datatype rtype, MPI_Comm comm)
{
    (void)rcount;
    (void)rtype;
    (void)comm;
    copy_in(send, recv, (size_t)scount * type_bytes(stype));
    return MPI_SUCCESS;
}

int MPI_Alltoallv(const void *send, const int *scounts, const int *sdispls, MPI_Datatype stype,
                  void *recv, const int *rcounts, const int *rdispls, MPI_Datatype rtype,
                  MPI_Comm comm)
{
    (void)rcounts;
    (void)comm;
    size_t sb = type_bytes(stype), rb = type_bytes(rtype);
    if (scounts[0]) {
        memmove((char *)recv + (rdispls[0] * rb), (const char *)send + (sdispls[0] * sb),
                scounts[0] * sb);
    }
    return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)buf;
    (void)count;
    (void)type;
    (void)root;
    (void)comm;
    return MPI_SUCCESS;
}

/* ---- self-sends matched by tag in posting order --------------------------------------------- */

struct shim_request {
    int is_recv;
    int done;
    int tag;
    void *buf;
    size_t bytes;
    struct shim_request *next; /* pending list link */
};

typedef struct message {
    int tag;
    size_t bytes;
    struct message *next;
    char data[];
} Message;

static Message *queue_head = 0, *queue_tail = 0;
static struct shim_request *pending_head = 0, *pending_tail = 0;

static void fail(const char *what)
{
    fprintf(stderr, "mpi shim: %s\n", what);
    abort();
}

static void deliver(struct shim_request *recv, const void *data, size_t bytes)
{
    if (bytes > recv->bytes) {
        fail("message truncated");
    }
    memcpy(recv->buf, data, bytes);
    recv->done = 1;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request *req)
{
    (void)comm;
    size_t bytes = (size_t)count * type_bytes(type);
    struct shim_request *r = calloc(1, sizeof(*r));
    r->done = 1; /* eager: the payload is copied now */
    *req = r;
    if (dest == MPI_PROC_NULL) {
        return MPI_SUCCESS;
    }
    if (dest != 0) {
        fail("send to a rank other than 0");
    }
    for (struct shim_request **p = &pending_head, *prev = 0; *p; prev = *p, p = &(*p)->next) {
        if ((*p)->tag == tag) {
            struct shim_request *match = *p;
            *p = match->next;
            if (pending_tail == match) {
                pending_tail = prev;
            }
            deliver(match, buf, bytes);
            return MPI_SUCCESS;
        }
    }
    Message *m = malloc(sizeof(*m) + bytes);
    m->tag = tag;
    m->bytes = bytes;
    m->next = 0;
    if (bytes) {
        memcpy(m->data, buf, bytes);
    }
    if (queue_tail) {
        queue_tail->next = m;
    }
    else {
        queue_head = m;
    }
    queue_tail = m;
    return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
              MPI_Request *req)
{
    (void)comm;
    struct shim_request *r = calloc(1, sizeof(*r));
    r->is_recv = 1;
    r->tag = tag;
    r->buf = buf;
    r->bytes = (size_t)count * type_bytes(type);
    *req = r;
    if (source == MPI_PROC_NULL) {
        r->done = 1;
        return MPI_SUCCESS;
    }
    if (source != 0) {
        fail("receive from a rank other than 0");
    }
    for (Message **p = &queue_head, *prev = 0; *p; prev = *p, p = &(*p)->next) {
        if ((*p)->tag == tag) {
            Message *m = *p;
            *p = m->next;
            if (queue_tail == m) {
                queue_tail = prev;
            }
            deliver(r, m->data, m->bytes);
            free(m);
            return MPI_SUCCESS;
        }
    }
    r->next = 0;
    if (pending_tail) {
        pending_tail->next = r;
    }
    else {
        pending_head = r;
    }
    pending_tail = r;
    return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
    (void)statuses;
    for (int i = 0; i < count; i++) {
        if (!reqs[i]) {
            continue;
        }
        if (!reqs[i]->done) {
            fail("wait on a receive that no send matches (single rank deadlock)");
        }
        free(reqs[i]);
        reqs[i] = 0;
    }
    return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
    MPI_Request r;
    MPI_Isend(buf, count, type, dest, tag, comm, &r);
    return MPI_Waitall(1, &r, MPI_STATUSES_IGNORE);
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status *status)
{
    (void)status;
    MPI_Request r;
    MPI_Irecv(buf, count, type, source, tag, comm, &r);
    return MPI_Waitall(1, &r, MPI_STATUSES_IGNORE);
}

int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag, void *rbuf,
                 int rcount, MPI_Datatype rtype, int source, int rtag, MPI_Comm comm,
                 MPI_Status *status)
{
    (void)status;
    MPI_Request r[2];
    MPI_Irecv(rbuf, rcount, rtype, source, rtag, comm, &r[0]);
    MPI_Isend(sbuf, scount, stype, dest, stag, comm, &r[1]);
    return MPI_Waitall(2, r, MPI_STATUSES_IGNORE);
}

int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype type, int dest, int stag, int source,
                         int rtag, MPI_Comm comm, MPI_Status *status)
{
    size_t bytes = (size_t)count * type_bytes(type);
    void *tmp = malloc(bytes ? bytes : 1);
    memcpy(tmp, buf, bytes);
    int ret = MPI_Sendrecv(tmp, count, type, dest, stag, buf, count, type, source, rtag, comm,
                           status);
    free(tmp);
    return ret;
}

/* ---- Cartesian topology on one rank --------------------------------------------------------- */

static int cart_periods[3] = {0, 0, 0};
static int cart_ndims = 0;

int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder,
                    MPI_Comm *comm)
{
    (void)reorder;
    if (ndims > 3) {
        fail("more than 3 Cartesian dimensions");
    }
    for (int i = 0; i < ndims; i++) {
        if (dims[i] != 1) {
            fail("Cartesian grid with more than one rank");
        }
        cart_periods[i] = periods[i];
    }
    cart_ndims = ndims;
    *comm = old;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords)
{
    (void)comm;
    (void)rank;
    for (int i = 0; i < maxdims; i++) {
        coords[i] = 0;
    }
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *source, int *dest)
{
    (void)comm;
    (void)disp;
    if (direction < 0 || direction >= cart_ndims) {
        fail("invalid Cartesian shift direction");
    }
    int nbr = cart_periods[direction] ? 0 : MPI_PROC_NULL;
    *source = nbr;
    *dest = nbr;
    return MPI_SUCCESS;
}

/* ---- derived types, names and counts ---------------------------------------------------------- */

int MPI_Type_create_struct(int count, const int *lens, const MPI_Aint *offs, const MPI_Datatype *types,
                           MPI_Datatype *type)
{
    long end = 0;
    for (int i = 0; i < count; i++) {
        long e = offs[i] + (long)lens[i] * type_bytes(types[i]);
        if (e > end) end = e;
    }
    *type = (18 << 20) | (int)end;
    return MPI_SUCCESS;
}

int MPI_Type_get_name(MPI_Datatype type, char *name, int *len)
{
    static const char *names[] = {"?",         "MPI_CHAR",     "MPI_INT",      "MPI_UINT",     "MPI_LONG",
                                  "MPI_FLOAT", "MPI_DOUBLE",   "contiguous",   "resized",      "MPI_INT8_T",
                                  "MPI_INT16_T", "MPI_INT32_T", "MPI_INT64_T", "MPI_UINT8_T", "MPI_UINT16_T",
                                  "MPI_UINT32_T", "MPI_UINT64_T", "MPI_OFFSET", "struct"};
    int kind = type >> 20;
    const char *n = (kind >= 0 && kind < (int)(sizeof(names) / sizeof(*names))) ? names[kind] : "?";
    *len = (int)strlen(n);
    memcpy(name, n, (size_t)*len + 1);
    return MPI_SUCCESS;
}

/* the status of a file read carries the bytes read */
int MPI_Get_count(const MPI_Status *status, MPI_Datatype type, int *count)
{
    *count = status->count / type_bytes(type);
    return MPI_SUCCESS;
}

/* one rank: the neighbourhood graph has no edges to anyone else */
int MPI_Dist_graph_create_adjacent(MPI_Comm old, int indegree, const int *sources, const int *sourceweights,
                                   int outdegree, const int *dests, const int *destweights, MPI_Info info,
                                   int reorder, MPI_Comm *comm)
{
    (void)sources;
    (void)sourceweights;
    (void)dests;
    (void)destweights;
    (void)info;
    (void)reorder;
    for (int i = 0; i < indegree; i++) {
        if (sources[i] != 0) return 1;
    }
    for (int i = 0; i < outdegree; i++) {
        if (dests[i] != 0) return 1;
    }
    *comm = old;
    return MPI_SUCCESS;
}

/* ---- files: stdio reads at explicit offsets ------------------------------------------------- */

struct shim_file {
    FILE *f;
    MPI_Offset pos;
};

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh)
{
    (void)comm;
    (void)info;
    if (amode != MPI_MODE_RDONLY) return 1;
    FILE *f = fopen(name, "rb");
    if (!f) return 1;
    struct shim_file *h = calloc(1, sizeof(*h));
    h->f = f;
    *fh = h;
    return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh)
{
    if (*fh) {
        fclose((*fh)->f);
        free(*fh);
        *fh = 0;
    }
    return MPI_SUCCESS;
}

int MPI_File_set_errhandler(MPI_File fh, MPI_Errhandler handler)
{
    (void)fh;
    (void)handler;
    return MPI_SUCCESS;
}

int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype type,
                     MPI_Status *status)
{
    size_t bytes = (size_t)count * (size_t)type_bytes(type);
    size_t got = 0;
    if (fseeko(fh->f, (off_t)offset, SEEK_SET) == 0) {
        got = fread(buf, 1, bytes, fh->f);
    }
    if (status) {
        status->MPI_SOURCE = 0;
        status->MPI_TAG = 0;
        status->MPI_ERROR = MPI_SUCCESS;
        status->count = (int)got;
    }
    return MPI_SUCCESS;
}

int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence)
{
    if (whence == MPI_SEEK_SET) fh->pos = offset;
    else if (whence == MPI_SEEK_CUR) fh->pos += offset;
    else return 1;
    return MPI_SUCCESS;
}

int MPI_File_get_position(MPI_File fh, MPI_Offset *offset)
{
    *offset = fh->pos;
    return MPI_SUCCESS;
}
