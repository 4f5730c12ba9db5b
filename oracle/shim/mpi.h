/*
 * MPI stand-ins used ONLY to compile and run the reference solver's sources in place as a test
 * oracle and CPU baseline (no MPI library exists in this image). Test infrastructure, never product
 * code. Two implementations of this subset:
 *
 * shim_mpi.c (linked into _ref/libteal_ref.so, loaded in-process by the tests): one process, rank 0,
 * size 1. Collectives reduce over one rank (in place = no-op, otherwise a copy). Point-to-point
 * messages are self-sends matched by tag in posting order, which is what the reference's periodic
 * halo exchange needs on one rank (equations/exchange.c:8-51, mesh/create.c:351-440: a periodic
 * Cartesian axis makes the rank its own neighbour). Cartesian topology: every coordinate is 0; a
 * periodic axis shifts to rank 0, a non-periodic axis to MPI_PROC_NULL. Files (the reference's .msh
 * reader): stdio reads at explicit offsets.
 *
 * shim_mpi_fork.c (linked into _ref/teal_ref_mpi): TEAL_SHIM_RANKS processes forked by MPI_Init,
 * messages through shared-memory inboxes; see that file.
 */
#pragma once

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype; /* (kind << 20) | size-in-bytes */
typedef int MPI_Op;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef long long MPI_Offset;
typedef struct shim_request *MPI_Request;
typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    int count;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_PROC_NULL (-1)
#define MPI_INFO_NULL 0
#define MPI_MAX_OBJECT_NAME 64
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

#define MPI_CHAR ((1 << 20) | 1)
#define MPI_INT ((2 << 20) | 4)
#define MPI_UINT ((3 << 20) | 4)
#define MPI_LONG ((4 << 20) | 8)
#define MPI_FLOAT ((5 << 20) | 4)
#define MPI_DOUBLE ((6 << 20) | 8)
/* fixed-width types and file offsets of the reference's .msh reader (core/parse.c, mesh/gmsh.c);
   kinds 7 and 8 are the derived types of MPI_Type_contiguous / MPI_Type_create_resized */
#define MPI_INT8_T ((9 << 20) | 1)
#define MPI_INT16_T ((10 << 20) | 2)
#define MPI_INT32_T ((11 << 20) | 4)
#define MPI_INT64_T ((12 << 20) | 8)
#define MPI_UINT8_T ((13 << 20) | 1)
#define MPI_UINT16_T ((14 << 20) | 2)
#define MPI_UINT32_T ((15 << 20) | 4)
#define MPI_UINT64_T ((16 << 20) | 8)
#define MPI_OFFSET ((17 << 20) | 8)

/* files: one process reading with stdio (shim_mpi.c only) */
typedef struct shim_file *MPI_File;
typedef int MPI_Errhandler;
#define MPI_ERRORS_ARE_FATAL 1
#define MPI_MODE_RDONLY 2
#define MPI_SEEK_SET 600
#define MPI_SEEK_CUR 602
#define MPI_SEEK_END 604

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

int MPI_Init(int *argc, char ***argv);
int MPI_Initialized(int *flag);
int MPI_Finalize(void);
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
double MPI_Wtime(void);

int MPI_Type_size(MPI_Datatype type, int *size);
int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *type);
int MPI_Type_create_resized(MPI_Datatype old, MPI_Aint lb, MPI_Aint extent, MPI_Datatype *type);
int MPI_Type_commit(MPI_Datatype *type);
int MPI_Type_free(MPI_Datatype *type);
int MPI_Type_create_struct(int count, const int *lens, const MPI_Aint *offs, const MPI_Datatype *types,
                           MPI_Datatype *type);
int MPI_Type_get_name(MPI_Datatype type, char *name, int *len);
int MPI_Get_count(const MPI_Status *status, MPI_Datatype type, int *count);

int MPI_Dist_graph_create_adjacent(MPI_Comm old, int indegree, const int *sources, const int *sourceweights,
                                   int outdegree, const int *dests, const int *destweights, MPI_Info info,
                                   int reorder, MPI_Comm *comm);

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_set_errhandler(MPI_File fh, MPI_Errhandler handler);
int MPI_File_read_at(MPI_File fh, MPI_Offset offset, void *buf, int count, MPI_Datatype type,
                     MPI_Status *status);
int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence);
int MPI_File_get_position(MPI_File fh, MPI_Offset *offset);

int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm);
int MPI_Exscan(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op,
               MPI_Comm comm);
int MPI_Scan(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op, MPI_Comm comm);
int MPI_Allgather(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoall(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
                 MPI_Datatype rtype, MPI_Comm comm);
int MPI_Alltoallv(const void *send, const int *scounts, const int *sdispls, MPI_Datatype stype,
                  void *recv, const int *rcounts, const int *rdispls, MPI_Datatype rtype,
                  MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm);

int MPI_Isend(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm,
              MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
              MPI_Request *req);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);
int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype type, int source, int tag, MPI_Comm comm,
             MPI_Status *status);
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag, void *rbuf,
                 int rcount, MPI_Datatype rtype, int source, int rtag, MPI_Comm comm,
                 MPI_Status *status);
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype type, int dest, int stag, int source,
                         int rtag, MPI_Comm comm, MPI_Status *status);

int MPI_Cart_create(MPI_Comm old, int ndims, const int *dims, const int *periods, int reorder,
                    MPI_Comm *comm);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *source, int *dest);
