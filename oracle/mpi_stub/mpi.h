/*
 * Single-rank MPI stand-in used ONLY to compile the reference's own C step
 * functions (DNS-solver/src/*.c) for the CPU oracle.  Test infrastructure:
 * nothing in the product library includes this header.
 *
 * Semantics (one process, rank 0 of 1, a 1x1 periodic Cartesian grid):
 *   - collectives copy send -> receive buffers (a sum over one rank);
 *   - MPI_Sendrecv copies the send buffer into the receive buffer;
 *   - persistent requests (MPI_Send_init / MPI_Recv_init) are matched, on
 *     MPI_Startall, k-th receive of a tag with k-th send of that tag in the
 *     order they were created, which is MPI's ordered matching on self;
 *   - MPI-IO supports the single-rank case where a file view covers the whole
 *     global array: reads/writes are plain contiguous stdio transfers at the
 *     view's displacement.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long long MPI_Offset;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count_bytes; } MPI_Status;
typedef FILE *MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_SUM 0
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL (-1)
#define MPI_ORDER_C 0
#define MPI_MODE_RDONLY 1
#define MPI_MODE_WRONLY 2
#define MPI_MODE_CREATE 4
#define MPI_SUCCESS 0

/* predefined datatypes are handles 1..4; derived types are appended */
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_INTEGER 4  /* the Fortran INTEGER handle, 4 bytes here */

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm c, int code);
int MPI_Comm_size(MPI_Comm c, int *size);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Barrier(MPI_Comm c);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Cart_create(MPI_Comm old, int nd, const int *dims, const int *periods, int reorder, MPI_Comm *cart);
int MPI_Cart_coords(MPI_Comm c, int rank, int maxdims, int *coords);
int MPI_Cart_rank(MPI_Comm c, const int *coords, int *rank);
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype st, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rt, int src, int rtag,
                 MPI_Comm c, MPI_Status *status);
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype t, int dest, int stag, int src, int rtag, MPI_Comm c,
                         MPI_Status *status);
int MPI_Send_init(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *req);
int MPI_Recv_init(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req);
int MPI_Startall(int n, MPI_Request *reqs);
int MPI_Testall(int n, MPI_Request *reqs, int *flag, MPI_Status *st);
int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *st);
int MPI_Request_free(MPI_Request *req);
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count);
double MPI_Wtime(void);

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *nt);
int MPI_Type_create_subarray(int nd, const int *gsizes, const int *lsizes, const int *starts,
                             int order, MPI_Datatype old, MPI_Datatype *nt);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);

int MPI_Info_create(MPI_Info *info);
int MPI_Info_set(MPI_Info info, const char *key, const char *value);
int MPI_Info_free(MPI_Info *info);

int MPI_File_open(MPI_Comm c, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype et, MPI_Datatype ft,
                      const char *rep, MPI_Info info);
int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_close(MPI_File *fh);

#ifdef __cplusplus
}
#endif
#endif
