/*
 * Single-rank MPI stand-in for the CPU oracle (test infrastructure only).
 * See mpi.h for the semantics.  Everything here is rank 0 of 1.
 */
#include "mpi.h"

#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ---- datatypes: a handle indexes a table of byte sizes ------------------ */
#define MAX_TYPES 4096
static long long type_bytes[MAX_TYPES] = {0, 1, 4, 8, 4};
static int n_types = 5;

static long long tsize(MPI_Datatype t)
{
    if (t <= 0 || t >= n_types) {
        fprintf(stderr, "mpi_stub: bad datatype handle %d\n", t);
        abort();
    }
    return type_bytes[t];
}

static MPI_Datatype new_type(long long bytes)
{
    if (n_types >= MAX_TYPES) {
        fprintf(stderr, "mpi_stub: datatype table full\n");
        abort();
    }
    type_bytes[n_types] = bytes;
    return n_types++;
}

int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype *nt)
{
    *nt = new_type((long long)count * tsize(old));
    return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int nd, const int *gsizes, const int *lsizes, const int *starts,
                             int order, MPI_Datatype old, MPI_Datatype *nt)
{
    (void)gsizes; (void)starts; (void)order;
    long long n = 1;
    for (int d = 0; d < nd; d++) n *= lsizes[d];
    *nt = new_type(n * tsize(old));
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }

/* ---- environment --------------------------------------------------------- */
int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm c, int code) { (void)c; exit(code); }
int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)buf; (void)count; (void)t; (void)root; (void)c;
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    memmove(r, s, (size_t)(count * tsize(t)));
    return MPI_SUCCESS;
}

/* one rank: the reduction of one contribution is that contribution */
int MPI_Reduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{
    (void)op; (void)root; (void)c;
    memmove(r, s, (size_t)(count * tsize(t)));
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm old, int nd, const int *dims, const int *periods, int reorder, MPI_Comm *cart)
{
    (void)old; (void)nd; (void)dims; (void)periods; (void)reorder;
    *cart = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm c, int rank, int maxdims, int *coords)
{
    (void)c; (void)rank;
    for (int d = 0; d < maxdims; d++) coords[d] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm c, const int *coords, int *rank)
{
    (void)c; (void)coords;
    *rank = 0;
    return MPI_SUCCESS;
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ---- point to point (to self) -------------------------------------------- */
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype st, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rt, int src, int rtag,
                 MPI_Comm c, MPI_Status *status)
{
    (void)dest; (void)src; (void)c; (void)stag; (void)rtag;
    long long sb = (long long)scount * tsize(st), rb = (long long)rcount * tsize(rt);
    long long n = sb < rb ? sb : rb;
    memmove(rbuf, sbuf, (size_t)n);
    if (status) status->count_bytes = (int)n;
    return MPI_SUCCESS;
}

/* one rank sends to itself: the buffer holds what it sent */
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype t, int dest, int stag, int src, int rtag, MPI_Comm c,
                         MPI_Status *status)
{
    (void)buf; (void)dest; (void)src; (void)c; (void)stag; (void)rtag;
    if (status) status->count_bytes = (int)((long long)count * tsize(t));
    return MPI_SUCCESS;
}

#define MAX_REQ 256
typedef struct { void *buf; long long bytes; int tag; int is_send; int live; } stub_req;
static stub_req reqs_tab[MAX_REQ];
static int n_reqs = 0;

static int new_req(void *buf, long long bytes, int tag, int is_send)
{
    if (n_reqs >= MAX_REQ) {
        fprintf(stderr, "mpi_stub: request table full\n");
        abort();
    }
    reqs_tab[n_reqs] = (stub_req){buf, bytes, tag, is_send, 1};
    return n_reqs++;
}

int MPI_Send_init(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *req)
{
    (void)dest; (void)c;
    *req = new_req((void *)buf, (long long)count * tsize(t), tag, 1);
    return MPI_SUCCESS;
}

int MPI_Recv_init(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req)
{
    (void)src; (void)c;
    *req = new_req(buf, (long long)count * tsize(t), tag, 0);
    return MPI_SUCCESS;
}

/* k-th started receive of a tag takes the k-th started send of that tag, in
 * creation (handle) order. */
int MPI_Startall(int n, MPI_Request *reqs)
{
    int used[MAX_REQ] = {0};
    int order[MAX_REQ];
    int m = 0;
    for (int i = 0; i < n; i++)
        if (reqs[i] >= 0) order[m++] = reqs[i];
    /* sort handles ascending = creation order */
    for (int i = 1; i < m; i++)
        for (int j = i; j > 0 && order[j - 1] > order[j]; j--) {
            int t = order[j]; order[j] = order[j - 1]; order[j - 1] = t;
        }
    for (int i = 0; i < m; i++) {
        stub_req *r = &reqs_tab[order[i]];
        if (r->is_send) continue;
        for (int j = 0; j < m; j++) {
            stub_req *s = &reqs_tab[order[j]];
            if (!s->is_send || used[j] || s->tag != r->tag) continue;
            used[j] = 1;
            long long nb = s->bytes < r->bytes ? s->bytes : r->bytes;
            memmove(r->buf, s->buf, (size_t)nb);
            break;
        }
    }
    return MPI_SUCCESS;
}

int MPI_Testall(int n, MPI_Request *reqs, int *flag, MPI_Status *st)
{
    (void)n; (void)reqs; (void)st;
    *flag = 1;
    return MPI_SUCCESS;
}

int MPI_Waitall(int n, MPI_Request *reqs, MPI_Status *st)
{
    (void)n; (void)reqs; (void)st;
    return MPI_SUCCESS;
}

int MPI_Request_free(MPI_Request *req)
{
    if (*req >= 0 && *req < n_reqs) reqs_tab[*req].live = 0;
    *req = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}

int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count)
{
    *count = (int)(st->count_bytes / tsize(t));
    return MPI_SUCCESS;
}

/* ---- info / MPI-IO ------------------------------------------------------- */
int MPI_Info_create(MPI_Info *info) { *info = 0; return MPI_SUCCESS; }
int MPI_Info_set(MPI_Info info, const char *key, const char *value)
{
    (void)info; (void)key; (void)value;
    return MPI_SUCCESS;
}
int MPI_Info_free(MPI_Info *info) { (void)info; return MPI_SUCCESS; }

int MPI_File_open(MPI_Comm c, const char *name, int amode, MPI_Info info, MPI_File *fh)
{
    (void)c; (void)info;
    *fh = fopen(name, (amode & MPI_MODE_RDONLY) ? "rb" : "wb");
    if (!*fh) {
        fprintf(stderr, "mpi_stub: cannot open %s\n", name);
        abort();
    }
    return MPI_SUCCESS;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype et, MPI_Datatype ft,
                      const char *rep, MPI_Info info)
{
    (void)et; (void)ft; (void)rep; (void)info;
    fseeko(fh, (off_t)disp, SEEK_SET);
    return MPI_SUCCESS;
}

int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st)
{
    size_t nb = (size_t)((long long)count * tsize(t));
    size_t got = fread(buf, 1, nb, fh);
    if (st) st->count_bytes = (int)got;
    return MPI_SUCCESS;
}

int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *st)
{
    size_t nb = (size_t)((long long)count * tsize(t));
    size_t put = fwrite(buf, 1, nb, fh);
    if (st) st->count_bytes = (int)put;
    return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh)
{
    if (*fh) fclose(*fh);
    *fh = NULL;
    return MPI_SUCCESS;
}
