/*
 * Single-rank MPI stand-in: implementation of the subset declared in mpi.h.
 * Test infrastructure only: it exists so the unmodified fdfault reference
 * sources can be compiled into the CPU oracle binary oracle/_ref/fdfault_ref.
 *
 * Semantics for one rank:
 *  - Cartesian topology is 1x1x1, every shift returns MPI_PROC_NULL, and the
 *    reference's ghost exchanges (fields.cpp:276-291) become no-ops;
 *  - collectives copy their send buffer;
 *  - MPI-IO files are POSIX files; a file view of an etype plus a subarray
 *    filetype maps the stream of etype elements onto file offsets exactly as
 *    MPI-2 defines it (tiling the filetype), memory datatypes (vector,
 *    indexed block, basic) are gathered/scattered element by element.
 */
#define _POSIX_C_SOURCE 200809L
#include "mpi.h"

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

struct mpistub_type mpistub_double_t = {0, 8, 1, 1, 1, NULL, 0, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
struct mpistub_type mpistub_int_t = {0, 4, 1, 1, 1, NULL, 0, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};

struct mpistub_file {
    int fd;
    long long disp;       /* view displacement in bytes */
    int esize;            /* etype size in bytes */
    MPI_Datatype ftype;   /* filetype (basic or subarray) */
    long long pos;        /* individual file pointer, in etype units */
};

static double g_barrier_t[2] = {0.0, 0.0};
static int g_nbarrier = 0;

static double now_seconds(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void die(const char *what) {
    fprintf(stderr, "mpi stub: unsupported use of %s with one rank\n", what);
    exit(134);
}

int MPI_Init(int *argc, char ***argv) {
    (void)argc;
    (void)argv;
    return MPI_SUCCESS;
}

int MPI_Finalize(void) {
    const char *path = getenv("FDF_REF_TIMING");
    if (path && g_nbarrier >= 2) {
        FILE *fp = fopen(path, "a");
        if (fp) {
            fprintf(fp, "solve_seconds %.9f\n", g_barrier_t[1] - g_barrier_t[0]);
            fclose(fp);
        }
    }
    return MPI_SUCCESS;
}

int MPI_Abort(MPI_Comm comm, int errorcode) {
    (void)comm;
    fprintf(stderr, "MPI_Abort called with code %d\n", errorcode);
    fflush(stderr);
    exit(134);
}

int MPI_Comm_size(MPI_Comm comm, int *size) {
    (void)comm;
    *size = 1;
    return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank) {
    (void)comm;
    *rank = 0;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) {
    (void)comm;
    g_barrier_t[0] = g_barrier_t[1];
    g_barrier_t[1] = now_seconds();
    g_nbarrier++;
    return MPI_SUCCESS;
}

static size_t type_bytes(MPI_Datatype t, int count) {
    if (t->kind != 0) die("derived type in a collective");
    return (size_t)t->basic_size * (size_t)count;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
                  MPI_Comm comm) {
    (void)op;
    (void)comm;
    memmove(recvbuf, sendbuf, type_bytes(datatype, count));
    return MPI_SUCCESS;
}

int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm) {
    (void)recvcount;
    (void)recvtype;
    (void)comm;
    memmove(recvbuf, sendbuf, type_bytes(sendtype, sendcount));
    return MPI_SUCCESS;
}

int MPI_Dims_create(int nnodes, int ndims, int dims[]) {
    if (nnodes != 1) die("MPI_Dims_create");
    for (int i = 0; i < ndims; i++) {
        if (dims[i] == 0) dims[i] = 1;
        if (dims[i] != 1) die("MPI_Dims_create (manual decomposition)");
    }
    return MPI_SUCCESS;
}

int MPI_Cart_create(MPI_Comm comm_old, int ndims, const int dims[], const int periods[], int reorder,
                    MPI_Comm *comm_cart) {
    (void)comm_old;
    (void)ndims;
    (void)dims;
    (void)periods;
    (void)reorder;
    *comm_cart = MPI_COMM_WORLD;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]) {
    (void)comm;
    (void)rank;
    for (int i = 0; i < maxdims; i++) coords[i] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *rank_source, int *rank_dest) {
    (void)comm;
    (void)direction;
    (void)disp;
    *rank_source = MPI_PROC_NULL;
    *rank_dest = MPI_PROC_NULL;
    return MPI_SUCCESS;
}

int MPI_Comm_group(MPI_Comm comm, MPI_Group *group) {
    (void)comm;
    *group = 1;
    return MPI_SUCCESS;
}

int MPI_Group_incl(MPI_Group group, int n, const int ranks[], MPI_Group *newgroup) {
    (void)group;
    (void)ranks;
    *newgroup = (n > 0) ? 1 : 0;
    return MPI_SUCCESS;
}

int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm *newcomm) {
    (void)comm;
    *newcomm = group ? MPI_COMM_WORLD : MPI_COMM_NULL;
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status) {
    (void)sendbuf;
    (void)sendcount;
    (void)sendtype;
    (void)sendtag;
    (void)recvbuf;
    (void)recvcount;
    (void)recvtype;
    (void)recvtag;
    (void)comm;
    (void)status;
    if (dest != MPI_PROC_NULL || source != MPI_PROC_NULL) die("MPI_Sendrecv to a real rank");
    return MPI_SUCCESS;
}

static MPI_Datatype new_type(void) {
    MPI_Datatype t = (MPI_Datatype)calloc(1, sizeof(struct mpistub_type));
    if (!t) die("allocation");
    return t;
}

int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype,
                    MPI_Datatype *newtype) {
    if (oldtype->kind != 0) die("nested vector type");
    MPI_Datatype t = new_type();
    t->kind = 1;
    t->basic_size = oldtype->basic_size;
    t->count = count;
    t->blocklen = blocklength;
    t->stride = stride;
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_create_indexed_block(int count, int blocklength, const int displacements[],
                                  MPI_Datatype oldtype, MPI_Datatype *newtype) {
    if (oldtype->kind != 0) die("nested indexed type");
    MPI_Datatype t = new_type();
    t->kind = 2;
    t->basic_size = oldtype->basic_size;
    t->count = count;
    t->blocklen = blocklength;
    t->disp = (int *)malloc(sizeof(int) * (size_t)(count > 0 ? count : 1));
    if (!t->disp) die("allocation");
    if (count > 0) memcpy(t->disp, displacements, sizeof(int) * (size_t)count);
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[],
                             int order, MPI_Datatype oldtype, MPI_Datatype *newtype) {
    if (order != MPI_ORDER_C || ndims < 1 || ndims > 3 || oldtype->kind != 0) die("subarray type");
    MPI_Datatype t = new_type();
    t->kind = 3;
    t->basic_size = oldtype->basic_size;
    t->ndims = ndims;
    for (int i = 0; i < ndims; i++) {
        t->sizes[i] = sizes[i];
        t->subsizes[i] = subsizes[i];
        t->starts[i] = starts[i];
    }
    *newtype = t;
    return MPI_SUCCESS;
}

int MPI_Type_commit(MPI_Datatype *datatype) {
    (void)datatype;
    return MPI_SUCCESS;
}

int MPI_Type_free(MPI_Datatype *datatype) {
    if (datatype && *datatype && (*datatype)->kind != 0) {
        free((*datatype)->disp);
        free(*datatype);
        *datatype = NULL;
    }
    return MPI_SUCCESS;
}

int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh) {
    (void)info;
    if (comm == MPI_COMM_NULL) die("MPI_File_open on a null communicator");
    int flags = (amode & MPI_MODE_RDONLY) ? O_RDONLY : O_WRONLY;
    if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
    int fd = open(filename, flags, 0644);
    if (fd < 0) return MPI_ERR_OTHER;
    MPI_File f = (MPI_File)calloc(1, sizeof(struct mpistub_file));
    if (!f) die("allocation");
    f->fd = fd;
    f->esize = 1;
    f->ftype = NULL;
    *fh = f;
    return MPI_SUCCESS;
}

int MPI_File_close(MPI_File *fh) {
    if (fh && *fh) {
        close((*fh)->fd);
        free(*fh);
        *fh = NULL;
    }
    return MPI_SUCCESS;
}

int MPI_File_set_size(MPI_File fh, MPI_Offset size) {
    return ftruncate(fh->fd, (off_t)size) == 0 ? MPI_SUCCESS : MPI_ERR_OTHER;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char *datarep, MPI_Info info) {
    (void)datarep;
    (void)info;
    if (etype->kind != 0) die("derived etype");
    fh->disp = disp;
    fh->esize = etype->basic_size;
    fh->ftype = filetype;
    fh->pos = 0;
    return MPI_SUCCESS;
}

/* Byte offset in the file of stream element p under the current view. */
static long long view_offset(MPI_File fh, long long p) {
    MPI_Datatype ft = fh->ftype;
    if (!ft || ft->kind == 0) return fh->disp + p * fh->esize;
    if (ft->kind != 3) die("non-subarray filetype");
    long long nsub = 1, extent = 1;
    for (int d = 0; d < ft->ndims; d++) {
        nsub *= ft->subsizes[d];
        extent *= ft->sizes[d];
    }
    long long q = p / nsub, r = p % nsub;
    long long idx[3] = {0, 0, 0};
    for (int d = ft->ndims - 1; d >= 0; d--) {
        idx[d] = r % ft->subsizes[d] + ft->starts[d];
        r /= ft->subsizes[d];
    }
    long long lin = 0;
    for (int d = 0; d < ft->ndims; d++) lin = lin * ft->sizes[d] + idx[d];
    return fh->disp + (q * extent + lin) * fh->esize;
}

/* Element offsets (in basic elements) of a memory datatype instance. */
static long long mem_count(MPI_Datatype t) {
    switch (t->kind) {
        case 0: return 1;
        case 1: return t->count * t->blocklen;
        case 2: return t->count * t->blocklen;
        default: die("subarray memory type"); return 0;
    }
}

static long long mem_elem(MPI_Datatype t, long long e) {
    switch (t->kind) {
        case 0: return e;
        case 1: return (e / t->blocklen) * t->stride + e % t->blocklen;
        case 2: return (long long)t->disp[e / t->blocklen] + e % t->blocklen;
        default: die("subarray memory type"); return 0;
    }
}

static long long mem_extent(MPI_Datatype t) {
    /* extent between consecutive instances when count > 1 */
    switch (t->kind) {
        case 0: return 1;
        case 1: return (t->count - 1) * t->stride + t->blocklen;
        default: {
            long long mx = 0;
            for (long i = 0; i < t->count; i++) {
                long long e = (long long)t->disp[i] + t->blocklen;
                if (e > mx) mx = e;
            }
            return mx;
        }
    }
}

/* one contiguous piece of file I/O, repeated until every byte is moved */
static int io_run(int fd, char *mp, long long len, long long off, int write_mode) {
    while (len > 0) {
        ssize_t n = write_mode ? pwrite(fd, mp, (size_t)len, (off_t)off) : pread(fd, mp, (size_t)len, (off_t)off);
        if (n <= 0) return MPI_ERR_OTHER;
        mp += n;
        off += n;
        len -= n;
    }
    return MPI_SUCCESS;
}

/* Elements are visited in the order the view and the memory type define;
 * runs that are contiguous both in memory and in the file are moved by one
 * system call each. */
static int file_io(MPI_File fh, void *buf, int count, MPI_Datatype datatype, int write_mode) {
    int bsz = datatype->basic_size;
    if (bsz != fh->esize) die("etype/memory type size mismatch");
    long long per = mem_count(datatype), ext = mem_extent(datatype);
    char *base = (char *)buf;
    char *run_mp = NULL;
    long long run_off = 0, run_len = 0;
    for (int c = 0; c < count; c++) {
        for (long long e = 0; e < per; e++) {
            char *mp = base + ((long long)c * ext + mem_elem(datatype, e)) * bsz;
            long long off = view_offset(fh, fh->pos);
            if (run_len > 0 && mp == run_mp + run_len && off == run_off + run_len) {
                run_len += bsz;
            } else {
                if (run_len > 0 && io_run(fh->fd, run_mp, run_len, run_off, write_mode) != MPI_SUCCESS)
                    return MPI_ERR_OTHER;
                run_mp = mp;
                run_off = off;
                run_len = bsz;
            }
            fh->pos++;
        }
    }
    if (run_len > 0 && io_run(fh->fd, run_mp, run_len, run_off, write_mode) != MPI_SUCCESS) return MPI_ERR_OTHER;
    return MPI_SUCCESS;
}

int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype datatype, MPI_Status *status) {
    (void)status;
    return file_io(fh, buf, count, datatype, 0);
}

int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype datatype,
                   MPI_Status *status) {
    (void)status;
    return file_io(fh, (void *)buf, count, datatype, 1);
}
