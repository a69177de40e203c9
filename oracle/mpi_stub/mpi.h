/*
 * Single-rank MPI stand-in used ONLY to compile the fdfault reference
 * sources (test infrastructure, never linked into the product).
 *
 * The reference solver (src/*.cpp) talks to MPI for its Cartesian domain
 * decomposition, ghost exchange and MPI-IO output. With exactly one rank all
 * of that collapses: every Cartesian neighbour is MPI_PROC_NULL, every
 * Sendrecv is a no-op, reductions copy, and MPI-IO file views of a subarray
 * that covers the whole global array are plain sequential files.  This header
 * declares exactly the subset of the MPI-3 C API the reference calls
 * (fields.cpp, cartesian.cpp, outputunit.cpp, front.cpp, friction.cpp,
 * slipweak.cpp, stz.cpp, utilities.cpp, domain.cpp, main.cpp) with the
 * standard signatures, so the reference compiles without a single edit.
 *
 * Timing hook: when FDF_REF_TIMING is set in the environment, MPI_Finalize
 * appends one line "solve_seconds <t>" to that file, where <t> is the wall
 * time between the last two MPI_Barrier calls.  In the reference's main.cpp
 * those two barriers bracket problem::solve() (main.cpp:42 and :59), so this
 * times the time-stepping loop only, excluding set-up.
 */
#ifndef FDF_MPI_STUB_H
#define FDF_MPI_STUB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Group;
typedef int MPI_Info;
typedef int MPI_Op;
typedef long long MPI_Offset;
typedef struct mpistub_type *MPI_Datatype;
typedef struct mpistub_file *MPI_File;

typedef struct {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
} MPI_Status;

struct mpistub_type {
    int kind;          /* 0 = basic, 1 = vector, 2 = indexed block, 3 = subarray */
    int basic_size;    /* bytes of the basic element */
    long count;        /* vector: count; indexed: number of blocks */
    long blocklen;     /* elements per block */
    long stride;       /* vector stride (elements) */
    int *disp;         /* indexed block displacements (elements) */
    int ndims;         /* subarray */
    int sizes[3];
    int subsizes[3];
    int starts[3];
};

extern struct mpistub_type mpistub_double_t;
extern struct mpistub_type mpistub_int_t;

#define MPI_DOUBLE (&mpistub_double_t)
#define MPI_INT (&mpistub_int_t)

#define MPI_SUCCESS 0
#define MPI_ERR_OTHER 15
#define MPI_COMM_WORLD 1
#define MPI_COMM_NULL 0
#define MPI_PROC_NULL (-1)
#define MPI_INFO_NULL 0
#define MPI_MIN 1
#define MPI_MAX 2
#define MPI_SUM 3
#define MPI_ORDER_C 56
#define MPI_MODE_RDONLY 2
#define MPI_MODE_WRONLY 4
#define MPI_MODE_CREATE 1
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int errorcode);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Barrier(MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype datatype, MPI_Op op,
                  MPI_Comm comm);
int MPI_Allgather(const void *sendbuf, int sendcount, MPI_Datatype sendtype, void *recvbuf,
                  int recvcount, MPI_Datatype recvtype, MPI_Comm comm);
int MPI_Dims_create(int nnodes, int ndims, int dims[]);
int MPI_Cart_create(MPI_Comm comm_old, int ndims, const int dims[], const int periods[], int reorder,
                    MPI_Comm *comm_cart);
int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int coords[]);
int MPI_Cart_shift(MPI_Comm comm, int direction, int disp, int *rank_source, int *rank_dest);
int MPI_Comm_group(MPI_Comm comm, MPI_Group *group);
int MPI_Group_incl(MPI_Group group, int n, const int ranks[], MPI_Group *newgroup);
int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm *newcomm);
int MPI_Sendrecv(const void *sendbuf, int sendcount, MPI_Datatype sendtype, int dest, int sendtag,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int source, int recvtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Type_vector(int count, int blocklength, int stride, MPI_Datatype oldtype,
                    MPI_Datatype *newtype);
int MPI_Type_create_indexed_block(int count, int blocklength, const int displacements[],
                                  MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_create_subarray(int ndims, const int sizes[], const int subsizes[], const int starts[],
                             int order, MPI_Datatype oldtype, MPI_Datatype *newtype);
int MPI_Type_commit(MPI_Datatype *datatype);
int MPI_Type_free(MPI_Datatype *datatype);
int MPI_File_open(MPI_Comm comm, const char *filename, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_set_size(MPI_File fh, MPI_Offset size);
int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char *datarep, MPI_Info info);
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype datatype, MPI_Status *status);
int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype datatype,
                   MPI_Status *status);

#ifdef __cplusplus
}
#endif

#endif
