/*
 * mpi.h -- single-rank MPI shim for building the reference (OpenCFD-SCU)
 * as a checker on one GPU.  TEST INFRASTRUCTURE ONLY.
 *
 * Covers exactly the MPI surface the reference calls: one process, rank 0 of
 * size 1; point-to-point messages go to self (Sendrecv copies, Send/Bsend
 * queue, Recv dequeues); collectives copy; MPI-IO maps onto pread/pwrite.
 * Handles are plain ints (MPICH style) because the reference casts
 * integer literals to MPI_Comm (head/cuda_commen.h:27).
 */
#ifndef OCFD_MPI_SHIM_H
#define OCFD_MPI_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef int MPI_File;
typedef long long MPI_Offset;
typedef long MPI_Aint;

typedef struct MPI_Status {
    int MPI_SOURCE;
    int MPI_TAG;
    int MPI_ERROR;
    long long count_bytes;
} MPI_Status;

#define MPI_COMM_WORLD   ((MPI_Comm)0x44000000)
#define MPI_COMM_SELF    ((MPI_Comm)0x44000001)
#define MPI_COMM_NULL    ((MPI_Comm)0x04000000)

#define MPI_CHAR         ((MPI_Datatype)0x4c000101)
#define MPI_BYTE         ((MPI_Datatype)0x4c00010d)
#define MPI_INT          ((MPI_Datatype)0x4c000405)
#define MPI_FLOAT        ((MPI_Datatype)0x4c00040a)
#define MPI_REAL         ((MPI_Datatype)0x4c00041c)
#define MPI_LONG         ((MPI_Datatype)0x4c000807)
#define MPI_DOUBLE       ((MPI_Datatype)0x4c00080b)
#define MPI_DATATYPE_NULL ((MPI_Datatype)0x0c000000)

#define MPI_SUM          ((MPI_Op)0x58000003)
#define MPI_MAX          ((MPI_Op)0x58000001)
#define MPI_MIN          ((MPI_Op)0x58000002)

#define MPI_INFO_NULL    ((MPI_Info)0x1c000000)
#define MPI_PROC_NULL    (-1)
#define MPI_ANY_SOURCE   (-2)
#define MPI_ANY_TAG      (-1)
#define MPI_SUCCESS      0
#define MPI_ERR_OTHER    15
#define MPI_THREAD_SINGLE     0
#define MPI_THREAD_FUNNELED   1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE   3
#define MPI_MODE_CREATE  1
#define MPI_MODE_RDONLY  2
#define MPI_MODE_WRONLY  4
#define MPI_MODE_RDWR    8
#define MPI_SEEK_SET     600
#define MPI_SEEK_CUR     602
#define MPI_SEEK_END     604
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE     ((void *)-1)
#define MPI_MAX_PROCESSOR_NAME 128

int MPI_Init(int *argc, char ***argv);
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided);
int MPI_Initialized(int *flag);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm comm, int code);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *out);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
double MPI_Wtime(void);

int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm);
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm);
int MPI_Gatherv(const void *sbuf, int scount, MPI_Datatype st, void *rbuf, const int *rcounts,
                const int *displs, MPI_Datatype rt, int root, MPI_Comm comm);
int MPI_Scatterv(const void *sbuf, const int *scounts, const int *displs, MPI_Datatype st,
                 void *rbuf, int rcount, MPI_Datatype rt, int root, MPI_Comm comm);

int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Bsend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm);
int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status *st);
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype st, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rt, int src, int rtag,
                 MPI_Comm comm, MPI_Status *status);
int MPI_Buffer_attach(void *buf, int size);
int MPI_Buffer_detach(void *buf, int *size);

int MPI_Type_vector(int count, int blocklen, int stride, MPI_Datatype old, MPI_Datatype *out);
int MPI_Type_create_hvector(int count, int blocklen, MPI_Aint stride, MPI_Datatype old, MPI_Datatype *out);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);
int MPI_Type_size(MPI_Datatype t, int *size);

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh);
int MPI_File_close(MPI_File *fh);
int MPI_File_seek(MPI_File fh, MPI_Offset off, int whence);
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_read_at_all(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *st);
int MPI_File_write_at_all(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *st);

#ifdef __cplusplus
}
#endif
#endif
