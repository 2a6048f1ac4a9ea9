/*
 * mpi_shim.c -- single-rank MPI implementation used only to link and run
 * the reference build as a checker (see mpi.h).  TEST INFRASTRUCTURE ONLY.
 */
#define _GNU_SOURCE
#include "mpi.h"

#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

static int g_initialized = 0;

static void shim_fail(const char *what) {
    fprintf(stderr, "mpi_shim: unsupported operation: %s\n", what);
    fflush(stderr);
    exit(97);
}

/* ---------------------------------------------------------------- types */

typedef struct {
    int used;
    int count, blocklen;
    long long stride_bytes;   /* between block starts */
    MPI_Datatype old;
} derived_t;

#define MAX_DERIVED 64
#define DERIVED_BASE 0x10000
static derived_t g_types[MAX_DERIVED];

static long long basic_size(MPI_Datatype t) {
    switch (t) {
    case MPI_CHAR: case MPI_BYTE: return 1;
    case MPI_INT: case MPI_FLOAT: case MPI_REAL: return 4;
    case MPI_LONG: case MPI_DOUBLE: return 8;
    }
    return -1;
}

static derived_t *derived(MPI_Datatype t) {
    int i = t - DERIVED_BASE;
    if (i < 0 || i >= MAX_DERIVED || !g_types[i].used) return NULL;
    return &g_types[i];
}

static long long type_size(MPI_Datatype t) {
    long long b = basic_size(t);
    if (b > 0) return b;
    derived_t *d = derived(t);
    if (!d) shim_fail("unknown datatype");
    return (long long)d->count * d->blocklen * type_size(d->old);
}

static long long type_extent(MPI_Datatype t) {
    long long b = basic_size(t);
    if (b > 0) return b;
    derived_t *d = derived(t);
    if (!d) shim_fail("unknown datatype");
    long long ext_old = type_extent(d->old);
    if (d->count == 0) return 0;
    return (long long)(d->count - 1) * d->stride_bytes + (long long)d->blocklen * ext_old;
}

/* pack `count` items of type t from buf into out (contiguous); returns bytes */
static long long pack(const char *buf, int count, MPI_Datatype t, char *out) {
    long long b = basic_size(t);
    if (b > 0) { memcpy(out, buf, (size_t)(b * count)); return b * count; }
    derived_t *d = derived(t);
    long long ext = type_extent(t), n = 0, ext_old = type_extent(d->old);
    for (int c = 0; c < count; c++)
        for (int blk = 0; blk < d->count; blk++)
            n += pack(buf + c * ext + blk * d->stride_bytes, d->blocklen, d->old, out + n);
    (void)ext_old;
    return n;
}

static long long unpack(const char *in, int count, MPI_Datatype t, char *buf) {
    long long b = basic_size(t);
    if (b > 0) { memcpy(buf, in, (size_t)(b * count)); return b * count; }
    derived_t *d = derived(t);
    long long ext = type_extent(t), n = 0;
    for (int c = 0; c < count; c++)
        for (int blk = 0; blk < d->count; blk++)
            n += unpack(in + n, d->blocklen, d->old, buf + c * ext + blk * d->stride_bytes);
    return n;
}

static int new_derived(int count, int blocklen, long long stride_bytes, MPI_Datatype old, MPI_Datatype *out) {
    for (int i = 0; i < MAX_DERIVED; i++)
        if (!g_types[i].used) {
            g_types[i].used = 1; g_types[i].count = count; g_types[i].blocklen = blocklen;
            g_types[i].stride_bytes = stride_bytes; g_types[i].old = old;
            *out = DERIVED_BASE + i;
            return MPI_SUCCESS;
        }
    shim_fail("too many derived datatypes");
    return MPI_ERR_OTHER;
}

int MPI_Type_vector(int count, int blocklen, int stride, MPI_Datatype old, MPI_Datatype *out) {
    return new_derived(count, blocklen, (long long)stride * type_extent(old), old, out);
}
int MPI_Type_create_hvector(int count, int blocklen, MPI_Aint stride, MPI_Datatype old, MPI_Datatype *out) {
    return new_derived(count, blocklen, (long long)stride, old, out);
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return MPI_SUCCESS; }
int MPI_Type_free(MPI_Datatype *t) {
    /* types built on a freed type stay valid in MPI; keep the entry */
    *t = MPI_DATATYPE_NULL;
    return MPI_SUCCESS;
}
int MPI_Type_size(MPI_Datatype t, int *size) { *size = (int)type_size(t); return MPI_SUCCESS; }

/* ------------------------------------------------------------ process */

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; g_initialized = 1; return MPI_SUCCESS; }
int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
    (void)required; MPI_Init(argc, argv); *provided = MPI_THREAD_MULTIPLE; return MPI_SUCCESS;
}
int MPI_Initialized(int *flag) { *flag = g_initialized; return MPI_SUCCESS; }
int MPI_Finalize(void) { g_initialized = 0; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) {
    (void)comm;
    fprintf(stderr, "mpi_shim: MPI_Abort(%d)\n", code);
    fflush(stdout); fflush(stderr);
    exit(code ? code : 1);
}
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *out) {
    (void)comm; (void)color; (void)key; *out = MPI_COMM_SELF; return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }
double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* -------------------------------------------------------- collectives */

int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm comm) {
    (void)buf; (void)count; (void)t; (void)root; (void)comm; return MPI_SUCCESS;
}
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm comm) {
    (void)op; (void)root; (void)comm;
    if (sbuf != MPI_IN_PLACE && sbuf != rbuf) memcpy(rbuf, sbuf, (size_t)(count * type_size(t)));
    return MPI_SUCCESS;
}
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm comm) {
    return MPI_Reduce(sbuf, rbuf, count, t, op, 0, comm);
}
int MPI_Gatherv(const void *sbuf, int scount, MPI_Datatype st, void *rbuf, const int *rcounts,
                const int *displs, MPI_Datatype rt, int root, MPI_Comm comm) {
    (void)rcounts; (void)root; (void)comm;
    char *tmp = (char *)malloc((size_t)(scount * type_size(st)) + 1);
    pack((const char *)sbuf, scount, st, tmp);
    unpack(tmp, scount, rt, (char *)rbuf + (long long)displs[0] * type_extent(rt));
    free(tmp);
    return MPI_SUCCESS;
}
int MPI_Scatterv(const void *sbuf, const int *scounts, const int *displs, MPI_Datatype st,
                 void *rbuf, int rcount, MPI_Datatype rt, int root, MPI_Comm comm) {
    (void)scounts; (void)root; (void)comm;
    char *tmp = (char *)malloc((size_t)(rcount * type_size(rt)) + 1);
    pack((const char *)sbuf + (long long)displs[0] * type_extent(st), rcount, rt, tmp);
    unpack(tmp, rcount, rt, (char *)rbuf);
    free(tmp);
    return MPI_SUCCESS;
}

/* ---------------------------------------------------- point to point */

typedef struct msg_t { int tag; long long bytes; char *data; struct msg_t *next; } msg_t;
static msg_t *g_queue = NULL;

static int post_self(const void *buf, int count, MPI_Datatype t, int dest, int tag) {
    if (dest == MPI_PROC_NULL) return MPI_SUCCESS;
    if (dest != 0) shim_fail("send to a rank other than self");
    msg_t *m = (msg_t *)malloc(sizeof(msg_t));
    m->tag = tag;
    m->bytes = type_size(t) * count;
    m->data = (char *)malloc((size_t)m->bytes + 1);
    pack((const char *)buf, count, t, m->data);
    m->next = NULL;
    msg_t **p = &g_queue;
    while (*p) p = &(*p)->next;
    *p = m;
    return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm) {
    (void)comm; return post_self(buf, count, t, dest, tag);
}
int MPI_Bsend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm comm) {
    (void)comm; return post_self(buf, count, t, dest, tag);
}
int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm comm, MPI_Status *st) {
    (void)comm; (void)count;
    if (src == MPI_PROC_NULL) {
        if (st) { st->MPI_SOURCE = MPI_PROC_NULL; st->MPI_TAG = MPI_ANY_TAG; st->count_bytes = 0; }
        return MPI_SUCCESS;
    }
    msg_t **p = &g_queue;
    while (*p && !((*p)->tag == tag || tag == MPI_ANY_TAG)) p = &(*p)->next;
    if (!*p) shim_fail("receive with no matching self message (would deadlock)");
    msg_t *m = *p;
    *p = m->next;
    unpack(m->data, (int)(m->bytes / type_size(t)), t, (char *)buf);
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = m->tag; st->MPI_ERROR = 0; st->count_bytes = m->bytes; }
    free(m->data); free(m);
    return MPI_SUCCESS;
}
int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype st, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rt, int src, int rtag,
                 MPI_Comm comm, MPI_Status *status) {
    post_self(sbuf, scount, st, dest, stag);
    if (src == MPI_PROC_NULL) {
        if (status) { status->MPI_SOURCE = MPI_PROC_NULL; status->count_bytes = 0; }
        return MPI_SUCCESS;
    }
    return MPI_Recv(rbuf, rcount, rt, src, rtag, comm, status);
}
int MPI_Buffer_attach(void *buf, int size) { (void)buf; (void)size; return MPI_SUCCESS; }
int MPI_Buffer_detach(void *buf, int *size) { (void)buf; (void)size; return MPI_SUCCESS; }

/* -------------------------------------------------------------- MPI-IO */

#define MAX_FILES 32
static struct { int fd; long long pos; } g_files[MAX_FILES];

int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh) {
    (void)comm; (void)info;
    int flags = 0;
    if (amode & MPI_MODE_RDWR) flags = O_RDWR;
    else if (amode & MPI_MODE_WRONLY) flags = O_WRONLY;
    else flags = O_RDONLY;
    if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
    int fd = open(name, flags, 0644);
    if (fd < 0) return MPI_ERR_OTHER;
    for (int i = 0; i < MAX_FILES; i++)
        if (g_files[i].fd == 0) {
            g_files[i].fd = fd + 1;   /* 0 marks a free slot */
            g_files[i].pos = 0;
            *fh = i;
            return MPI_SUCCESS;
        }
    close(fd);
    shim_fail("too many open files");
    return MPI_ERR_OTHER;
}
int MPI_File_close(MPI_File *fh) {
    if (*fh >= 0 && *fh < MAX_FILES && g_files[*fh].fd) {
        close(g_files[*fh].fd - 1);
        g_files[*fh].fd = 0;
    }
    *fh = -1;
    return MPI_SUCCESS;
}
int MPI_File_seek(MPI_File fh, MPI_Offset off, int whence) {
    if (whence == MPI_SEEK_SET) g_files[fh].pos = off;
    else if (whence == MPI_SEEK_CUR) g_files[fh].pos += off;
    else {
        struct stat sb; fstat(g_files[fh].fd - 1, &sb);
        g_files[fh].pos = (long long)sb.st_size + off;
    }
    return MPI_SUCCESS;
}

static int io_read(MPI_File fh, long long off, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    long long n = type_size(t) * count;
    char *tmp = (char *)malloc((size_t)n + 1);
    long long got = 0;
    while (got < n) {
        ssize_t r = pread(g_files[fh].fd - 1, tmp + got, (size_t)(n - got), (off_t)(off + got));
        if (r <= 0) break;
        got += r;
    }
    if (got < n) memset(tmp + got, 0, (size_t)(n - got));
    unpack(tmp, count, t, (char *)buf);
    free(tmp);
    if (st) { st->count_bytes = got; st->MPI_ERROR = 0; }
    return MPI_SUCCESS;
}
static int io_write(MPI_File fh, long long off, const void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    long long n = type_size(t) * count;
    char *tmp = (char *)malloc((size_t)n + 1);
    pack((const char *)buf, count, t, tmp);
    long long put = 0;
    while (put < n) {
        ssize_t r = pwrite(g_files[fh].fd - 1, tmp + put, (size_t)(n - put), (off_t)(off + put));
        if (r <= 0) break;
        put += r;
    }
    free(tmp);
    if (st) { st->count_bytes = put; st->MPI_ERROR = 0; }
    return put == n ? MPI_SUCCESS : MPI_ERR_OTHER;
}

int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    return io_read(fh, off, buf, count, t, st);
}
int MPI_File_read_at_all(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    return io_read(fh, off, buf, count, t, st);
}
int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    return io_write(fh, off, buf, count, t, st);
}
int MPI_File_write_at_all(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    return io_write(fh, off, buf, count, t, st);
}
int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    int r = io_read(fh, g_files[fh].pos, buf, count, t, st);
    g_files[fh].pos += type_size(t) * count;
    return r;
}
int MPI_File_read_all(MPI_File fh, void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    return MPI_File_read(fh, buf, count, t, st);
}
int MPI_File_write(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    int r = io_write(fh, g_files[fh].pos, buf, count, t, st);
    g_files[fh].pos += type_size(t) * count;
    return r;
}
int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype t, MPI_Status *st) {
    return MPI_File_write(fh, buf, count, t, st);
}
