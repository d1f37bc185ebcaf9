/*
 * mpi.h -- single-process stand-in for the MPI surface that
 * RuanPetrus/cuda-graph-traversal uses (src/worker.cu:6-109,
 * src/traversal.cu:408,558,666,685,705, src/graph_generation.cu:327-390,
 * src/visualization.cu:64-108, examples/graph500_runner.cu:199,250,277-412).
 *
 * One rank, rank 0: reductions, gathers and barriers are copies or no-ops,
 * MPI_Wtime is CLOCK_MONOTONIC, and the MPI-IO calls map to POSIX file
 * descriptors with 64-bit offsets.  Everything is header-only (static
 * inline) so a translation unit that includes it needs no MPI library.
 */
#ifndef G5_SHIM_MPI_H
#define G5_SHIM_MPI_H

#include <fcntl.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef int MPI_File;
typedef struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_INFO_NULL 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_IN_PLACE ((void *)1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

#define MPI_MODE_RDONLY 0x1
#define MPI_MODE_WRONLY 0x2
#define MPI_MODE_RDWR 0x4
#define MPI_MODE_CREATE 0x8

/* Datatypes carry their size in bytes so copies need no lookup table. */
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_INT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 0x104
#define MPI_INT64_T 8
#define MPI_UINT64_T 0x108
#define MPI_LONG_LONG 8
#define MPI_UNSIGNED_LONG_LONG 0x108
#define MPI_DOUBLE 0x208

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t g5_mpi_type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); return code; }
static inline int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_split_type(MPI_Comm comm, int type, int key, MPI_Info info, MPI_Comm *out) {
    (void)comm; (void)type; (void)key; (void)info; *out = MPI_COMM_WORLD; return MPI_SUCCESS;
}
static inline int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *out) {
    (void)comm; (void)color; (void)key; *out = MPI_COMM_WORLD; return MPI_SUCCESS;
}
static inline int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

/* With one rank every reduction is the identity on the local buffer. */
static inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype type, MPI_Op op,
                                MPI_Comm comm) {
    (void)op; (void)comm;
    if (send != MPI_IN_PLACE && send != recv) memcpy(recv, send, (size_t)count * g5_mpi_type_size(type));
    return MPI_SUCCESS;
}
static inline int MPI_Gather(const void *send, int scount, MPI_Datatype stype, void *recv, int rcount,
                             MPI_Datatype rtype, int root, MPI_Comm comm) {
    (void)rcount; (void)rtype; (void)root; (void)comm;
    if (send != MPI_IN_PLACE && recv) memcpy(recv, send, (size_t)scount * g5_mpi_type_size(stype));
    return MPI_SUCCESS;
}
static inline int MPI_Gatherv(const void *send, int scount, MPI_Datatype stype, void *recv,
                              const int *rcounts, const int *displs, MPI_Datatype rtype, int root,
                              MPI_Comm comm) {
    (void)rcounts; (void)root; (void)comm;
    if (send != MPI_IN_PLACE && recv)
        memcpy((char *)recv + (size_t)(displs ? displs[0] : 0) * g5_mpi_type_size(rtype), send,
               (size_t)scount * g5_mpi_type_size(stype));
    return MPI_SUCCESS;
}

static inline double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static inline int MPI_File_open(MPI_Comm comm, const char *name, int amode, MPI_Info info, MPI_File *fh) {
    (void)comm; (void)info;
    int flags = (amode & MPI_MODE_RDWR) ? O_RDWR : (amode & MPI_MODE_WRONLY) ? O_WRONLY : O_RDONLY;
    if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
    *fh = open(name, flags, 0644);
    return *fh < 0 ? 1 : MPI_SUCCESS;
}
static inline int MPI_File_set_size(MPI_File fh, MPI_Offset size) {
    return fh < 0 || ftruncate(fh, (off_t)size) != 0;
}
static inline int g5_mpi_pio(MPI_File fh, MPI_Offset off, void *buf, size_t bytes, int write_) {
    char *p = (char *)buf;
    while (bytes) {
        ssize_t n = write_ ? pwrite(fh, p, bytes, (off_t)off) : pread(fh, p, bytes, (off_t)off);
        if (n <= 0) return 1;
        p += n; off += n; bytes -= (size_t)n;
    }
    return MPI_SUCCESS;
}
static inline int MPI_File_write_at(MPI_File fh, MPI_Offset off, const void *buf, int count, MPI_Datatype type,
                                    MPI_Status *st) {
    (void)st;
    return g5_mpi_pio(fh, off, (void *)buf, (size_t)(unsigned)count * g5_mpi_type_size(type), 1);
}
static inline int MPI_File_read_at(MPI_File fh, MPI_Offset off, void *buf, int count, MPI_Datatype type,
                                   MPI_Status *st) {
    (void)st;
    return g5_mpi_pio(fh, off, buf, (size_t)(unsigned)count * g5_mpi_type_size(type), 0);
}
static inline int MPI_File_close(MPI_File *fh) {
    if (*fh >= 0) close(*fh);
    *fh = -1;
    return MPI_SUCCESS;
}

#endif /* G5_SHIM_MPI_H */
