/*
 * Single-rank stand-in for <mpi.h>, used ONLY to compile the reference KuQCD sources as a CPU oracle
 * (test infrastructure; nothing in the kuqcd_b200 product path includes this file).
 *
 * Every communicator has exactly one rank.  Collectives copy send buffers to receive buffers, point-to-point
 * calls are never reached when the process grid is 1x1x1x1 (the reference only calls them for np > 1,
 * dirac_hisq.cpp:412-414,452-454), and they abort if they are reached anyway.
 *
 * Covers the calls and constants the reference uses: communication.cpp:23-71,113-131,
 * command_line.cpp:34-83, kuqcd_utils.h:40-59, spinor_field.cpp:207-243, test/test_solver.cpp:13-15.
 */
#ifndef KQ_ORACLE_MPI_SHIM_H
#define KQ_ORACLE_MPI_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
    int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD ((MPI_Comm)0x44000000)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3
#define MPI_REQUEST_NULL ((MPI_Request)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_SUM ((MPI_Op)1)

/* the datatype handle encodes the element size in bytes */
#define MPI_CHAR ((MPI_Datatype)1)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_UINT ((MPI_Datatype)4)
#define MPI_UINT32_T ((MPI_Datatype)4)
#define MPI_INT32_T ((MPI_Datatype)4)
#define MPI_FLOAT ((MPI_Datatype)4)
#define MPI_LONG ((MPI_Datatype)8)
#define MPI_INT64_T ((MPI_Datatype)8)
#define MPI_DOUBLE ((MPI_Datatype)8)

static int kq_shim_initialized = 0;

static inline int MPI_Init(int *argc, char ***argv)
{
    (void)argc;
    (void)argv;
    kq_shim_initialized = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Init_thread(int *argc, char ***argv, int required, int *provided)
{
    (void)argc;
    (void)argv;
    if (provided) *provided = required;
    kq_shim_initialized = 1;
    return MPI_SUCCESS;
}
/* A single-rank world is always usable, so report it as initialised (command_line.cpp:34 checks this). */
static inline int MPI_Initialized(int *flag)
{
    *flag = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Finalize(void)
{
    kq_shim_initialized = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_rank(MPI_Comm c, int *r)
{
    (void)c;
    *r = 0;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_size(MPI_Comm c, int *n)
{
    (void)c;
    *n = 1;
    return MPI_SUCCESS;
}
static inline int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c)
{
    (void)buf;
    (void)count;
    (void)t;
    (void)root;
    (void)c;
    return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *s, void *r, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op;
    (void)c;
    if (s != r) memcpy(r, s, (size_t)count * (size_t)t);
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void *s, int sc, MPI_Datatype st, void *r, int rc, MPI_Datatype rt, MPI_Comm c)
{
    (void)rc;
    (void)rt;
    (void)c;
    if (s != r) memcpy(r, s, (size_t)sc * (size_t)st);
    return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm c)
{
    (void)c;
    return MPI_SUCCESS;
}
static inline int MPI_Issend(const void *b, int n, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request *q)
{
    (void)b; (void)n; (void)t; (void)dst; (void)tag; (void)c; (void)q;
    fprintf(stderr, "mpi shim: point-to-point send reached in a single-rank build\n");
    abort();
}
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *q)
{
    (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c; (void)q;
    fprintf(stderr, "mpi shim: point-to-point receive reached in a single-rank build\n");
    abort();
}
static inline int MPI_Wait(MPI_Request *q, MPI_Status *st)
{
    (void)st;
    if (q) *q = MPI_REQUEST_NULL;
    return MPI_SUCCESS;
}
static inline double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#endif
