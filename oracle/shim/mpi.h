/*
 * Single-rank MPI shim used only to compile the reference's own C++ sources
 * as a CPU oracle (test infrastructure; never linked into the product).
 *
 * With one rank every partition is local, so the reference's point-to-point
 * fetch path (engine.cc:297-616) never sends.  Collectives degenerate to
 * copies, one-sided windows to plain memory, Fetch_and_op to an atomic add
 * on the local window (engine.cc:1471, 1528) and MPI_Get to memcpy
 * (engine.cc:1543-1562).  Receives never complete (the handler thread in
 * engine.cc:539-548 spins on MPI_Test until it is told to terminate).
 */
#ifndef KHZ_ORACLE_MPI_SHIM_H
#define KHZ_ORACLE_MPI_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE; int MPI_TAG; int MPI_ERROR; } MPI_Status;
typedef struct khz_shim_win { char *base; long size; int disp_unit; } *MPI_Win;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_THREAD_MULTIPLE 3
#define MPI_INFO_NULL 0
#define MPI_LOCK_SHARED 1
#define MPI_LOCK_EXCLUSIVE 2
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_MAX_PROCESSOR_NAME 256
#define MPI_STATUS_IGNORE ((MPI_Status *)0)

/* datatype = (kind << 8) | byte size */
#define MPI_CHAR ((1 << 8) | 1)
#define MPI_UNSIGNED_CHAR ((2 << 8) | 1)
#define MPI_INT ((3 << 8) | 4)
#define MPI_UNSIGNED ((4 << 8) | 4)
#define MPI_LONG ((5 << 8) | 8)
#define MPI_UNSIGNED_LONG ((6 << 8) | 8)
#define MPI_LONG_LONG_INT ((7 << 8) | 8)
#define MPI_FLOAT ((8 << 8) | 4)
#define MPI_DOUBLE ((9 << 8) | 8)

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline int khz_shim_tsize(MPI_Datatype t) { return t & 0xff; }

static inline int MPI_Init_thread(int *argc, char ***argv, int required, int *provided) {
    (void)argc; (void)argv; *provided = required; return MPI_SUCCESS;
}
static inline int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Get_processor_name(char *name, int *len) {
    if (gethostname(name, 127) != 0) strcpy(name, "localhost");
    name[127] = 0; *len = (int)strlen(name); return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)root; (void)c; return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c; if (s != r) memmove(r, s, (size_t)n * khz_shim_tsize(t)); return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c) {
    (void)rn; (void)rt; (void)c; memmove(r, s, (size_t)sn * khz_shim_tsize(st)); return MPI_SUCCESS;
}
static inline void khz_shim_unexpected(const char *what) {
    fprintf(stderr, "single-rank MPI shim: unexpected %s\n", what); abort();
}
static inline int MPI_Send(const void *b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)d; (void)tag; (void)c; khz_shim_unexpected("MPI_Send"); return 1;
}
static inline int MPI_Recv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status *st) {
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; (void)st; khz_shim_unexpected("MPI_Recv"); return 1;
}
static inline int MPI_Irecv(void *b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Request *rq) {
    (void)b; (void)n; (void)t; (void)s; (void)tag; (void)c; *rq = 0; return MPI_SUCCESS;
}
static inline int MPI_Test(MPI_Request *rq, int *flag, MPI_Status *st) {
    (void)rq; (void)st; *flag = 0; usleep(1000); return MPI_SUCCESS;
}
static inline int MPI_Win_create(void *base, MPI_Aint size, int disp_unit, MPI_Info info, MPI_Comm c, MPI_Win *w) {
    (void)info; (void)c;
    *w = (MPI_Win)malloc(sizeof(struct khz_shim_win));
    (*w)->base = (char *)base; (*w)->size = (long)size; (*w)->disp_unit = disp_unit;
    return MPI_SUCCESS;
}
static inline int MPI_Win_free(MPI_Win *w) { free(*w); *w = 0; return MPI_SUCCESS; }
static inline int MPI_Win_lock(int type, int rank, int assert_, MPI_Win w) {
    (void)type; (void)rank; (void)assert_; (void)w; return MPI_SUCCESS;
}
static inline int MPI_Win_unlock(int rank, MPI_Win w) { (void)rank; (void)w; return MPI_SUCCESS; }
static inline int MPI_Win_flush(int rank, MPI_Win w) { (void)rank; (void)w; return MPI_SUCCESS; }
static inline int MPI_Fetch_and_op(const void *origin, void *result, MPI_Datatype t, int rank,
                                   MPI_Aint disp, MPI_Op op, MPI_Win w) {
    (void)rank;
    char *target = w->base + disp * w->disp_unit;
    if (op != MPI_SUM) khz_shim_unexpected("MPI_Fetch_and_op op");
    if (khz_shim_tsize(t) == 4) {
        *(unsigned *)result = __sync_fetch_and_add((unsigned *)target, *(const unsigned *)origin);
    } else if (khz_shim_tsize(t) == 8) {
        *(unsigned long *)result = __sync_fetch_and_add((unsigned long *)target, *(const unsigned long *)origin);
    } else {
        khz_shim_unexpected("MPI_Fetch_and_op size");
    }
    return MPI_SUCCESS;
}
static inline int MPI_Get(void *origin, int on, MPI_Datatype ot, int rank, MPI_Aint disp, int tn,
                          MPI_Datatype tt, MPI_Win w) {
    (void)rank; (void)tn; (void)tt;
    memcpy(origin, w->base + disp * w->disp_unit, (size_t)on * khz_shim_tsize(ot));
    return MPI_SUCCESS;
}
static inline int MPI_Put(const void *origin, int on, MPI_Datatype ot, int rank, MPI_Aint disp, int tn,
                          MPI_Datatype tt, MPI_Win w) {
    (void)origin; (void)on; (void)ot; (void)rank; (void)disp; (void)tn; (void)tt; (void)w;
    khz_shim_unexpected("MPI_Put"); return 1;
}

#endif
