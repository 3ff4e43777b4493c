/* Single-rank MPI stand-in (see mpi.h): test infrastructure only. */
#include "mpi.h"
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static int type_sizes[4096] = {0, 1, 4, 8, 4, 8, 8, 8, 1, 4};
static int n_types = 10;

static size_t tsize(MPI_Datatype t)
{
    if (t < 0 || t >= n_types) { fprintf(stderr, "mpi shim: bad datatype %d\n", t); abort(); }
    return (size_t)type_sizes[t];
}
static void copy(void *r, const void *s, size_t bytes)
{
    if (s == MPI_IN_PLACE || s == r || bytes == 0) return;
    memmove(r, s, bytes);
}
static int no_peer(const char *what, int peer)
{
    fprintf(stderr, "mpi shim: %s with peer %d in a one-rank run\n", what, peer);
    abort();
    return 1;
}
int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm c, int code) { (void)c; fprintf(stderr, "MPI_Abort(%d)\n", code); exit(code ? code : 1); }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out) { (void)color; (void)key; *out = c; return 0; }
int MPI_Comm_split_type(MPI_Comm c, int type, int key, MPI_Info info, MPI_Comm *out)
{ (void)type; (void)key; (void)info; *out = c; return 0; }
int MPI_Comm_free(MPI_Comm *c) { (void)c; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
int MPI_Type_size(MPI_Datatype t, int *size) { *size = (int)tsize(t); return 0; }
int MPI_Type_create_struct(int n, const int *lens, const MPI_Aint *disp, const MPI_Datatype *types, MPI_Datatype *out)
{
    size_t end = 0;
    for (int i = 0; i < n; i++) {
        size_t e = (size_t)disp[i] + (size_t)lens[i] * tsize(types[i]);
        if (e > end) end = e;
    }
    type_sizes[n_types] = (int)end;
    *out = n_types++;
    return 0;
}
int MPI_Type_commit(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Type_free(MPI_Datatype *t) { (void)t; return 0; }
int MPI_Get_address(const void *p, MPI_Aint *a) { *a = (MPI_Aint)p; return 0; }
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{ (void)op; (void)c; copy(r, s, n * tsize(t)); return 0; }
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{ (void)op; (void)root; (void)c; copy(r, s, n * tsize(t)); return 0; }
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c) { (void)b; (void)n; (void)t; (void)root; (void)c; return 0; }
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void)rn; (void)rt; (void)c; copy(r, s, sn * tsize(st)); return 0; }
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c)
{ (void)rn; (void)rt; (void)root; (void)c; copy(r, s, sn * tsize(st)); return 0; }
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt,
                   MPI_Comm c)
{
    (void)c;
    if (s == MPI_IN_PLACE) return 0;
    copy((char *)r + (size_t)rd[0] * tsize(rt), s, (size_t)(sn < rc[0] ? sn : rc[0]) * tsize(st));
    return 0;
}
int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt,
                int root, MPI_Comm c)
{ (void)root; return MPI_Allgatherv(s, sn, st, r, rc, rd, rt, c); }
int MPI_Scatterv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                 int root, MPI_Comm c)
{
    (void)root; (void)c; (void)rn;
    if (r == MPI_IN_PLACE) return 0;
    copy(r, (const char *)s + (size_t)sd[0] * tsize(st), (size_t)sc[0] * tsize(rt));
    return 0;
}
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c)
{ (void)rn; (void)rt; (void)c; copy(r, s, sn * tsize(st)); return 0; }
int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, const int *rc,
                  const int *rd, MPI_Datatype rt, MPI_Comm c)
{
    (void)rc; (void)c;
    copy((char *)r + (size_t)rd[0] * tsize(rt), (const char *)s + (size_t)sd[0] * tsize(st), (size_t)sc[0] * tsize(st));
    return 0;
}
int MPI_Sendrecv(const void *s, int sn, MPI_Datatype st, int dest, int stag, void *r, int rn, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm c, MPI_Status *status)
{
    (void)stag; (void)rtag; (void)c; (void)rn; (void)rt;
    if (dest != 0 || src != 0) return no_peer("MPI_Sendrecv", dest);
    copy(r, s, sn * tsize(st));
    if (status) { status->MPI_SOURCE = 0; status->MPI_TAG = rtag; status->count = sn * (int)tsize(st); }
    return 0;
}
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)tag; (void)c; return no_peer("MPI_Send", dest); }
int MPI_Ssend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{ (void)b; (void)n; (void)t; (void)tag; (void)c; return no_peer("MPI_Ssend", dest); }
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{ (void)b; (void)n; (void)t; (void)tag; (void)c; (void)st; return no_peer("MPI_Recv", src); }
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq)
{ (void)b; (void)n; (void)t; (void)tag; (void)c; (void)rq; return no_peer("MPI_Isend", dest); }
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *rq)
{ (void)b; (void)n; (void)t; (void)tag; (void)c; (void)rq; return no_peer("MPI_Irecv", src); }
int MPI_Waitall(int n, MPI_Request *rq, MPI_Status *st) { (void)n; (void)rq; (void)st; return 0; }
int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st) { (void)tag; (void)c; (void)st; return no_peer("MPI_Probe", src); }
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) { *count = st ? st->count / (int)tsize(t) : 0; return 0; }
