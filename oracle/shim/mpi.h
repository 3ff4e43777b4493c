/* Single-rank stand-in for the MPI interface GIZMO compiles against.
 * Test infrastructure for building the reference as a CPU oracle/baseline:
 * one process, rank 0 of 1; collectives copy send buffers to receive
 * buffers; point-to-point messages to another rank cannot occur and abort. */
#ifndef GG_SHIM_MPI_H
#define GG_SHIM_MPI_H
#include <stddef.h>
typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long MPI_Aint;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR, count; } MPI_Status;
#define MPI_COMM_WORLD 0
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL 0
#define MPI_BYTE 1
#define MPI_INT 2
#define MPI_DOUBLE 3
#define MPI_FLOAT 4
#define MPI_LONG 5
#define MPI_LONG_LONG 6
#define MPI_UNSIGNED_LONG_LONG 7
#define MPI_CHAR 8
#define MPI_UNSIGNED 9
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_ANY_TAG (-1)
#define MPI_ANY_SOURCE (-2)
#define MPI_SUCCESS 0
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)
int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm c, int code);
int MPI_Comm_rank(MPI_Comm c, int *r);
int MPI_Comm_size(MPI_Comm c, int *s);
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out);
int MPI_Comm_split_type(MPI_Comm c, int type, int key, MPI_Info info, MPI_Comm *out);
int MPI_Comm_free(MPI_Comm *c);
int MPI_Barrier(MPI_Comm c);
double MPI_Wtime(void);
int MPI_Type_size(MPI_Datatype t, int *size);
int MPI_Type_create_struct(int n, const int *lens, const MPI_Aint *disp, const MPI_Datatype *types, MPI_Datatype *out);
int MPI_Type_commit(MPI_Datatype *t);
int MPI_Type_free(MPI_Datatype *t);
int MPI_Get_address(const void *p, MPI_Aint *a);
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Allgather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Gather(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, int root, MPI_Comm c);
int MPI_Allgatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt,
                   MPI_Comm c);
int MPI_Gatherv(const void *s, int sn, MPI_Datatype st, void *r, const int *rc, const int *rd, MPI_Datatype rt,
                int root, MPI_Comm c);
int MPI_Scatterv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, int rn, MPI_Datatype rt,
                 int root, MPI_Comm c);
int MPI_Alltoall(const void *s, int sn, MPI_Datatype st, void *r, int rn, MPI_Datatype rt, MPI_Comm c);
int MPI_Alltoallv(const void *s, const int *sc, const int *sd, MPI_Datatype st, void *r, const int *rc,
                  const int *rd, MPI_Datatype rt, MPI_Comm c);
int MPI_Sendrecv(const void *s, int sn, MPI_Datatype st, int dest, int stag, void *r, int rn, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm c, MPI_Status *status);
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Ssend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Isend(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *rq);
int MPI_Irecv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *rq);
int MPI_Waitall(int n, MPI_Request *rq, MPI_Status *st);
int MPI_Probe(int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count);
#endif
