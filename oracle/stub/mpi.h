/*
 * Single-rank MPI stand-in used ONLY to compile the reference's force-path
 * sources (Cosmos/pmmain.c, Cosmos/psolver.c, Cosmos/fda4.c,
 * Cosmos/treecorrection.c, Cosmos/BasicCell.c, OST/ost.ver2.c,
 * OST/Model4TreeForce.c) into the CPU oracle library under oracle/_ref.
 *
 * This is test infrastructure: with one rank every collective the force path
 * makes (MPI_Reduce/MPI_Bcast of scalars, MPI_Barrier) is a copy or a no-op.
 * The definitions live in oracle/ref_shim.c.
 */
#ifndef ORACLE_STUB_MPI_H
#define ORACLE_STUB_MPI_H
#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;
typedef int MPI_Request;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_SUCCESS 0

#define MPI_CHAR 1
#define MPI_BYTE 2
#define MPI_INT 4
#define MPI_LONG 8
#define MPI_LONG_LONG 9
#define MPI_FLOAT 14
#define MPI_DOUBLE 18
#define MPI_UNSIGNED_LONG 28
#define MPI_INT64_T 38

#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3

#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_THREAD_FUNNELED 1

int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Bcast(void *b, int n, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Barrier(MPI_Comm c);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int *r);
int MPI_Comm_size(MPI_Comm c, int *s);
int MPI_Sendrecv(const void *sb, int sc, MPI_Datatype st, int dest, int stag,
                 void *rb, int rc, MPI_Datatype rt, int src, int rtag,
                 MPI_Comm c, MPI_Status *status);
int MPI_Send(const void *b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *s);
int MPI_Get_count(const MPI_Status *s, MPI_Datatype t, int *n);
double MPI_Wtime(void);

#endif
