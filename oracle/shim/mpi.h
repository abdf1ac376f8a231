/*
 * Single-rank MPI stand-in used only to compile the reference's CPU sources
 * as a test oracle (oracle/_ref).  It is test infrastructure: nothing in the
 * product library includes it.
 *
 * Semantics (one process, rank 0 of size 1):
 *   - point-to-point messages to self go through a FIFO: MPI_Bsend/MPI_Send
 *     enqueue a copy, MPI_Recv dequeues it.  The reference's matcopy() relies
 *     on this on one rank: its self-Bsend/Recv wraps the model periodically
 *     (matcopy_elastic.c:57-60 in the reference); a no-op shim would leave
 *     zeros in the model halo instead.
 *   - MPI_Sendrecv_replace to self is the identity.
 *   - collectives on one rank copy the send buffer to the receive buffer.
 */
#ifndef DSH_ORACLE_MPI_SHIM_H
#define DSH_ORACLE_MPI_SHIM_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_PROC_NULL (-2)
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_BSEND_OVERHEAD 64

#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_FLOAT 3
#define MPI_DOUBLE 4
#define MPI_LONG 5
#define MPI_BYTE 6

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

int MPI_Init(int *argc, char ***argv);
int MPI_Finalize(void);
int MPI_Comm_rank(MPI_Comm c, int *rank);
int MPI_Comm_size(MPI_Comm c, int *size);
double MPI_Wtime(void);
int MPI_Abort(MPI_Comm c, int code);
int MPI_Barrier(MPI_Comm c);
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c);
int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c);
int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c);
int MPI_Bsend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c);
int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st);
int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype t, int dest, int stag, int src, int rtag,
                         MPI_Comm c, MPI_Status *st);
int MPI_Buffer_attach(void *buf, int size);
int MPI_Buffer_detach(void *buf, int *size);
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Wait(MPI_Request *r, MPI_Status *st);
int MPI_Waitall(int n, MPI_Request *r, MPI_Status *st);
int MPI_Send_init(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Recv_init(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *r);
int MPI_Startall(int n, MPI_Request *r);
int MPI_Request_free(MPI_Request *r);
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out);

#endif
