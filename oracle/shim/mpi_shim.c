/*
 * Single-rank MPI stand-in for the test oracle (see mpi.h for semantics).
 * Test infrastructure only.
 */
#include "mpi.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

static size_t type_size(MPI_Datatype t)
{
    switch (t) {
    case MPI_CHAR: case MPI_BYTE: return 1;
    case MPI_INT: return sizeof(int);
    case MPI_FLOAT: return sizeof(float);
    case MPI_DOUBLE: return sizeof(double);
    case MPI_LONG: return sizeof(long);
    default: return 1;
    }
}

/* FIFO of self-messages: MPI_Bsend enqueues, MPI_Recv dequeues in order. */
typedef struct msg { struct msg *next; size_t n; unsigned char data[]; } msg;
static msg *q_head = NULL, *q_tail = NULL;

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return MPI_SUCCESS; }
int MPI_Finalize(void) { return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm c, int *rank) { (void)c; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm c, int *size) { (void)c; *size = 1; return MPI_SUCCESS; }
double MPI_Wtime(void) { struct timeval tv; gettimeofday(&tv, NULL); return tv.tv_sec + 1e-6 * tv.tv_usec; }
int MPI_Abort(MPI_Comm c, int code) { (void)c; fprintf(stderr, "oracle MPI_Abort(%d)\n", code); exit(code ? code : 1); }
int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
int MPI_Bcast(void *buf, int count, MPI_Datatype t, int root, MPI_Comm c)
{ (void)buf; (void)count; (void)t; (void)root; (void)c; return MPI_SUCCESS; }

int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, MPI_Comm c)
{
    (void)op; (void)c;
    if (sbuf != rbuf) memmove(rbuf, sbuf, (size_t)count * type_size(t));
    return MPI_SUCCESS;
}

int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c)
{ (void)root; return MPI_Allreduce(sbuf, rbuf, count, t, op, c); }

int MPI_Bsend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{
    (void)dest; (void)tag; (void)c;
    size_t n = (size_t)count * type_size(t);
    msg *m = (msg *)malloc(sizeof(msg) + n);
    if (!m) { fprintf(stderr, "oracle MPI shim: out of memory\n"); exit(1); }
    m->next = NULL; m->n = n;
    memcpy(m->data, buf, n);
    if (q_tail) q_tail->next = m; else q_head = m;
    q_tail = m;
    return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c)
{ return MPI_Bsend(buf, count, t, dest, tag, c); }

int MPI_Recv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status *st)
{
    (void)src; (void)tag; (void)c;
    msg *m = q_head;
    if (!m) { fprintf(stderr, "oracle MPI shim: MPI_Recv with empty self-queue\n"); exit(1); }
    q_head = m->next;
    if (!q_head) q_tail = NULL;
    size_t n = (size_t)count * type_size(t);
    memcpy(buf, m->data, n < m->n ? n : m->n);
    free(m);
    if (st) { st->MPI_SOURCE = 0; st->MPI_TAG = tag; st->MPI_ERROR = 0; }
    return MPI_SUCCESS;
}

int MPI_Sendrecv_replace(void *buf, int count, MPI_Datatype t, int dest, int stag, int src, int rtag,
                         MPI_Comm c, MPI_Status *st)
{ (void)buf; (void)count; (void)t; (void)dest; (void)stag; (void)src; (void)rtag; (void)c; (void)st; return MPI_SUCCESS; }

int MPI_Buffer_attach(void *buf, int size) { (void)buf; (void)size; return MPI_SUCCESS; }
int MPI_Buffer_detach(void *buf, int *size) { (void)buf; if (size) *size = 0; return MPI_SUCCESS; }
int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *r)
{ if (r) *r = 0; return MPI_Bsend(buf, count, t, dest, tag, c); }
int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *r)
{ if (r) *r = 0; return MPI_Recv(buf, count, t, src, tag, c, NULL); }
int MPI_Wait(MPI_Request *r, MPI_Status *st) { (void)r; (void)st; return MPI_SUCCESS; }
int MPI_Waitall(int n, MPI_Request *r, MPI_Status *st) { (void)n; (void)r; (void)st; return MPI_SUCCESS; }
int MPI_Send_init(const void *buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request *r)
{ (void)buf; (void)count; (void)t; (void)dest; (void)tag; (void)c; if (r) *r = 0; return MPI_SUCCESS; }
int MPI_Recv_init(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *r)
{ (void)buf; (void)count; (void)t; (void)src; (void)tag; (void)c; if (r) *r = 0; return MPI_SUCCESS; }
int MPI_Startall(int n, MPI_Request *r) { (void)n; (void)r; return MPI_SUCCESS; }
int MPI_Request_free(MPI_Request *r) { (void)r; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm *out) { (void)color; (void)key; *out = c; return MPI_SUCCESS; }
