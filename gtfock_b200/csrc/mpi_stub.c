/*
 * mpi_stub.c -- single-process MPI (see include/mpi_stub/mpi.h).
 *
 * Every communicator has one rank (rank 0).  Collectives copy the send buffer
 * to the receive buffer; a message sent to oneself is parked until the
 * matching receive (the only pattern the reference uses with one rank is
 * MPI_Sendrecv to itself, pscf/purif.c:548-552).
 */
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "mpi.h"

static int g_initialized = 0;
static void *g_parked = NULL;
static size_t g_parked_len = 0;

static size_t type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; g_initialized = 1; return MPI_SUCCESS; }

int MPI_Init_thread(int *argc, char ***argv, int required, int *provided)
{
    (void)argc; (void)argv;
    g_initialized = 1;
    if (provided) *provided = required;
    return MPI_SUCCESS;
}

int MPI_Initialized(int *flag) { *flag = g_initialized; return MPI_SUCCESS; }
int MPI_Finalize(void) { g_initialized = 0; free(g_parked); g_parked = NULL; return MPI_SUCCESS; }
int MPI_Abort(MPI_Comm comm, int code) { (void)comm; exit(code); }
int MPI_Comm_rank(MPI_Comm comm, int *rank) { (void)comm; *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_size(MPI_Comm comm, int *size) { (void)comm; *size = 1; return MPI_SUCCESS; }

int MPI_Comm_split(MPI_Comm comm, int color, int key, MPI_Comm *newcomm)
{
    (void)comm; (void)key;
    *newcomm = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : MPI_COMM_SELF;
    return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }

int MPI_Cart_create(MPI_Comm comm, int ndims, const int *dims, const int *periods,
                    int reorder, MPI_Comm *cart)
{
    (void)comm; (void)ndims; (void)dims; (void)periods; (void)reorder;
    *cart = MPI_COMM_SELF;
    return MPI_SUCCESS;
}

int MPI_Cart_coords(MPI_Comm comm, int rank, int maxdims, int *coords)
{
    (void)comm; (void)rank;
    for (int i = 0; i < maxdims; i++) coords[i] = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_rank(MPI_Comm comm, const int *coords, int *rank)
{
    (void)comm; (void)coords;
    *rank = 0;
    return MPI_SUCCESS;
}

int MPI_Cart_sub(MPI_Comm comm, const int *remain_dims, MPI_Comm *newcomm)
{
    (void)comm; (void)remain_dims;
    *newcomm = MPI_COMM_SELF;
    return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm) { (void)comm; return MPI_SUCCESS; }

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
    (void)buf; (void)count; (void)type; (void)root; (void)comm;
    return MPI_SUCCESS;
}

static void copy_if_needed(const void *s, void *r, size_t n)
{
    if (s != MPI_IN_PLACE && s != r && n > 0) memmove(r, s, n);
}

int MPI_Reduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
               int root, MPI_Comm comm)
{
    (void)op; (void)root; (void)comm;
    copy_if_needed(sbuf, rbuf, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
    (void)op; (void)comm;
    copy_if_needed(sbuf, rbuf, (size_t)count * type_size(type));
    return MPI_SUCCESS;
}

int MPI_Gather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount,
               MPI_Datatype rtype, int root, MPI_Comm comm)
{
    (void)rcount; (void)rtype; (void)root; (void)comm;
    copy_if_needed(sbuf, rbuf, (size_t)scount * type_size(stype));
    return MPI_SUCCESS;
}

int MPI_Allgather(const void *sbuf, int scount, MPI_Datatype stype, void *rbuf, int rcount,
                  MPI_Datatype rtype, MPI_Comm comm)
{
    (void)rcount; (void)rtype; (void)comm;
    copy_if_needed(sbuf, rbuf, (size_t)scount * type_size(stype));
    return MPI_SUCCESS;
}

int MPI_Send(const void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
    (void)dest; (void)tag; (void)comm;
    size_t n = (size_t)count * type_size(type);
    free(g_parked);
    g_parked = malloc(n ? n : 1);
    if (g_parked == NULL) return 1;
    memcpy(g_parked, buf, n);
    g_parked_len = n;
    return MPI_SUCCESS;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm,
             MPI_Status *status)
{
    (void)src; (void)tag; (void)comm;
    size_t n = (size_t)count * type_size(type);
    if (g_parked && n <= g_parked_len) memcpy(buf, g_parked, n);
    if (status) { status->MPI_SOURCE = 0; status->MPI_TAG = tag; status->MPI_ERROR = 0; }
    return MPI_SUCCESS;
}

int MPI_Sendrecv(const void *sbuf, int scount, MPI_Datatype stype, int dest, int stag,
                 void *rbuf, int rcount, MPI_Datatype rtype, int src, int rtag,
                 MPI_Comm comm, MPI_Status *status)
{
    (void)dest; (void)stag; (void)rcount; (void)rtype; (void)src; (void)comm;
    copy_if_needed(sbuf, rbuf, (size_t)scount * type_size(stype));
    if (status) { status->MPI_SOURCE = 0; status->MPI_TAG = rtag; status->MPI_ERROR = 0; }
    return MPI_SUCCESS;
}

double MPI_Wtime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
