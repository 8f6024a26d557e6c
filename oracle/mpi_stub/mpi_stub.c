/*
 * Single-rank MPI stand-in (see mpi.h).  TEST INFRASTRUCTURE ONLY.
 *
 * Self-messages: MPI_Isend records (buffer, bytes) under its tag; the
 * matching MPI_Irecv copies it out.  If the receive is posted first, the
 * copy happens when the send arrives.  All requests complete at post time,
 * so MPI_Waitall has nothing to wait for.
 */
#include <stdlib.h>
#include <string.h>

#include "mpi.h"

#ifdef MPI_STUB_CUDA
#include <cuda_runtime_api.h>
static void stub_copy(void *dst, const void *src, size_t n)
{
	cudaMemcpy(dst, src, n, cudaMemcpyDefault);
}
#else
static void stub_copy(void *dst, const void *src, size_t n)
{
	memcpy(dst, src, n);
}
#endif

#define STUB_SLOTS 4096

static struct slot {
	const void *sbuf;
	void *rbuf;
	size_t bytes;
	int has_send, has_recv;
} SLOTS[STUB_SLOTS];

static int INITIALIZED;

static size_t dt_size(MPI_Datatype dt)
{
	return dt == MPI_DOUBLE ? sizeof(double) : 1;
}

int MPI_Init(int *argc, char ***argv)
{
	(void)argc;
	(void)argv;
	INITIALIZED = 1;
	return MPI_SUCCESS;
}

int MPI_Initialized(int *flag)
{
	*flag = INITIALIZED;
	return MPI_SUCCESS;
}

int MPI_Finalize(void)
{
	INITIALIZED = 0;
	return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
	(void)comm;
	*size = 1;
	return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
	(void)comm;
	*rank = 0;
	return MPI_SUCCESS;
}

int MPI_Comm_split_type(MPI_Comm comm, int split_type, int key,
	MPI_Info info, MPI_Comm *newcomm)
{
	(void)split_type;
	(void)key;
	(void)info;
	*newcomm = comm;
	return MPI_SUCCESS;
}

int MPI_Comm_free(MPI_Comm *comm)
{
	(void)comm;
	return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm comm)
{
	(void)comm;
	return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm)
{
	(void)buf;
	(void)count;
	(void)dt;
	(void)root;
	(void)comm;
	return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
	MPI_Datatype dt, MPI_Op op, MPI_Comm comm)
{
	(void)op;
	(void)comm;
	if (sendbuf != MPI_IN_PLACE)
		memcpy(recvbuf, sendbuf, (size_t)count * dt_size(dt));
	return MPI_SUCCESS;
}

static void try_complete(struct slot *s)
{
	if (s->has_send && s->has_recv) {
		stub_copy(s->rbuf, s->sbuf, s->bytes);
		memset(s, 0, sizeof *s);
	}
}

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest,
	int tag, MPI_Comm comm, MPI_Request *req)
{
	(void)dest;
	(void)comm;
	struct slot *s = &SLOTS[(unsigned)tag % STUB_SLOTS];
	s->sbuf = buf;
	s->bytes = (size_t)count * dt_size(dt);
	s->has_send = 1;
	try_complete(s);
	*req = 0;
	return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag,
	MPI_Comm comm, MPI_Request *req)
{
	(void)source;
	(void)comm;
	struct slot *s = &SLOTS[(unsigned)tag % STUB_SLOTS];
	s->rbuf = buf;
	s->bytes = (size_t)count * dt_size(dt);
	s->has_recv = 1;
	try_complete(s);
	*req = 0;
	return MPI_SUCCESS;
}

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
	(void)count;
	(void)reqs;
	(void)statuses;
	return MPI_SUCCESS;
}
