/*
 * Single-rank stand-in for the subset of MPI that the phase2 CPU path
 * calls.  TEST INFRASTRUCTURE ONLY: it exists so that the reference
 * sources compile unmodified into oracle/_ref/ (the checker), and is never
 * linked into the product library.
 *
 * Semantics are those of an MPI job with exactly one rank:
 *   - MPI_Comm_size = 1, MPI_Comm_rank = 0;
 *   - Bcast/Barrier are no-ops (the root is the only rank);
 *   - Allreduce copies send -> recv;
 *   - Isend/Irecv to self are matched by tag and completed with a copy.
 * With -DMPI_STUB_CUDA the self-copy goes through cudaMemcpy with
 * cudaMemcpyDefault so that device pointers (CUDA-aware MPI) also work.
 */
#ifndef ORACLE_MPI_STUB_H
#define ORACLE_MPI_STUB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Info;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD ((MPI_Comm)1)
#define MPI_COMM_TYPE_SHARED 1
#define MPI_INFO_NULL ((MPI_Info)0)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_SUM ((MPI_Op)1)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

int MPI_Init(int *argc, char ***argv);
int MPI_Initialized(int *flag);
int MPI_Finalize(void);
int MPI_Comm_size(MPI_Comm comm, int *size);
int MPI_Comm_rank(MPI_Comm comm, int *rank);
int MPI_Comm_split_type(MPI_Comm comm, int split_type, int key,
	MPI_Info info, MPI_Comm *newcomm);
int MPI_Comm_free(MPI_Comm *comm);
int MPI_Barrier(MPI_Comm comm);
int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm);
int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
	MPI_Datatype dt, MPI_Op op, MPI_Comm comm);
int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest,
	int tag, MPI_Comm comm, MPI_Request *req);
int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag,
	MPI_Comm comm, MPI_Request *req);
int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_MPI_STUB_H */
