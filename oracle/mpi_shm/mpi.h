/*
 * Multi-rank shared-memory stand-in for the subset of MPI that the phase2
 * CPU path calls (TEST INFRASTRUCTURE ONLY; mpi_shm.c).  The MPI
 * declarations are those of the single-rank stand-in; the three calls
 * below start and end a job of R ranks on one host.
 */
#ifndef ORACLE_MPI_SHM_H
#define ORACLE_MPI_SHM_H

#include "../mpi_stub/mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Fork R - 1 ranks; returns this process's rank (-1 on failure).
 * mbox_bytes: per-rank mailbox for messages when the host refuses
 * cross-process reads (0: none). */
int mpi_shm_spawn(int ranks, size_t mbox_bytes);

/* 1 when messages go through the shared mailboxes (two copies), 0 for
 * the single-copy transport. */
int mpi_shm_mailbox(void);

/* Rank 0: wait for the other ranks, return the worst status; the other
 * ranks exit with `status`. */
int mpi_shm_join(int status);

#ifdef __cplusplus
}
#endif

#endif /* ORACLE_MPI_SHM_H */
