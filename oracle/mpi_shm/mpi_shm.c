/*
 * mpi_shm.c -- multi-rank shared-memory stand-in for the subset of MPI that
 * the phase2 CPU path calls (TEST INFRASTRUCTURE ONLY: it lets the
 * reference's CPU path, compiled unmodified, run as R ranks on one host's
 * cores for the CPU baseline; it is never linked into the product).
 *
 * The header is oracle/mpi_stub/mpi.h (the same declarations as the
 * single-rank stand-in) plus mpi_shm_spawn below.
 *
 * Ranks are processes: mpi_shm_spawn(R) maps one shared control block,
 * forks R - 1 children and returns each process's rank; MPI_Init then only
 * marks the library initialised.  Without a spawn the job has one rank.
 *
 *   Barrier     sense-reversing counter in the shared block
 *   Bcast       root writes a shared slot, barrier, the others read, barrier
 *   Allreduce   (MPI_SUM of doubles) every rank writes its row, barrier,
 *               every rank sums the rows in rank order (the same bits on
 *               every rank), barrier
 *   Isend       publishes (address, size, destination, tag) in the
 *               sender's message table; with shared mailboxes the data is
 *               copied into the sender's mailbox at once
 *   Irecv       is recorded locally
 *   Waitall     completes requests and makes progress on this rank's
 *               posted receives meanwhile: a receive finds the matching
 *               published message (source, destination, tag) and copies it
 *               straight out of the sender's memory (process_vm_readv, one
 *               copy, as a single-copy MPI transport on one node does) or
 *               out of the sender's mailbox where the kernel refuses
 *               cross-process reads; a send completes when its receiver
 *               has consumed it.  Progress inside the send wait is what
 *               lets two ranks that both wait on their sends before their
 *               receives (phase2/qreg_qreg.c:97-101) finish.
 *
 * Every wait gives up after MPI_SHM_WAIT_S seconds and aborts the job, so a
 * mismatched exchange ends the run instead of hanging it.
 */
#define _GNU_SOURCE

#include <errno.h>
#include <sched.h>
#include <signal.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/prctl.h>
#include <sys/types.h>
#include <sys/uio.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#include "mpi.h"

#define MPI_SHM_MAX_RANKS 256
#define MPI_SHM_MAX_MSGS 64
#define MPI_SHM_MAX_SCALARS 16
#define MPI_SHM_WAIT_S 1200.0

enum { MSG_FREE = 0, MSG_PUBLISHED = 1, MSG_CONSUMED = 2 };

struct shm_msg {
	_Atomic int state;
	int dest, tag;
	uint64_t addr;   /* sender's buffer (single-copy transport) */
	size_t bytes;
	size_t mbox_off; /* offset in the sender's mailbox (mailbox mode) */
};

struct shm_rank {
	pid_t pid;
	struct shm_msg msg[MPI_SHM_MAX_MSGS];
	double red[MPI_SHM_MAX_SCALARS];
	_Atomic int cma_ok;
};

struct shm_ctl {
	int size;
	int mailbox;         /* 1: copies go through per-rank mailboxes */
	size_t mbox_bytes;   /* per rank */
	_Atomic int bar_count;
	_Atomic int bar_sense;
	double bcast[MPI_SHM_MAX_SCALARS];
	struct shm_rank r[MPI_SHM_MAX_RANKS];
};

static struct shm_ctl *CTL;
static unsigned char *MBOX; /* size * mbox_bytes, after the control block */
static int RANK, SIZE = 1, INITIALIZED, SENSE;
static size_t MBOX_USED;

/* posted requests of this rank */
#define MPI_SHM_MAX_REQS 256
static struct req {
	int live, is_send, done;
	int peer, tag;
	void *buf;
	size_t bytes;
	int slot; /* send: message slot in this rank's table */
} REQS[MPI_SHM_MAX_REQS];

static double now_s(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static void die(const char *what)
{
	fprintf(stderr, "mpi_shm rank %d: %s\n", RANK, what);
	fflush(stderr);
	if (CTL)
		for (int k = 0; k < SIZE; k++)
			if (k != RANK && CTL->r[k].pid > 0)
				kill(CTL->r[k].pid, SIGTERM);
	_exit(3);
}

/* one round of a wait loop: spin briefly, then yield the core */
static void relax(unsigned *spins, double t0)
{
	if (++*spins < 256)
		return;
	*spins = 0;
	sched_yield();
	if (now_s() - t0 > MPI_SHM_WAIT_S)
		die("wait limit reached (mismatched exchange?)");
}

static size_t dt_size(MPI_Datatype dt)
{
	return dt == MPI_DOUBLE ? sizeof(double) : 1;
}

int mpi_shm_spawn(int ranks, size_t mbox_bytes)
{
	if (ranks < 1 || ranks > MPI_SHM_MAX_RANKS)
		return -1;
	const size_t ctl_bytes = (sizeof(struct shm_ctl) + 4095) & ~(size_t)4095;
	void *p = mmap(NULL, ctl_bytes, PROT_READ | PROT_WRITE,
		MAP_SHARED | MAP_ANONYMOUS, -1, 0);
	if (p == MAP_FAILED)
		return -1;
	CTL = (struct shm_ctl *)p;
	memset(CTL, 0, sizeof *CTL);
	CTL->size = ranks;
	CTL->mbox_bytes = mbox_bytes;
	if (mbox_bytes) {
		/* reserved before the fork so that every rank shares it; pages
		 * are only backed once a mailbox copy touches them */
		void *m = mmap(NULL, (size_t)ranks * mbox_bytes,
			PROT_READ | PROT_WRITE,
			MAP_SHARED | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
		if (m == MAP_FAILED)
			return -1;
		MBOX = (unsigned char *)m;
	}
	SIZE = ranks;
	RANK = 0;
	CTL->r[0].pid = getpid();
	for (int k = 1; k < ranks; k++) {
		const pid_t pid = fork();
		if (pid < 0)
			die("fork failed");
		if (pid == 0) {
			RANK = k;
			CTL->r[k].pid = getpid();
			prctl(PR_SET_PDEATHSIG, SIGTERM);
			break;
		}
		CTL->r[k].pid = pid;
	}
	/* allow the other ranks to read this process's memory (Yama) */
	prctl(PR_SET_PTRACER, PR_SET_PTRACER_ANY, 0, 0, 0);
	MPI_Barrier(MPI_COMM_WORLD);
	/* single-copy transport if every rank can read its neighbour */
	static const uint64_t probe = UINT64_C(0x6d70695f73686d21);
	const int nb = (RANK + 1) % SIZE;
	uint64_t got = 0;
	struct iovec li = { &got, sizeof got };
	struct iovec ri = { (void *)&probe, sizeof probe };
	atomic_store(&CTL->r[RANK].cma_ok,
		process_vm_readv(CTL->r[nb].pid, &li, 1, &ri, 1, 0) ==
				(ssize_t)sizeof got &&
			got == probe);
	MPI_Barrier(MPI_COMM_WORLD);
	int all = 1;
	for (int k = 0; k < SIZE; k++)
		all &= atomic_load(&CTL->r[k].cma_ok);
	MPI_Barrier(MPI_COMM_WORLD);
	if (RANK == 0)
		CTL->mailbox = !all || getenv("MPI_SHM_MAILBOX") != NULL;
	MPI_Barrier(MPI_COMM_WORLD);
	if (CTL->mailbox && !MBOX)
		die("no single-copy transport and no mailbox size");
	return RANK;
}

int mpi_shm_mailbox(void)
{
	return CTL ? CTL->mailbox : 0;
}

/* The parent waits for its children (rank 0 after the run); children
 * never return from here. */
int mpi_shm_join(int status)
{
	if (!CTL || SIZE == 1)
		return status;
	if (RANK != 0)
		_exit(status);
	int worst = status;
	for (int k = 1; k < SIZE; k++) {
		int st = 0;
		if (waitpid(CTL->r[k].pid, &st, 0) < 0 || !WIFEXITED(st) ||
			WEXITSTATUS(st) != 0)
			worst = worst ? worst : 1;
	}
	return worst;
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
	MPI_Barrier(MPI_COMM_WORLD);
	INITIALIZED = 0;
	return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
	(void)comm;
	*size = SIZE;
	return MPI_SUCCESS;
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
	(void)comm;
	*rank = RANK;
	return MPI_SUCCESS;
}

int MPI_Comm_split_type(MPI_Comm comm, int split_type, int key,
	MPI_Info info, MPI_Comm *newcomm)
{
	(void)split_type;
	(void)key;
	(void)info;
	*newcomm = comm; /* every rank is on this node */
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
	if (SIZE == 1)
		return MPI_SUCCESS;
	SENSE = !SENSE;
	if (atomic_fetch_add(&CTL->bar_count, 1) == SIZE - 1) {
		atomic_store(&CTL->bar_count, 0);
		atomic_store(&CTL->bar_sense, SENSE);
	} else {
		unsigned spins = 0;
		const double t0 = now_s();
		while (atomic_load(&CTL->bar_sense) != SENSE)
			relax(&spins, t0);
	}
	return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm comm)
{
	const size_t bytes = (size_t)count * dt_size(dt);
	if (SIZE == 1)
		return MPI_SUCCESS;
	if (bytes > sizeof CTL->bcast)
		die("Bcast larger than the shared slot");
	if (RANK == root)
		memcpy(CTL->bcast, buf, bytes);
	MPI_Barrier(comm);
	if (RANK != root)
		memcpy(buf, CTL->bcast, bytes);
	MPI_Barrier(comm);
	return MPI_SUCCESS;
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count,
	MPI_Datatype dt, MPI_Op op, MPI_Comm comm)
{
	(void)op; /* MPI_SUM is the only reduction the path uses */
	if (dt != MPI_DOUBLE || count > MPI_SHM_MAX_SCALARS)
		die("Allreduce of an unsupported type or size");
	const double *src =
		sendbuf == MPI_IN_PLACE ? (const double *)recvbuf : sendbuf;
	if (SIZE == 1) {
		if (sendbuf != MPI_IN_PLACE)
			memcpy(recvbuf, sendbuf, (size_t)count * sizeof(double));
		return MPI_SUCCESS;
	}
	memcpy(CTL->r[RANK].red, src, (size_t)count * sizeof(double));
	MPI_Barrier(comm);
	double *out = recvbuf;
	for (int i = 0; i < count; i++) {
		double s = 0.0;
		for (int k = 0; k < SIZE; k++)
			s += CTL->r[k].red[i];
		out[i] = s;
	}
	MPI_Barrier(comm);
	return MPI_SUCCESS;
}

static int new_req(void)
{
	for (int i = 0; i < MPI_SHM_MAX_REQS; i++)
		if (!REQS[i].live) {
			memset(&REQS[i], 0, sizeof REQS[i]);
			REQS[i].live = 1;
			return i;
		}
	die("too many outstanding requests");
	return -1;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest,
	int tag, MPI_Comm comm, MPI_Request *req)
{
	(void)comm;
	const size_t bytes = (size_t)count * dt_size(dt);
	struct shm_rank *me = &CTL->r[RANK];
	int slot = -1;
	for (int i = 0; i < MPI_SHM_MAX_MSGS && slot < 0; i++)
		if (atomic_load(&me->msg[i].state) == MSG_FREE)
			slot = i;
	if (slot < 0)
		die("message table full");
	struct shm_msg *m = &me->msg[slot];
	m->dest = dest;
	m->tag = tag;
	m->addr = (uint64_t)(uintptr_t)buf;
	m->bytes = bytes;
	if (CTL->mailbox) {
		if (MBOX_USED + bytes > CTL->mbox_bytes)
			die("mailbox overflow");
		m->mbox_off = MBOX_USED;
		memcpy(MBOX + (size_t)RANK * CTL->mbox_bytes + MBOX_USED, buf,
			bytes);
		MBOX_USED += bytes;
	}
	atomic_store_explicit(&m->state, MSG_PUBLISHED, memory_order_release);
	const int r = new_req();
	REQS[r].is_send = 1;
	REQS[r].peer = dest;
	REQS[r].tag = tag;
	REQS[r].slot = slot;
	*req = r;
	return MPI_SUCCESS;
}

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag,
	MPI_Comm comm, MPI_Request *req)
{
	(void)comm;
	const int r = new_req();
	REQS[r].peer = source;
	REQS[r].tag = tag;
	REQS[r].buf = buf;
	REQS[r].bytes = (size_t)count * dt_size(dt);
	*req = r;
	return MPI_SUCCESS;
}

static void copy_from(int src, const struct shm_msg *m, void *dst)
{
	if (src == RANK) {
		memcpy(dst, (const void *)(uintptr_t)m->addr, m->bytes);
		return;
	}
	if (CTL->mailbox) {
		memcpy(dst, MBOX + (size_t)src * CTL->mbox_bytes + m->mbox_off,
			m->bytes);
		return;
	}
	size_t done = 0;
	while (done < m->bytes) {
		struct iovec li = { (char *)dst + done, m->bytes - done };
		struct iovec ri = { (void *)(uintptr_t)(m->addr + done),
			m->bytes - done };
		const ssize_t n =
			process_vm_readv(CTL->r[src].pid, &li, 1, &ri, 1, 0);
		if (n <= 0)
			die("process_vm_readv failed");
		done += (size_t)n;
	}
}

/* Complete every posted receive whose message has been published. */
static void progress(void)
{
	for (int i = 0; i < MPI_SHM_MAX_REQS; i++) {
		struct req *q = &REQS[i];
		if (!q->live || q->is_send || q->done)
			continue;
		struct shm_rank *src = &CTL->r[q->peer];
		for (int s = 0; s < MPI_SHM_MAX_MSGS; s++) {
			struct shm_msg *m = &src->msg[s];
			if (atomic_load_explicit(&m->state,
				    memory_order_acquire) != MSG_PUBLISHED ||
				m->dest != RANK || m->tag != q->tag)
				continue;
			if (m->bytes != q->bytes)
				die("message size mismatch");
			copy_from(q->peer, m, q->buf);
			atomic_store_explicit(&m->state, MSG_CONSUMED,
				memory_order_release);
			q->done = 1;
			break;
		}
	}
}

int MPI_Waitall(int count, MPI_Request *reqs, MPI_Status *statuses)
{
	(void)statuses;
	for (int k = 0; k < count; k++) {
		struct req *q = &REQS[reqs[k]];
		unsigned spins = 0;
		const double t0 = now_s();
		if (q->is_send) {
			struct shm_msg *m = &CTL->r[RANK].msg[q->slot];
			for (;;) {
				progress();
				if (atomic_load_explicit(&m->state,
					    memory_order_acquire) ==
					MSG_CONSUMED)
					break;
				relax(&spins, t0);
			}
			atomic_store(&m->state, MSG_FREE);
		} else {
			for (;;) {
				progress();
				if (q->done)
					break;
				relax(&spins, t0);
			}
		}
		q->live = 0;
	}
	/* the mailbox is reused once every message in it was consumed */
	int busy = 0;
	for (int i = 0; i < MPI_SHM_MAX_MSGS; i++)
		busy |= atomic_load(&CTL->r[RANK].msg[i].state) != MSG_FREE;
	if (!busy)
		MBOX_USED = 0;
	return MPI_SUCCESS;
}
