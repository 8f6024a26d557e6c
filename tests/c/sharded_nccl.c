/*
 * sharded_nccl.c -- a sharded register across GPUs from C, one process per
 * GPU, the transport NCCL (include/phase2_sharded.h).
 *
 * Launch one process per GPU with RANK, WORLD_SIZE and LOCAL_RANK set (for
 * example `torchrun --no-python --nproc-per-node 2 ./sharded_nccl <dir>`;
 * WORLD_SIZE a power of two) and a directory shared by the processes: rank
 * 0 writes the NCCL unique id there, the others wait for it (bounded).
 * Each process holds one rank of a 14-qubit FP64 register and runs
 * first- and second-order Trotter and qDRIFT over NCCL; it also runs the
 * same problems with every rank held in this process (no transport) and
 * compares: the overlaps must agree bit for bit.  Prints "ok" on rank 0
 * and exits 0 on success.
 *
 * Every call of this build has one GPU, and NCCL ranks whose kernels wait
 * on one another must not share one, so this program is compiled by the
 * CPU tests and run only where two or more GPUs are available.
 */
#include <complex.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <cuda_runtime.h>
#include <nccl.h>

#include "phase2.h"
#include "phase2_b200.h"
#include "phase2_sharded.h"

#define NQB 14
#define NTERMS 400
#define STEPS 3
#define SAMPLES 2
#define DEPTH 300

struct nccl_io {
	ncclComm_t comm;
	cudaStream_t stream;
	double *dsum; /* device scratch of the sums */
	size_t nsum;
};

static int xchg(void *ctx, uint32_t rank, uint32_t peer, const void *send,
	void *recv, size_t bytes)
{
	struct nccl_io *c = ctx;
	(void)rank;
	if (ncclGroupStart() != ncclSuccess ||
		ncclSend(send, bytes, ncclUint8, (int)peer, c->comm,
			c->stream) != ncclSuccess ||
		ncclRecv(recv, bytes, ncclUint8, (int)peer, c->comm,
			c->stream) != ncclSuccess ||
		ncclGroupEnd() != ncclSuccess)
		return -1;
	return cudaStreamSynchronize(c->stream) == cudaSuccess ? 0 : -1;
}

static int sum(void *ctx, double *v, size_t n)
{
	struct nccl_io *c = ctx;
	if (n > c->nsum) {
		cudaFree(c->dsum);
		c->dsum = NULL;
		if (cudaMalloc((void **)&c->dsum, n * sizeof *v) != cudaSuccess)
			return -1;
		c->nsum = n;
	}
	if (cudaMemcpy(c->dsum, v, n * sizeof *v, cudaMemcpyHostToDevice) !=
			cudaSuccess ||
		ncclAllReduce(c->dsum, c->dsum, n, ncclDouble, ncclSum, c->comm,
			c->stream) != ncclSuccess ||
		cudaStreamSynchronize(c->stream) != cudaSuccess ||
		cudaMemcpy(v, c->dsum, n * sizeof *v, cudaMemcpyDeviceToHost) !=
			cudaSuccess)
		return -1;
	return 0;
}

static uint64_t mix(uint64_t x)
{
	x ^= x >> 31;
	x *= UINT64_C(0x7fb5d329728ea185);
	x ^= x >> 27;
	x *= UINT64_C(0x81dadef4bc2dd44d);
	x ^= x >> 33;
	return x;
}

static int make_problem(struct circ_hamil *hm, struct circ_muldet *md)
{
	if (circ_hamil_init(hm, NQB, NTERMS) != 0 ||
		circ_muldet_init(md, 2) != 0)
		return -1;
	for (size_t k = 0; k < NTERMS; k++) {
		uint64_t f = 0;
		const uint64_t h = mix(k + 1);
		for (int j = 0; j < (int)(h % 4); j++)
			f |= UINT64_C(1) << (mix(h + j) % NQB);
		hm->terms[k].op.pak[0] = f;
		hm->terms[k].op.pak[1] = mix(h ^ 0x55) & ((1u << NQB) - 1);
		hm->terms[k].cf = (double)(mix(h ^ 0xAA) >> 11) * 0x1p-53 - 0.5;
	}
	md->dets[0].idx = 0x0F3;
	md->dets[0].cf = 0.6;
	md->dets[1].idx = 0x2A05;
	md->dets[1].cf = 0.8 * I;
	return 0;
}

static int run(struct phase2_sharded *s, const struct circ_hamil *hm,
	const struct circ_muldet *md, _Complex double out[3][STEPS])
{
	return phase2_sharded_trott(s, hm, md, STEPS, 0.07, 0, out[0]) ||
		phase2_sharded_trott(s, hm, md, STEPS, 0.07, 1, out[1]) ||
		phase2_sharded_qdrift(s, hm, md, SAMPLES, DEPTH, 0.02, 77,
			out[2]);
}

/* rank 0 writes the id; the others wait for it (at most a minute) */
static int share_id(const char *dir, int rank, ncclUniqueId *id)
{
	char path[4096];
	snprintf(path, sizeof path, "%s/nccl_id", dir);
	if (rank == 0) {
		char tmp[4096];
		snprintf(tmp, sizeof tmp, "%s/nccl_id.tmp", dir);
		FILE *f = fopen(tmp, "wb");
		if (!f || fwrite(id, sizeof *id, 1, f) != 1) {
			if (f)
				fclose(f);
			return -1;
		}
		fclose(f);
		return rename(tmp, path);
	}
	for (int tries = 0; tries < 6000; tries++) {
		FILE *f = fopen(path, "rb");
		if (f) {
			const size_t got = fread(id, sizeof *id, 1, f);
			fclose(f);
			if (got == 1)
				return 0;
		}
		const struct timespec ts = { 0, 10000000 };
		nanosleep(&ts, NULL);
	}
	return -1;
}

int main(int argc, char **argv)
{
	const char *er = getenv("RANK"), *ew = getenv("WORLD_SIZE");
	if (argc < 2 || !er || !ew) {
		fprintf(stderr, "usage: RANK, WORLD_SIZE, LOCAL_RANK set; "
				"sharded_nccl <shared dir>\n");
		return 2;
	}
	const int rank = atoi(er), world = atoi(ew);
	/* world_init binds device LOCAL_RANK */
	if (world_init(NULL, NULL, 7) != WORLD_READY)
		return 1;
	ncclUniqueId id;
	if (rank == 0 && ncclGetUniqueId(&id) != ncclSuccess)
		return 1;
	if (share_id(argv[1], rank, &id) != 0) {
		fprintf(stderr, "rank %d: no NCCL id\n", rank);
		return 1;
	}
	struct nccl_io nio;
	memset(&nio, 0, sizeof nio);
	if (cudaStreamCreate(&nio.stream) != cudaSuccess ||
		ncclCommInitRank(&nio.comm, world, id, rank) != ncclSuccess) {
		fprintf(stderr, "rank %d: NCCL init failed\n", rank);
		return 1;
	}
	struct circ_hamil hm;
	struct circ_muldet md;
	int rc = 1;
	_Complex double got[3][STEPS], want[3][STEPS];
	memset(got, 0, sizeof got);
	memset(want, 0, sizeof want);
	if (make_problem(&hm, &md) != 0)
		goto out;
	const struct phase2_shard_io io = { xchg, sum, &nio };
	const uint32_t me = (uint32_t)rank;
	struct phase2_sharded *s = phase2_sharded_new(NQB, (uint32_t)world,
		&me, 1, PHASE2_PREC_FP64, &io, 1000);
	if (!s || run(s, &hm, &md, got) != 0) {
		fprintf(stderr, "rank %d: sharded run failed\n", rank);
		phase2_sharded_free(s);
		goto out;
	}
	phase2_sharded_free(s);
	uint32_t all[64];
	for (int r = 0; r < world && r < 64; r++)
		all[r] = (uint32_t)r;
	s = phase2_sharded_new(NQB, (uint32_t)world, all, (uint32_t)world,
		PHASE2_PREC_FP64, NULL, 0);
	if (!s || run(s, &hm, &md, want) != 0) {
		phase2_sharded_free(s);
		goto out;
	}
	phase2_sharded_free(s);
	if (memcmp(got, want, sizeof got) != 0) {
		fprintf(stderr, "rank %d: overlaps differ from one holder\n",
			rank);
		goto out;
	}
	if (rank == 0)
		printf("ok\n");
	rc = 0;
out:
	circ_hamil_free(&hm);
	circ_muldet_free(&md);
	ncclCommDestroy(nio.comm);
	cudaFree(nio.dsum);
	cudaStreamDestroy(nio.stream);
	world_free();
	return rc;
}
