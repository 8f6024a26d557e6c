/*
 * sharded_threads.c -- the C sharded register (include/phase2_sharded.h)
 * with ranks split between two holders that talk through the caller's
 * transport, against one holder of every rank.
 *
 * Two host threads stand for two processes on one GPU: each creates a
 * phase2_sharded object for its share of the ranks and runs the same
 * driver.  Their transport meets at a two-party barrier: exchange posts
 * this rank's send buffer, waits for the partner's, copies it device to
 * device into the receive buffer and waits again (where processes on two
 * GPUs would call ncclSend/ncclRecv); sum adds the holders' partial
 * vectors.  Both holders must report the overlaps of the single holder
 * bit for bit (FP64): Trotter (first and second order) and qDRIFT, for
 * world 2 (one rank each), world 4 (ranks {1,0} and {2,3}: swaps of rank
 * bit 0 stay inside a holder, swaps of bit 1 go through the transport)
 * and world 8 (ranks {6,4,2,0} and {1,3,5,7}: swaps of bit 0 make four
 * exchanges per holder, which must pair up in the same order), with small
 * exchange chunks.  Exit 0 and "ok" on success.
 */
#include <complex.h>
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "phase2.h"
#include "phase2_b200.h"
#include "phase2_sharded.h"

#define NQB 12
#define NTERMS 300
#define STEPS 3
#define SAMPLES 2
#define DEPTH 200

struct meet {
	pthread_barrier_t bar;
	pthread_mutex_t mu;
	const void *slot[8]; /* send buffer posted by each rank */
	double acc[1 << 14];
	int bad;
};

static struct meet M;

static int xchg(void *ctx, uint32_t rank, uint32_t peer, const void *send,
	void *recv, size_t bytes)
{
	struct meet *m = ctx;
	m->slot[rank] = send;
	pthread_barrier_wait(&m->bar);
	const int rc = cudaMemcpy(recv, m->slot[peer], bytes,
				       cudaMemcpyDeviceToDevice) == cudaSuccess
		? 0 : -1;
	pthread_barrier_wait(&m->bar);
	return rc;
}

static int sum(void *ctx, double *vals, size_t n)
{
	struct meet *m = ctx;
	if (n > sizeof m->acc / sizeof m->acc[0])
		return -1;
	if (pthread_barrier_wait(&m->bar) == PTHREAD_BARRIER_SERIAL_THREAD)
		memset(m->acc, 0, n * sizeof *vals);
	pthread_barrier_wait(&m->bar);
	pthread_mutex_lock(&m->mu);
	for (size_t i = 0; i < n; i++)
		m->acc[i] += vals[i];
	pthread_mutex_unlock(&m->mu);
	pthread_barrier_wait(&m->bar);
	memcpy(vals, m->acc, n * sizeof *vals);
	pthread_barrier_wait(&m->bar);
	return 0;
}

static struct circ_hamil HM;
static struct circ_muldet MD;

static uint64_t mix(uint64_t x)
{
	x ^= x >> 31;
	x *= UINT64_C(0x7fb5d329728ea185);
	x ^= x >> 27;
	x *= UINT64_C(0x81dadef4bc2dd44d);
	x ^= x >> 33;
	return x;
}

/* Terms flipping at most three qubits, random phases and coefficients;
 * two determinants. */
static int make_problem(void)
{
	if (circ_hamil_init(&HM, NQB, NTERMS) != 0 ||
		circ_muldet_init(&MD, 2) != 0)
		return -1;
	for (size_t k = 0; k < NTERMS; k++) {
		uint64_t f = 0;
		const uint64_t h = mix(k + 1);
		for (int j = 0; j < (int)(h % 4); j++)
			f |= UINT64_C(1) << (mix(h + j) % NQB);
		HM.terms[k].op.pak[0] = f;
		HM.terms[k].op.pak[1] = mix(h ^ 0x55) & ((1u << NQB) - 1);
		HM.terms[k].cf = (double)(mix(h ^ 0xAA) >> 11) * 0x1p-53 - 0.5;
	}
	MD.dets[0].idx = 0x0F3;
	MD.dets[0].cf = 0.6;
	MD.dets[1].idx = 0xA05;
	MD.dets[1].cf = 0.8 * I;
	return 0;
}

struct job {
	uint32_t world, ranks[8], nranks;
	int use_io;
	_Complex double out[3][STEPS > SAMPLES ? STEPS : SAMPLES];
	int rc;
};

static void *run(void *arg)
{
	struct job *j = arg;
	const struct phase2_shard_io io = { xchg, sum, &M };
	struct phase2_sharded *s = phase2_sharded_new(NQB, j->world, j->ranks,
		j->nranks, PHASE2_PREC_FP64, j->use_io ? &io : NULL, 100);
	j->rc = -1;
	if (!s)
		return NULL;
	if (phase2_sharded_trott(s, &HM, &MD, STEPS, 0.07, 0, j->out[0]) == 0 &&
		phase2_sharded_trott(s, &HM, &MD, STEPS, 0.07, 1, j->out[1]) ==
			0 &&
		phase2_sharded_qdrift(s, &HM, &MD, SAMPLES, DEPTH, 0.02, 77,
			j->out[2]) == 0)
		j->rc = 0;
	phase2_sharded_free(s);
	return NULL;
}

static int same(const _Complex double *a, const _Complex double *b, size_t n)
{
	return memcmp(a, b, n * sizeof *a) == 0;
}

/* Holder t holds the upper or lower half of the ranks (interleave 0) or
 * the odd or even ranks (interleave 1); holder 0 lists its ranks in
 * decreasing order, holder 1 in increasing order. */
static int check_world(uint32_t world, int interleave)
{
	struct job all = { .world = world, .nranks = world };
	for (uint32_t r = 0; r < world; r++)
		all.ranks[r] = r;
	run(&all);
	if (all.rc != 0) {
		fprintf(stderr, "world %u: single holder failed\n", world);
		return -1;
	}
	struct job part[2];
	memset(part, 0, sizeof part);
	for (int t = 0; t < 2; t++) {
		part[t].world = world;
		part[t].nranks = world / 2;
		part[t].use_io = 1;
		for (uint32_t r = 0; r < world / 2; r++) {
			const uint32_t i = t == 0 ? world / 2 - 1 - r : r;
			part[t].ranks[r] = interleave ? 2 * i + (uint32_t)t
						      : (uint32_t)t * (world / 2) + i;
		}
	}
	pthread_t th[2];
	for (int t = 0; t < 2; t++)
		pthread_create(&th[t], NULL, run, &part[t]);
	for (int t = 0; t < 2; t++)
		pthread_join(th[t], NULL);
	for (int t = 0; t < 2; t++) {
		if (part[t].rc != 0) {
			fprintf(stderr, "world %u/%d: holder %d failed\n", world,
				interleave, t);
			return -1;
		}
		if (!same(part[t].out[0], all.out[0], STEPS) ||
			!same(part[t].out[1], all.out[1], STEPS) ||
			!same(part[t].out[2], all.out[2], SAMPLES)) {
			fprintf(stderr, "world %u/%d: holder %d differs: "
					"%.17g%+.17gi vs %.17g%+.17gi\n",
				world, interleave, t, creal(part[t].out[0][0]),
				cimag(part[t].out[0][0]), creal(all.out[0][0]),
				cimag(all.out[0][0]));
			return -1;
		}
	}
	return 0;
}

int main(void)
{
	if (world_init(NULL, NULL, 7) != WORLD_READY) {
		fprintf(stderr, "world_init failed\n");
		return 1;
	}
	pthread_barrier_init(&M.bar, NULL, 2);
	pthread_mutex_init(&M.mu, NULL);
	int rc = 1;
	if (make_problem() == 0 && check_world(2, 0) == 0 &&
		check_world(4, 0) == 0 && check_world(8, 1) == 0) {
		printf("ok\n");
		rc = 0;
	}
	circ_hamil_free(&HM);
	circ_muldet_free(&MD);
	world_free();
	return rc;
}
