/*
 * slab_exchange.c -- the C host loop of a sharded register's qubit swap,
 * written against the library's C-ABI only (include/phase2_b200.h): two
 * ranks of an nqb-qubit FP64 register split by its top qubit, held by one
 * process on one GPU, swap global qubit nqb-1 (the rank bit) with local
 * position L, chunk by chunk, through caller-owned device buffers.  The
 * partner's send buffer reaches this rank's receive buffer by a
 * device-to-device copy, where ranks on different GPUs would use
 * ncclSend/ncclRecv in a group.  Then the same swap again through
 * qreg_slab_swap (the in-place kernel for paired ranks on one GPU), which
 * must restore the original layout.
 *
 * Checked against the host copy of the global state: after the first swap
 * rank r's local amplitude i holds global amplitude G(i, r), where G has
 * bit nqb-1 = bit L of i, bit L = r, and i's other bits; after the second
 * swap every rank holds its original half again.  Exit status 0 and "ok"
 * on success.  Usage: slab_exchange [nqb] [L] [chunk]
 */
#include <complex.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <cuda_runtime.h>

#include "phase2.h"
#include "phase2_b200.h"

static uint64_t mix(uint64_t x)
{
	x ^= x >> 33;
	x *= UINT64_C(0xff51afd7ed558ccd);
	x ^= x >> 33;
	x *= UINT64_C(0xc4ceb9fe1a85ec53);
	x ^= x >> 33;
	return x;
}

/* Global amplitude g: a fixed pseudo-random complex value. */
static void amp(uint64_t g, double *re, double *im)
{
	*re = (double)(mix(2 * g + 1) >> 11) * 0x1p-53 - 0.5;
	*im = (double)(mix(2 * g + 2) >> 11) * 0x1p-53 - 0.5;
}

static int check(struct qreg *regs, uint32_t nloc, uint32_t l, int swapped)
{
	const uint64_t n = UINT64_C(1) << nloc;
	double *st = malloc(2 * n * sizeof *st);
	int bad = 0;
	for (uint32_t r = 0; r < 2 && st && !bad; r++) {
		if (qreg_get_state(&regs[r], st) != 0) {
			bad = 1;
			break;
		}
		for (uint64_t i = 0; i < n && !bad; i++) {
			uint64_t g;
			if (swapped) {
				const uint64_t hi = i >> l & 1;
				g = (i & ~(UINT64_C(1) << l)) |
					((uint64_t)r << l) | (hi << nloc);
			} else {
				g = i | ((uint64_t)r << nloc);
			}
			double re, im;
			amp(g, &re, &im);
			if (st[2 * i] != re || st[2 * i + 1] != im) {
				fprintf(stderr, "rank %u amplitude %llu: %g%+gi, "
						"want %g%+gi\n",
					r, (unsigned long long)i, st[2 * i],
					st[2 * i + 1], re, im);
				bad = 1;
			}
		}
	}
	free(st);
	return st ? bad : 1;
}

int main(int argc, char **argv)
{
	const uint32_t nqb = argc > 1 ? (uint32_t)atoi(argv[1]) : 14;
	const uint32_t l = argc > 2 ? (uint32_t)atoi(argv[2]) : 3;
	const uint64_t chunk = argc > 3 ? strtoull(argv[3], NULL, 10) : 1000;
	const uint32_t nloc = nqb - 1;
	const uint64_t n = UINT64_C(1) << nloc, half = n / 2;
	if (nqb < 3 || l >= nloc || chunk == 0) {
		fprintf(stderr, "bad arguments\n");
		return 2;
	}
	if (world_init(NULL, NULL, 7) != WORLD_READY) {
		fprintf(stderr, "world_init failed\n");
		return 1;
	}
	struct qreg regs[2];
	double *st = malloc(2 * n * sizeof *st);
	int rc = 1;
	if (!st || qreg_init_prec(&regs[0], nloc, PHASE2_PREC_FP64) != 0 ||
		qreg_init_prec(&regs[1], nloc, PHASE2_PREC_FP64) != 0)
		goto out;
	for (uint32_t r = 0; r < 2; r++) {
		for (uint64_t i = 0; i < n; i++)
			amp(i | ((uint64_t)r << nloc), &st[2 * i], &st[2 * i + 1]);
		if (qreg_set_state(&regs[r], st) != 0)
			goto out;
	}

	/* rank r sends the half whose bit l differs from its own rank bit:
	 * v = 1 - r; partner = r ^ 1 */
	void *sbuf[2] = { NULL, NULL }, *rbuf[2] = { NULL, NULL };
	const size_t bytes = chunk * 2 * sizeof(double);
	for (int r = 0; r < 2; r++)
		if (cudaMalloc(&sbuf[r], bytes) != cudaSuccess ||
			cudaMalloc(&rbuf[r], bytes) != cudaSuccess)
			goto out_buf;
	for (uint64_t first = 0; first < half; first += chunk) {
		const uint64_t cnt = half - first < chunk ? half - first : chunk;
		for (uint32_t r = 0; r < 2; r++)
			if (qreg_slab_get(&regs[r], l, 1 - r, first, cnt,
				    sbuf[r]) != 0)
				goto out_buf;
		/* the transport: partner's send buffer -> my receive buffer */
		for (uint32_t r = 0; r < 2; r++)
			if (cudaMemcpy(rbuf[r], sbuf[r ^ 1],
				    cnt * 2 * sizeof(double),
				    cudaMemcpyDeviceToDevice) != cudaSuccess)
				goto out_buf;
		for (uint32_t r = 0; r < 2; r++)
			if (qreg_slab_put(&regs[r], l, 1 - r, first, cnt,
				    rbuf[r]) != 0)
				goto out_buf;
	}
	if (check(regs, nloc, l, 1)) {
		fprintf(stderr, "exchange through buffers: wrong state\n");
		goto out_buf;
	}
	/* the in-place kernel for the same pair: swapping again restores
	 * the original layout */
	if (qreg_slab_swap(&regs[0], &regs[1], l, 1, 0) != 0 ||
		check(regs, nloc, l, 0)) {
		fprintf(stderr, "in-place swap: wrong state\n");
		goto out_buf;
	}
	/* rejected: a host pointer as the device buffer */
	if (qreg_slab_get(&regs[0], l, 0, 0, 1, st) != -1) {
		fprintf(stderr, "host buffer accepted\n");
		goto out_buf;
	}
	printf("ok\n");
	rc = 0;
out_buf:
	for (int r = 0; r < 2; r++) {
		cudaFree(sbuf[r]);
		cudaFree(rbuf[r]);
	}
	qreg_free(&regs[0]);
	qreg_free(&regs[1]);
out:
	free(st);
	world_free();
	return rc;
}
