/*
 * ref_bench.c -- CPU baseline timing of the reference's own rotation path
 * (TEST INFRASTRUCTURE, run by bench.py's reference arm and cpu_baseline).
 *
 * Usage: ref_bench NQB NROT REPEATS
 *
 * Builds an NQB-qubit register with the reference's qreg_init (CPU
 * backend, single-rank MPI stand-in), sets a basis state, and times
 * REPEATS calls of qreg_paulirot (phase2/qreg.c:135-142) applying NROT
 * JW-like rotations (flip on 2 or 4 qubits, Z chains), the reference's
 * batch.  Prints one line: "<best_seconds> <rot_amp_per_s>" with the
 * minimum over repeats (the reference's own min-of-K convention,
 * bench/bench.h).
 *
 * Built with REF_BENCH_CUDA against the reference's CUDA backend
 * (oracle/Makefile ref-cuda) it times the reference's own GPU kernels
 * (phase2/qreg_cuda_lo.cu); qreg_paulirot only launches them, so every
 * timed call ends with a device synchronisation, and one untimed call
 * comes first (module load).
 */
#define _POSIX_C_SOURCE 200809L

#include <complex.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include "phase2.h"

#ifdef REF_BENCH_CUDA
#include <cuda_runtime_api.h>
#define DEVICE_SYNC() cudaDeviceSynchronize()
#else
#define DEVICE_SYNC() ((void)0)
#endif

static double now(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static uint64_t lcg(uint64_t *s)
{
	*s = *s * UINT64_C(6364136223846793005) + UINT64_C(1442695040888963407);
	return *s >> 33;
}

int main(int argc, char **argv)
{
	if (argc < 4) {
		fprintf(stderr, "usage: %s NQB NROT REPEATS\n", argv[0]);
		return 2;
	}
	const uint32_t nqb = (uint32_t)atoi(argv[1]);
	const size_t nrot = (size_t)atol(argv[2]);
	const int reps = atoi(argv[3]);
	if (world_init(NULL, NULL, UINT64_C(0x5eed)) != WORLD_READY)
		return 1;
	struct qreg reg;
	if (qreg_init(&reg, nqb) < 0)
		return 1;
	qreg_zero(&reg);
	qreg_setamp(&reg, 1, 1.0);
	struct paulis *lo = calloc(nrot, sizeof *lo);
	double *phi = calloc(nrot, sizeof *phi);
	uint64_t s = 12345;
	for (size_t k = 0; k < nrot; k++) {
		const int m = (lcg(&s) % 10) ? 4 : 2;
		int pos[4];
		for (int a = 0; a < m; a++) {
		again:
			pos[a] = (int)(lcg(&s) % nqb);
			for (int b = 0; b < a; b++)
				if (pos[b] == pos[a])
					goto again;
		}
		for (int a = 0; a < m; a++)
			paulis_set(&lo[k], (lcg(&s) & 1) ? PAULI_X : PAULI_Y,
				(uint32_t)pos[a]);
		phi[k] = 1e-3 * (double)(1 + lcg(&s) % 1000);
	}
	const struct paulis hi = paulis_new();
	double best = 1e300;
#ifdef REF_BENCH_CUDA
	qreg_paulirot(&reg, hi, lo, phi, nrot);
	DEVICE_SYNC();
#endif
	for (int r = 0; r < reps; r++) {
		const double t0 = now();
		qreg_paulirot(&reg, hi, lo, phi, nrot);
		DEVICE_SYNC();
		const double dt = now() - t0;
		if (dt < best)
			best = dt;
	}
	printf("%.6f %.6e\n", best,
		(double)nrot * (double)reg.namp / best);
	qreg_free(&reg);
	world_free();
	return 0;
}
