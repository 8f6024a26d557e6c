/*
 * ref_mpi.c -- times the reference's own CPU drivers run as R MPI ranks on
 * this host's cores (TEST INFRASTRUCTURE: the CPU baseline of bench.py).
 *
 * Usage: ref_mpi RANKS INPUT REPEATS [WARMUP]
 *
 * INPUT (written by bench.py) holds one driver run: a header
 *   char magic[8] = "P2REFIN1"; uint32 mode (0 qdrift, 1 trott2);
 *   uint32 nqb; uint64 nterms, ndets; uint64 count (qdrift: depth,
 *   trott2: steps); double angle (qdrift: step_size, trott2: delta);
 *   uint64 seed (qdrift)
 * then nterms terms in the reference's layout {double cf; uint64 flip,
 * phase} and ndets determinants {uint64 idx; double re, im}.
 *
 * The process forks into RANKS ranks (oracle/mpi_shm, a shared-memory
 * stand-in for the MPI calls of the reference core), each holding its
 * 2^(nqb - log2 RANKS) amplitudes as the reference distributes them
 * (phase2/qreg.c:46-66).  One driver object runs REPEATS times: qdrift
 * with one sample (circ/qdrift.c:105-134; every repeat draws a fresh
 * sample from the same stream) or trott2 (circ/trott2.c:44-74); each
 * repeat is bracketed by barriers and the minimum is kept (the reference's
 * min-of-K convention, bench/bench.h); WARMUP untimed runs come first.
 * Rank 0 prints one line:
 *   <ranks> <rotations per run> <best seconds> <rot.amp/s> <mailbox 0/1>
 *   <overlap re> <overlap im>
 */
#define _POSIX_C_SOURCE 200809L

#include <complex.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "circ/qdrift.h"
#include "circ/trott2.h"
#include "mpi.h"
#include "phase2.h"

struct ref_in_hdr {
	char magic[8];
	uint32_t mode, nqb;
	uint64_t nterms, ndets, count;
	double angle;
	uint64_t seed;
};

struct ref_in_det {
	uint64_t idx;
	double re, im;
};

static double now(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

int main(int argc, char **argv)
{
	if (argc < 4) {
		fprintf(stderr, "usage: %s RANKS INPUT REPEATS\n", argv[0]);
		return 2;
	}
	const int ranks = atoi(argv[1]);
	const int reps = atoi(argv[3]);
	const int warm = argc > 4 ? atoi(argv[4]) : 0;
	FILE *f = fopen(argv[2], "rb");
	struct ref_in_hdr h;
	if (!f || fread(&h, sizeof h, 1, f) != 1 ||
		memcmp(h.magic, "P2REFIN1", 8) != 0 || h.mode > 1 ||
		ranks < 1 || (ranks & (ranks - 1)) || reps < 1 || warm < 0) {
		fprintf(stderr, "ref_mpi: bad arguments or input\n");
		return 2;
	}
	struct circ_hamil hm;
	struct circ_muldet md;
	if (circ_hamil_init(&hm, h.nqb, h.nterms) < 0 ||
		circ_muldet_init(&md, h.ndets) < 0)
		return 2;
	hm.len = h.nterms;
	if (fread(hm.terms, sizeof hm.terms[0], h.nterms, f) != h.nterms)
		return 2;
	for (uint64_t d = 0; d < h.ndets; d++) {
		struct ref_in_det v;
		if (fread(&v, sizeof v, 1, f) != 1)
			return 2;
		md.dets[d].idx = v.idx;
		md.dets[d].cf = CMPLX(v.re, v.im);
	}
	fclose(f);

	/* mailboxes (only used where cross-process reads are refused) hold
	 * one rank's slab */
	const size_t slab = ((size_t)1 << h.nqb) / (size_t)ranks * 16;
	const int rank = mpi_shm_spawn(ranks, slab);
	if (rank < 0) {
		fprintf(stderr, "ref_mpi: spawn failed\n");
		return 2;
	}
	int rc = 0;
	if (world_init(NULL, NULL, UINT64_C(0x5eedc0de)) != WORLD_READY)
		return mpi_shm_join(2);

	double best = 1e300;
	size_t rots = 0;
	_Complex double z = 0;
	if (h.mode == 0) {
		struct qdrift qd;
		memset(&qd, 0, sizeof qd);
		const struct qdrift_data dt = { .samples = 1, .depth = h.count,
			.step_size = h.angle, .seed = h.seed };
		if (qdrift_init(&qd, &dt, hm, STPREP_MULTIDET, &md, NULL) < 0)
			return mpi_shm_join(2);
		rots = h.count;
		for (int r = 0; r < warm + reps && rc == 0; r++) {
			MPI_Barrier(MPI_COMM_WORLD);
			const double t0 = now();
			rc = qdrift_simul(&qd);
			MPI_Barrier(MPI_COMM_WORLD);
			const double t = now() - t0;
			if (r >= warm)
				best = t < best ? t : best;
			z = qd.ct.vals.z[0];
		}
		qdrift_free(&qd);
	} else {
		struct trott2 t2;
		memset(&t2, 0, sizeof t2);
		const struct trott2_data dt = { .steps = h.count,
			.delta = h.angle };
		if (trott2_init(&t2, &dt, hm, STPREP_MULTIDET, &md, NULL) < 0)
			return mpi_shm_join(2);
		rots = 2 * h.nterms * h.count;
		for (int r = 0; r < warm + reps && rc == 0; r++) {
			MPI_Barrier(MPI_COMM_WORLD);
			const double t0 = now();
			rc = trott2_simul(&t2);
			MPI_Barrier(MPI_COMM_WORLD);
			const double t = now() - t0;
			if (r >= warm)
				best = t < best ? t : best;
			z = t2.ct.vals.z[h.count - 1];
		}
		trott2_free(&t2);
	}
	const int mailbox = mpi_shm_mailbox();
	world_free();
	rc = mpi_shm_join(rc != 0);
	if (rank == 0 && rc == 0)
		printf("%d %zu %.9g %.9g %d %.17g %.17g\n", ranks, rots, best,
			(double)rots * (double)((uint64_t)1 << h.nqb) / best,
			mailbox, creal(z), cimag(z));
	return rc;
}
