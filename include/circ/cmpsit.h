#ifndef CMPSIT_H
#define CMPSIT_H

/*
 * Composite (partially randomised) second-order driver.  Replaces
 * include/circ/cmpsit.h of Quantum-for-Life/phase2 (lines 28-71).  The
 * `length` largest |c_k| terms (lex-sorted) are applied deterministically at
 * angle_det * c_k; the rest are sampled qDRIFT-style, `depth` draws per
 * half step at +-angle_rand.  A step is a forward half-sweep of one sample
 * and a reverse half-sweep of a fresh sample, both at omega = 0.5; one
 * overlap per sample after all steps.
 */

#include <stddef.h>

#include "phase2.h"
#include "phase2/step_writer.h"
#include "xoshiro256ss.h"

#ifdef __cplusplus
extern "C" {
#endif

struct cmpsit_data {
	size_t samples;
	size_t steps;
	size_t length;
	size_t depth;
	double angle_det;
	double angle_rand;
	uint64_t seed;
};

struct cmpsit_ranct {
	struct circ_hamil hm_det, hm_ran, hm_smpl;
	struct prob_cdf cdf;
	double lambda_r;
	size_t depth;
	double angle_rand;
};

struct cmpsit {
	struct circ ct;
	struct cmpsit_data dt;
	struct cmpsit_ranct ranct;
	struct xoshiro256ss rng;
	struct phase2_step_writer *sw;
};

int cmpsit_init(struct cmpsit *cp, const struct cmpsit_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw);

void cmpsit_free(struct cmpsit *cp);

int cmpsit_simul(struct cmpsit *cp);

#ifdef __cplusplus
}
#endif

#endif /* CMPSIT_H */
