#ifndef QDRIFT_H
#define QDRIFT_H

/*
 * qDRIFT driver.  Replaces include/circ/qdrift.h of Quantum-for-Life/phase2
 * (lines 26-61).  Per sample: prepare the initial state, draw `depth` terms
 * i.i.d. with probability |c_k| / sum |c|, apply
 * exp(i asin(step_size) sign(c_k) P_k) in draw order, record <psi0|psi>.
 * Draws use xoshiro256** seeded from `seed`; a zero seed selects the
 * driver default (the last non-zero seed used by this process, initially a
 * fixed constant), as the reference does.
 */

#include <stddef.h>

#include "phase2/circ.h"
#include "phase2/step_writer.h"
#include "prob.h"
#include "xoshiro256ss.h"

#ifdef __cplusplus
extern "C" {
#endif

struct qdrift_data {
	size_t samples;
	size_t depth;
	double step_size;
	uint64_t seed;
};

struct qdrift_ranct {
	struct circ_hamil hm_ran;
	struct prob_cdf cdf;
};

struct qdrift {
	struct circ ct;
	struct qdrift_data dt;
	struct qdrift_ranct ranct;
	struct xoshiro256ss rng;
	struct phase2_step_writer *sw;
};

int qdrift_init(struct qdrift *qd, const struct qdrift_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw);

void qdrift_free(struct qdrift *qd);

int qdrift_simul(struct qdrift *qd);

#ifdef __cplusplus
}
#endif

#endif /* QDRIFT_H */
