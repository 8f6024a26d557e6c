#ifndef TROTT2_H
#define TROTT2_H

/*
 * Second-order (Strang) Trotter driver.  Replaces include/circ/trott2.h of
 * Quantum-for-Life/phase2 (lines 18-41).  One step is a forward sweep at
 * delta/2 followed by a reverse sweep at delta/2 over the lex-sorted terms,
 * then <psi0|psi>.
 */

#include "phase2/circ.h"
#include "phase2/step_writer.h"

#ifdef __cplusplus
extern "C" {
#endif

struct trott2_data {
	size_t steps;
	double delta;
};

struct trott2 {
	struct circ ct;
	struct trott2_data dt;
	struct phase2_step_writer *sw;
};

int trott2_init(struct trott2 *t2, const struct trott2_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw);

void trott2_free(struct trott2 *t2);

int trott2_simul(struct trott2 *t2);

#ifdef __cplusplus
}
#endif

#endif /* TROTT2_H */
