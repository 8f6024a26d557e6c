#ifndef TROTT_H
#define TROTT_H

/*
 * First-order Lie-Trotter driver.  Replaces include/circ/trott.h of
 * Quantum-for-Life/phase2 (lines 17-40).  One step applies every term once,
 * phi_k = delta * c_k, in lexicographic Pauli order (trott_init sorts the
 * adopted Hamiltonian), then records <psi0|psi>.
 */

#include "phase2/circ.h"
#include "phase2/step_writer.h"

#ifdef __cplusplus
extern "C" {
#endif

struct trott_data {
	size_t steps;
	double delta;
};

struct trott {
	struct circ ct;
	struct trott_data dt;
	struct phase2_step_writer *sw;
};

/* Adopt hm and *sp_data (see circ_init); sw is borrowed and may be NULL.
 * 0 or -1 (reference: trott.h:32-34). */
int trott_init(struct trott *tt, const struct trott_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw);

void trott_free(struct trott *tt);

/* dt.steps steps; overlaps into ct.vals (and sw).  0 or -1. */
int trott_simul(struct trott *tt);

#ifdef __cplusplus
}
#endif

#endif /* TROTT_H */
