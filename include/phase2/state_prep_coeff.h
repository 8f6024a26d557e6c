#ifndef PHASE2_STATE_PREP_COEFF_H
#define PHASE2_STATE_PREP_COEFF_H

/*
 * Coefficient-matrix trial states (Slater-Condon expansion) and their
 * overlap with the register: the interface of the reference's
 * include/phase2/state_prep_coeff.h.
 *
 * A trial state is given by real orbital-coefficient matrices C_alpha
 * (n_sites x n_alpha, row-major) and C_beta (n_sites x n_beta; C_alpha
 * again when NULL).  Its amplitude on the basis state with alpha
 * occupation tuple a (bits 0..n_sites-1) and beta occupation tuple b (bits
 * n_sites..2 n_sites-1) is
 *     c = weight * det(C_alpha[a, :]) * det(C_beta[b, :]),
 * over all k-subsets a, b of the sites; |c| < 1e-12 is skipped.  tapered
 * drops bits 0 and n_sites of each index (a symmetry-reduced register of
 * 2 n_sites - 2 qubits).
 *
 * In this library the expansion and the overlap run on the GPU over the
 * register's device state; the scratch carries the k-subset tuples (in lex
 * order) and the determinants of the current block.
 */

#include <stddef.h>
#include <stdint.h>

#include "phase2/qreg.h"

struct data_coeff_matrix;

struct state_prep_coeff_scratch {
	uint32_t n_sites, n_alpha, n_beta;
	uint32_t *tup_a, *tup_b;
	double *det_a, *det_b;
	size_t Ma, Mb;
};

/* Fill the (n_sites choose n_alpha) and (n_sites choose n_beta) tuples;
 * 0, or -1 on size bounds (at most 16 particles per spin) or
 * allocation failure. */
int state_prep_coeff_scratch_init(struct state_prep_coeff_scratch *sc,
	uint32_t n_sites, uint32_t n_alpha, uint32_t n_beta);

void state_prep_coeff_scratch_free(struct state_prep_coeff_scratch *sc);

/* Write (accumulate = 0) or add (accumulate = 1) the weighted expansion
 * into the register.  0 or -1. */
int state_prep_coeff_expand(struct qreg *reg,
	struct state_prep_coeff_scratch *sc, const double *C_alpha,
	const double *C_beta, double weight, int tapered, int accumulate);

/* Zero the register, then expand the single block (n_components == 0) or
 * accumulate every block with its weight.  0 or -1. */
int state_prep_coeff_expand_all(struct qreg *reg,
	struct state_prep_coeff_scratch *sc,
	const struct data_coeff_matrix *cm);

/* *out = sum over the expansion of c * a[idx] (the trial state is real).
 * 0 or -1. */
int state_prep_coeff_inner(struct qreg *reg,
	struct state_prep_coeff_scratch *sc, const double *C_alpha,
	const double *C_beta, double weight, int tapered, _Complex double *out);

#endif /* PHASE2_STATE_PREP_COEFF_H */
