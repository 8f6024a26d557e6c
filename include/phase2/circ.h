#ifndef CIRC_H
#define CIRC_H

/*
 * Circuit context: Hamiltonian, initial state, register, batch cache and
 * per-step results.  Replaces include/phase2/circ.h of Quantum-for-Life/
 * phase2 (lines 42-299) with the same carriers, ownership rules and
 * functions.  The coefficient-matrix state-prep payload types are kept for
 * source compatibility; circ_init rejects STPREP_COEFF_MATRIX (-1), since
 * this library implements the multi-determinant path only.
 */

#include <stddef.h>
#include <stdint.h>

#include "phase2/paulis.h"
#include "phase2/qreg.h"
#include "phase2/state_prep_coeff.h"

#ifdef __cplusplus
extern "C" {
#endif

/* H = sum_k cf_k P_k (reference: circ.h:48-55). */
struct circ_hamil {
	uint32_t qb;
	struct circ_hamil_term {
		double cf;
		struct paulis op;
	} *terms;
	size_t len;
};

/* |psi> = sum_d cf_d |idx_d> (reference: circ.h:65-71). */
struct circ_muldet {
	struct {
		uint64_t idx;
		_Complex double cf;
	} *dets;
	size_t len;
};

/* One complex overlap per step or sample (reference: circ.h:78-81). */
struct circ_values {
	_Complex double *z;
	size_t len;
};

/* Reference: circ.h:91-94. */
enum stprep_kind {
	STPREP_MULTIDET = 1,
	STPREP_COEFF_MATRIX = 2,
};

/* Coefficient-matrix payload (reference: circ.h:131-149). */
struct data_coeff_block {
	double cf;
	const double *C_alpha;
	const double *C_beta;
};

struct data_coeff_matrix {
	uint32_t nqb;
	uint32_t n_sites;
	uint32_t n_alpha;
	uint32_t n_beta;
	int closed_shell;
	int tapered;
	size_t n_components;
	const double *C_alpha;
	const double *C_beta;
	struct data_coeff_block *blocks;
};

/* Reference: circ.h:169-178. */
struct circ {
	struct circ_hamil hm;
	struct circ_muldet md;
	struct circ_cache *cache;
	struct circ_values vals;
	struct qreg reg;
	enum stprep_kind stprep_kind;
	struct data_coeff_matrix cm;
	struct state_prep_coeff_scratch sp_scratch;
};

/* Carriers (reference: circ.h:202-226).  _init: 0 or -1; _free idempotent. */
int circ_hamil_init(struct circ_hamil *hm, uint32_t qb, size_t len);
void circ_hamil_free(struct circ_hamil *hm);
void circ_hamil_sort_lex(struct circ_hamil *hm);

int circ_muldet_init(struct circ_muldet *md, size_t len);
void circ_muldet_free(struct circ_muldet *md);

void data_coeff_matrix_free(struct data_coeff_matrix *cm);

int circ_values_init(struct circ_values *vals, size_t len);
void circ_values_free(struct circ_values *vals);

/* Adopt hm and *sp_data (freed by circ_free, and by circ_init itself on
 * failure), allocate the register, cache and vals_len result slots
 * (reference: circ.h:254-255).  0 or -1. */
int circ_init(struct circ *ct, struct circ_hamil hm,
	enum stprep_kind sp_kind, const void *sp_data, size_t vals_len);

void circ_free(struct circ *ct);

/* Zero the register and write the initial state (reference: circ.h:271). */
int circ_prepst(struct circ *ct);

/* One sweep exp(i omega H) over hm's terms, forward or reverse
 * (reference: circ.h:283-285).  0 or -1. */
int circ_step(struct circ *ct, const struct circ_hamil *hm, double omega);
int circ_step_reverse(
	struct circ *ct, const struct circ_hamil *hm, double omega);

/* <psi0|psi> = sum_d conj(cf_d) a[idx_d]; 0 for an unknown kind
 * (reference: circ.h:299). */
_Complex double circ_measure(struct circ *ct);

#ifdef __cplusplus
}
#endif

#endif /* CIRC_H */
