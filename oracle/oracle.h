/*
 * oracle.h -- CPU restatement of the phase2 state-vector hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the
 * smoke check and the CPU-baseline leg of bench.py call it to compute the
 * expected answer.  The product library (phase2_b200/libphase2.so) never
 * links or calls it.
 *
 * Every function restates the reference algorithm in plain C on a dense
 * FP64 state held in host memory (interleaved re/im doubles, index i =
 * basis state |i>, qubit k = bit k of i).  Each definition cites the
 * reference file:line it follows.  Rounding follows the reference's own
 * expression order (products and sums rounded separately; the build uses
 * -ffp-contract=off), so results are bit-identical to the reference CPU
 * path, which tests/test_oracle_pins.py checks against oracle/_ref and the
 * committed golden vectors in tests/golden/.
 *
 * A Pauli string is the pair (flip, phase) of 64-bit masks: flip bit k set
 * for X or Y on qubit k, phase bit k set for Z or Y on qubit k
 * (phase2/paulis.c:35-59).
 */
#ifndef PHASE2_ORACLE_H
#define PHASE2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

/* One Hamiltonian term, laid out like struct circ_hamil_term
 * (include/phase2/circ.h:48-55): 24 bytes, cf first. */
struct orc_term {
	double cf;
	uint64_t flip, phase;
};

/* xoshiro256** with splitmix64 seeding and 128 discarded draws
 * (lib/xoshiro256ss.c:34-85, include/xoshiro256ss.h:58-59). */
void orc_rng_init(uint64_t s[4], uint64_t seed);
uint64_t orc_rng_next(uint64_t s[4]);
double orc_rng_dbl01(uint64_t s[4]);

/* P|i> = i^r4 |j>; returns j (include/phase2/paulis.h:137-144). */
uint64_t orc_effect(uint64_t flip, uint64_t phase, uint64_t i, int *r4);

/* Lexicographic order, highest qubit first, I<X<Y<Z (phase2/paulis.c:190-205). */
int orc_pauli_cmp(uint64_t f1, uint64_t p1, uint64_t f2, uint64_t p2);

/* |w| CDF and its inverse (lib/prob.c:39-78).  Returns -1 if sum < eps. */
int orc_cdf_build(const double *w, size_t stride_bytes, size_t n, double *cdf,
	double *lambda);
size_t orc_cdf_inverse(const double *cdf, size_t n, double y);

/* Sign with dead zone |a| < DBL_EPSILON -> 0 (circ/internal.h:26-32). */
double orc_signof(double a);

/* Apply exp(+i phi P) to the dense state (phase2/qreg_qreg.c:149-160,181-198). */
void orc_rotate(double *amp, uint32_t nqb, uint64_t flip, uint64_t phase,
	double phi);
void orc_rotate_many(double *amp, uint32_t nqb, const uint64_t *flip,
	const uint64_t *phase, const double *phi, size_t n);

/* Sort terms as circ_hamil_sort_lex does (phase2/circ.c:60-81). */
void orc_sort_lex(struct orc_term *t, size_t n);

/* Multidet helpers (phase2/circ.c:215-224, 338-350).  dets_cf is
 * interleaved re/im. */
void orc_prepst(double *amp, uint32_t nqb, size_t ndets,
	const uint64_t *det_idx, const double *det_cf);
void orc_measure(const double *amp, size_t ndets, const uint64_t *det_idx,
	const double *det_cf, double out[2]);

/* Drivers.  `terms` is taken as given (not modified); out_z receives
 * 2*len doubles (one complex overlap per step or sample).  sort_lex = 1
 * reproduces trott_init/trott2_init (circ/trott.c:33, circ/trott2.c:33);
 * 0 keeps the given order (as the reference tests that build struct trott
 * by hand, test/t-circ_trott.c:162-201).  Return 0 or -1. */
int orc_trott(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t steps, double delta, int sort_lex, double *out_z);
int orc_trott2(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t steps, double delta, int sort_lex, double *out_z);
int orc_qdrift(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t samples, size_t depth, double step_size, uint64_t seed,
	double *out_z);
int orc_cmpsit(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t samples, size_t steps, size_t length, size_t depth,
	double angle_det, double angle_rand, uint64_t seed, double *out_z);

/* The qDRIFT / composite term sequences themselves (for schedule checks):
 * fills out_terms with the per-sample draws exactly as the drivers use
 * them.  qdrift: samples*depth terms with cf = signof(c) (circ/qdrift.c:95-103).
 * cmpsit: samples*steps*2*(length+depth) terms with cf already scaled
 * (circ/cmpsit.c:151-177). */
int orc_qdrift_draws(const struct orc_term *terms, size_t nterms,
	size_t samples, size_t depth, uint64_t seed, struct orc_term *out_terms);

/* One-shot entry (phase2/phase2_run.c:115-174). */
int orc_phase2_run(const char **pauli_strs, const double *coeffs,
	size_t nterms, double delta, const char *psi_str, double *out_re,
	double *out_im);

/* Squared norm with a plain sequential sum (diagnostics). */
double orc_norm2(const double *amp, uint32_t nqb);

/*
 * Coefficient-matrix trial state (phase2/state_prep_coeff.c:156-325).
 * Blocks: ncomp weights w with matrices Ca + k*n_sites*na and
 * Cb + k*n_sites*nb (Cb NULL = closed shell, C_beta = C_alpha); ncomp == 0
 * is the single block of weight 1.0 carried by Ca/Cb.
 * orc_coeff_expand_all: amp (2*2^nqb doubles) <- the expanded state
 * (state_prep_coeff_expand_all).  orc_coeff_inner: out <- sum over blocks
 * of the sequential inner product with amp (circ.c:315-336).  -1 on bad
 * sizes.
 */
int orc_coeff_expand_all(uint32_t nqb, uint32_t n_sites, uint32_t na,
	uint32_t nb, int tapered, size_t ncomp, const double *w,
	const double *Ca, const double *Cb, double *amp);
int orc_coeff_inner(uint32_t nqb, uint32_t n_sites, uint32_t na, uint32_t nb,
	int tapered, size_t ncomp, const double *w, const double *Ca,
	const double *Cb, const double *amp, double *out);

#endif /* PHASE2_ORACLE_H */
