/*
 * state_prep.c -- coefficient-matrix trial states
 * (include/phase2/state_prep_coeff.h): the reference's
 * phase2/state_prep_coeff.c with the expansion and the overlap on the
 * device.
 *
 * The host enumerates the k-subsets of the sites in lex order (as
 * lib/combinations.c does) and computes one small determinant per subset
 * and block by Gaussian elimination with partial pivoting, in the
 * operation order of lib/det_small.c, so the FP64 coefficients are
 * bit-identical to the reference's.  The device then forms every product
 * weight * det_a * det_b in the reference's order and writes or adds it at
 * its index (engine.cu k_cm_expand), or sums it against the register
 * (k_cm_inner, compensated; the reference sums sequentially, so the overlap
 * agrees to rounding, not bit for bit).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "prep"
#include "log.h"

#include "phase2/circ.h"
#include "phase2/state_prep_coeff.h"

#include "p2_host.h"
#include "p2_internal.h"

/* Largest particle count per spin (lib/det_small.h, lib/combinations.h). */
#define SPC_MAX_K 32u

/* C(n, k) as the reference computes it (state_prep_coeff.c:52-66); 0 when
 * k > n. */
static uint64_t choose(uint32_t n, uint32_t k)
{
	if (k > n)
		return 0;
	const uint32_t r = k > n - k ? n - k : k;
	uint64_t num = 1, den = 1;
	for (uint32_t i = 1; i <= r; i++) {
		num *= (uint64_t)(n - r + i);
		den *= (uint64_t)i;
	}
	return num / den;
}

/* All k-subsets of {0..n-1} in lex order, k entries each (one empty row
 * when k = 0).  Returns the count written, which must be C(n, k). */
static size_t lex_subsets(uint32_t n, uint32_t k, uint32_t *out, size_t cap)
{
	uint32_t c[SPC_MAX_K];
	for (uint32_t i = 0; i < k; i++)
		c[i] = i;
	size_t m = 0;
	for (;;) {
		if (m >= cap)
			return m + 1;
		for (uint32_t i = 0; i < k; i++)
			out[m * k + i] = c[i];
		m++;
		/* rightmost position that can still grow */
		int32_t j = (int32_t)k - 1;
		while (j >= 0 && c[j] == n - k + (uint32_t)j)
			j--;
		if (j < 0)
			return m;
		c[j]++;
		for (uint32_t i = (uint32_t)j + 1; i < k; i++)
			c[i] = c[i - 1] + 1;
	}
}

/* det of the k x k matrix a (row-major, overwritten): elimination with
 * partial pivoting (first row of largest |pivot|), det = product of the
 * pivots with one sign flip per row swap, rows below updated with the
 * multiplier pivot-row-entry / pivot -- lib/det_small.c:27-71. */
static double small_det(double *a, uint32_t k)
{
	double det = 1.0;
	for (uint32_t col = 0; col < k; col++) {
		uint32_t p = col;
		double best = fabs(a[col * k + col]);
		for (uint32_t r = col + 1; r < k; r++) {
			const double v = fabs(a[r * k + col]);
			if (v > best) {
				best = v;
				p = r;
			}
		}
		if (best == 0.0)
			return 0.0;
		if (p != col) {
			for (uint32_t c = col; c < k; c++) {
				const double t = a[col * k + c];
				a[col * k + c] = a[p * k + c];
				a[p * k + c] = t;
			}
			det = -det;
		}
		const double piv = a[col * k + col];
		det *= piv;
		const double inv = 1.0 / piv;
		for (uint32_t r = col + 1; r < k; r++) {
			const double f = a[r * k + col] * inv;
			if (f == 0.0)
				continue;
			for (uint32_t c = col + 1; c < k; c++)
				a[r * k + c] -= f * a[col * k + c];
		}
	}
	return det;
}

/* det(C[tuple, :]) for every tuple; C is n_sites x k row-major. */
static void subset_dets(const double *C, uint32_t k, const uint32_t *tup,
	size_t m, double *out)
{
	double a[SPC_MAX_K * SPC_MAX_K];
	for (size_t i = 0; i < m; i++) {
		if (k == 0) {
			out[i] = 1.0;
			continue;
		}
		for (uint32_t r = 0; r < k; r++)
			memcpy(&a[r * k], &C[(size_t)tup[i * k + r] * k],
				sizeof(double) * k);
		out[i] = small_det(a, k);
	}
}

int state_prep_coeff_scratch_init(struct state_prep_coeff_scratch *sc,
	uint32_t n_sites, uint32_t n_alpha, uint32_t n_beta)
{
	memset(sc, 0, sizeof *sc);
	if (n_alpha > n_sites || n_beta > n_sites || n_alpha > SPC_MAX_K ||
		n_beta > SPC_MAX_K || n_sites > 32) {
		log_error("scratch_init: n_sites=%u n_alpha=%u n_beta=%u out of"
			  " range",
			n_sites, n_alpha, n_beta);
		return -1;
	}
	sc->n_sites = n_sites;
	sc->n_alpha = n_alpha;
	sc->n_beta = n_beta;
	sc->Ma = (size_t)choose(n_sites, n_alpha);
	sc->Mb = (size_t)choose(n_sites, n_beta);
	const uint32_t ka = n_alpha ? n_alpha : 1, kb = n_beta ? n_beta : 1;
	sc->tup_a = malloc(sizeof *sc->tup_a * sc->Ma * ka);
	sc->tup_b = malloc(sizeof *sc->tup_b * sc->Mb * kb);
	sc->det_a = malloc(sizeof *sc->det_a * sc->Ma);
	sc->det_b = malloc(sizeof *sc->det_b * sc->Mb);
	if (!sc->tup_a || !sc->tup_b || !sc->det_a || !sc->det_b ||
		lex_subsets(n_sites, n_alpha, sc->tup_a, sc->Ma) != sc->Ma ||
		lex_subsets(n_sites, n_beta, sc->tup_b, sc->Mb) != sc->Mb) {
		log_error("scratch_init: tuples failed");
		state_prep_coeff_scratch_free(sc);
		return -1;
	}
	return 0;
}

void state_prep_coeff_scratch_free(struct state_prep_coeff_scratch *sc)
{
	free(sc->tup_a);
	free(sc->tup_b);
	free(sc->det_a);
	free(sc->det_b);
	memset(sc, 0, sizeof *sc);
}

/* Occupation masks of the tuples: alpha in bits 0..n_sites-1, beta in
 * bits n_sites..2 n_sites-1 (state_prep_coeff.c:34-45). */
static uint64_t *occ_masks(const uint32_t *tup, size_t m, uint32_t k,
	uint32_t shift)
{
	uint64_t *o = malloc(sizeof *o * (m ? m : 1));
	if (!o)
		return NULL;
	for (size_t i = 0; i < m; i++) {
		uint64_t v = 0;
		for (uint32_t r = 0; r < k; r++)
			v |= UINT64_C(1) << (shift + tup[i * k + r]);
		o[i] = v;
	}
	return o;
}

/* The register must hold every index of the expansion. */
static int fits(const struct qreg *reg, const struct state_prep_coeff_scratch *sc,
	int tapered)
{
	const uint32_t need = tapered ? 2 * sc->n_sites - 2 : 2 * sc->n_sites;
	if (sc->n_sites == 0 || need > reg->qb_lo) {
		log_error("coeff state: %u sites%s need %u qubits, register has %u",
			sc->n_sites, tapered ? " (tapered)" : "", need,
			reg->qb_lo);
		return 0;
	}
	return 1;
}

/* Expand `ncomp` blocks (weights w[k], matrices Ca[k], Cb[k]) in one
 * device pass: amplitude = (existing, or none) + sum_k of the unpruned
 * w_k da_k db_k, in block order. */
static int expand_blocks(struct qreg *reg, struct state_prep_coeff_scratch *sc,
	const double *w, const double *const *Ca, const double *const *Cb,
	size_t ncomp, int tapered, int accumulate)
{
	if (!fits(reg, sc, tapered))
		return -1;
	struct p2_dev *d = p2_qreg_direct(reg);
	if (!d)
		return -1;
	uint64_t *oa = occ_masks(sc->tup_a, sc->Ma, sc->n_alpha, 0);
	uint64_t *ob = occ_masks(sc->tup_b, sc->Mb, sc->n_beta, sc->n_sites);
	double *da = malloc(sizeof *da * sc->Ma * (ncomp ? ncomp : 1));
	double *db = malloc(sizeof *db * sc->Mb * (ncomp ? ncomp : 1));
	int rc = -1;
	if (oa && ob && da && db) {
		for (size_t k = 0; k < ncomp; k++) {
			subset_dets(Ca[k], sc->n_alpha, sc->tup_a, sc->Ma,
				da + k * sc->Ma);
			subset_dets(Cb[k] ? Cb[k] : Ca[k], sc->n_beta,
				sc->tup_b, sc->Mb, db + k * sc->Mb);
		}
		/* the scratch holds the last block's determinants, as the
		 * reference's does after a call */
		if (ncomp) {
			memcpy(sc->det_a, da + (ncomp - 1) * sc->Ma,
				sizeof *da * sc->Ma);
			memcpy(sc->det_b, db + (ncomp - 1) * sc->Mb,
				sizeof *db * sc->Mb);
		}
		rc = p2d_cm_expand(d, sc->n_sites, tapered, accumulate, oa,
			sc->Ma, ob, sc->Mb, w, da, db, ncomp);
	}
	free(oa);
	free(ob);
	free(da);
	free(db);
	return rc < 0 ? p2_qreg_fail(reg) : 0;
}

int state_prep_coeff_expand(struct qreg *reg,
	struct state_prep_coeff_scratch *sc, const double *C_alpha,
	const double *C_beta, double weight, int tapered, int accumulate)
{
	return expand_blocks(reg, sc, &weight, &C_alpha, &C_beta, 1, tapered,
		accumulate);
}

int state_prep_coeff_expand_all(struct qreg *reg,
	struct state_prep_coeff_scratch *sc,
	const struct data_coeff_matrix *cm)
{
	qreg_zero(reg);
	if (cm->n_components == 0)
		return state_prep_coeff_expand(reg, sc, cm->C_alpha,
			cm->closed_shell ? NULL : cm->C_beta, 1.0, cm->tapered,
			0);
	const size_t n = cm->n_components;
	double *w = malloc(sizeof *w * n);
	const double **ca = malloc(sizeof *ca * n);
	const double **cb = malloc(sizeof *cb * n);
	int rc = -1;
	if (w && ca && cb) {
		for (size_t k = 0; k < n; k++) {
			w[k] = cm->blocks[k].cf;
			ca[k] = cm->blocks[k].C_alpha;
			cb[k] = cm->closed_shell ? NULL : cm->blocks[k].C_beta;
		}
		rc = expand_blocks(reg, sc, w, ca, cb, n, cm->tapered, 1);
	}
	free(w);
	free(ca);
	free(cb);
	return rc;
}

int state_prep_coeff_inner(struct qreg *reg,
	struct state_prep_coeff_scratch *sc, const double *C_alpha,
	const double *C_beta, double weight, int tapered, _Complex double *out)
{
	*out = 0.0;
	if (!fits(reg, sc, tapered))
		return -1;
	struct p2_dev *d = p2_qreg_direct(reg);
	if (!d)
		return -1;
	subset_dets(C_alpha, sc->n_alpha, sc->tup_a, sc->Ma, sc->det_a);
	subset_dets(C_beta ? C_beta : C_alpha, sc->n_beta, sc->tup_b, sc->Mb,
		sc->det_b);
	uint64_t *oa = occ_masks(sc->tup_a, sc->Ma, sc->n_alpha, 0);
	uint64_t *ob = occ_masks(sc->tup_b, sc->Mb, sc->n_beta, sc->n_sites);
	double z[2] = { 0.0, 0.0 };
	int rc = -1;
	if (oa && ob)
		rc = p2d_cm_inner(d, sc->n_sites, tapered, oa, sc->Ma, ob,
			sc->Mb, weight, sc->det_a, sc->det_b, z);
	free(oa);
	free(ob);
	if (rc < 0)
		return p2_qreg_fail(reg);
	double *o = (double *)out;
	o[0] = z[0];
	o[1] = z[1];
	return 0;
}
