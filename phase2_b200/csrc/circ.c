/*
 * circ.c -- circuit carriers, lifecycle, step and measure
 * (include/phase2/circ.h).  Same semantics as phase2/circ.c of
 * Quantum-for-Life/phase2 (lines 40-361) for the multi-determinant state:
 *
 *   circ_step_generic  phi = omega * cf per term, forward or reverse, fed
 *                      through the 1024-term batch cache to qreg_paulirot
 *                      (circ.c:256-280);
 *   circ_prepst        zero, then write each determinant in order
 *                      (circ.c:215-224);
 *   circ_measure       sum_d a[idx_d] * conj(cf_d) in determinant order
 *                      (circ.c:338-350), evaluated on the host from one
 *                      batched device gather, with the same expression so
 *                      the FP64 result is bit-identical.
 *
 * and for the coefficient-matrix state (state_prep.c, on the device):
 * circ_prepst expands it (circ.c:225-229), circ_measure sums the blocks'
 * inner products in order (circ.c:303-336).
 */
#include <complex.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "circ"
#include "log.h"

#include "circ_cache.h"
#include "phase2/circ.h"
#include "phase2_b200.h"

#include "p2_host.h"

int circ_hamil_init(struct circ_hamil *hm, uint32_t qb, size_t len)
{
	hm->terms = malloc(sizeof *hm->terms * (len ? len : 1));
	if (!hm->terms)
		return -1;
	hm->len = len;
	hm->qb = qb;
	return 0;
}

void circ_hamil_free(struct circ_hamil *hm)
{
	free(hm->terms);
	hm->terms = NULL;
	hm->len = 0;
}

static int term_cmp_lex(const void *a, const void *b)
{
	return paulis_cmp(((const struct circ_hamil_term *)a)->op,
		((const struct circ_hamil_term *)b)->op);
}

/* Same comparator and element size as circ_hamil_sort_lex in the reference
 * (phase2/circ.c:60-81), so qsort yields the same permutation. */
void circ_hamil_sort_lex(struct circ_hamil *hm)
{
	if (hm->len > 1)
		qsort(hm->terms, hm->len, sizeof *hm->terms, term_cmp_lex);
}

/* Stable sort by (flip, phase): ties keep their input order. */
void circ_hamil_sort_flip(struct circ_hamil *hm)
{
	const size_t n = hm->len;
	if (n < 2)
		return;
	struct circ_hamil_term *tmp = malloc(sizeof *tmp * n);
	if (!tmp) {
		log_error("circ_hamil_sort_flip: allocation failed");
		return;
	}
	/* bottom-up merge sort */
	struct circ_hamil_term *src = hm->terms, *dst = tmp;
	for (size_t w = 1; w < n; w *= 2) {
		for (size_t lo = 0; lo < n; lo += 2 * w) {
			const size_t mid = lo + w < n ? lo + w : n;
			const size_t hi = lo + 2 * w < n ? lo + 2 * w : n;
			size_t i = lo, j = mid, k = lo;
			while (i < mid && j < hi) {
				const struct paulis a = src[i].op, b = src[j].op;
				const int le = a.pak[0] < b.pak[0] ||
					(a.pak[0] == b.pak[0] &&
						a.pak[1] <= b.pak[1]);
				dst[k++] = le ? src[i++] : src[j++];
			}
			while (i < mid)
				dst[k++] = src[i++];
			while (j < hi)
				dst[k++] = src[j++];
		}
		struct circ_hamil_term *t = src;
		src = dst;
		dst = t;
	}
	if (src != hm->terms)
		memcpy(hm->terms, src, sizeof *tmp * n);
	free(tmp);
}

int circ_muldet_init(struct circ_muldet *md, size_t len)
{
	md->dets = malloc(sizeof *md->dets * (len ? len : 1));
	if (!md->dets)
		return -1;
	md->len = len;
	return 0;
}

void circ_muldet_free(struct circ_muldet *md)
{
	free(md->dets);
	md->dets = NULL;
	md->len = 0;
}

void data_coeff_matrix_free(struct data_coeff_matrix *cm)
{
	if (!cm)
		return;
	if (cm->blocks) {
		for (size_t k = 0; k < cm->n_components; k++) {
			free((void *)cm->blocks[k].C_alpha);
			free((void *)cm->blocks[k].C_beta);
		}
		free(cm->blocks);
	}
	free((void *)cm->C_alpha);
	free((void *)cm->C_beta);
	memset(cm, 0, sizeof *cm);
}

int circ_values_init(struct circ_values *vals, size_t len)
{
	vals->z = malloc(sizeof *vals->z * (len ? len : 1));
	if (!vals->z)
		return -1;
	vals->len = len;
	return 0;
}

void circ_values_free(struct circ_values *vals)
{
	free(vals->z);
	vals->z = NULL;
	vals->len = 0;
}

static void free_payload(struct circ *ct, enum stprep_kind kind)
{
	if (kind == STPREP_MULTIDET) {
		circ_muldet_free(&ct->md);
	} else if (kind == STPREP_COEFF_MATRIX) {
		data_coeff_matrix_free(&ct->cm);
		state_prep_coeff_scratch_free(&ct->sp_scratch);
	}
}

int circ_init(struct circ *ct, struct circ_hamil hm, enum stprep_kind sp_kind,
	const void *sp_data, size_t vals_len)
{
	memset(&ct->md, 0, sizeof ct->md);
	memset(&ct->cm, 0, sizeof ct->cm);
	memset(&ct->sp_scratch, 0, sizeof ct->sp_scratch);
	memset(&ct->reg, 0, sizeof ct->reg);
	memset(&ct->vals, 0, sizeof ct->vals);
	ct->cache = NULL;
	ct->hm = hm;
	ct->stprep_kind = sp_kind;

	switch (sp_kind) {
	case STPREP_MULTIDET:
		ct->md = *(const struct circ_muldet *)sp_data;
		break;
	case STPREP_COEFF_MATRIX:
		ct->cm = *(const struct data_coeff_matrix *)sp_data;
		if (state_prep_coeff_scratch_init(&ct->sp_scratch,
			    ct->cm.n_sites, ct->cm.n_alpha, ct->cm.n_beta) < 0) {
			log_error("circ_init: sp_scratch init failed");
			goto err;
		}
		break;
	default:
		log_error("circ_init: unknown state-prep kind %d", (int)sp_kind);
		goto err;
	}
	if (qreg_init(&ct->reg, ct->hm.qb) < 0) {
		log_error("circ_init: qreg_init failed");
		goto err;
	}
	ct->cache = circ_cache_init((int)ct->reg.qb_hi, (int)ct->reg.qb_lo);
	if (!ct->cache) {
		log_error("circ_init: cache_init failed");
		goto err_reg;
	}
	if (circ_values_init(&ct->vals, vals_len) < 0) {
		log_error("circ_init: values_init failed (len=%zu)", vals_len);
		goto err_cache;
	}
	return 0;

err_cache:
	circ_cache_free(ct->cache);
	ct->cache = NULL;
err_reg:
	qreg_free(&ct->reg);
err:
	free_payload(ct, sp_kind);
	circ_hamil_free(&ct->hm);
	return -1;
}

void circ_free(struct circ *ct)
{
	circ_values_free(&ct->vals);
	circ_hamil_free(&ct->hm);
	free_payload(ct, ct->stprep_kind);
	circ_cache_free(ct->cache);
	ct->cache = NULL;
	qreg_free(&ct->reg);
}

int circ_prepst(struct circ *ct)
{
	if (ct->stprep_kind == STPREP_COEFF_MATRIX)
		return state_prep_coeff_expand_all(&ct->reg, &ct->sp_scratch,
			&ct->cm);
	if (ct->stprep_kind != STPREP_MULTIDET)
		return -1;
	qreg_zero(&ct->reg);
	const struct circ_muldet *md = &ct->md;
	if (md->len == 0)
		return p2_qreg_error(&ct->reg);
	uint64_t *idx = malloc(sizeof *idx * md->len);
	_Complex double *z = malloc(sizeof *z * md->len);
	int rc = -1;
	if (idx && z) {
		for (size_t d = 0; d < md->len; d++) {
			idx[d] = md->dets[d].idx;
			z[d] = md->dets[d].cf;
		}
		rc = qreg_setamps(&ct->reg, idx, z, md->len);
	}
	free(idx);
	free(z);
	return rc;
}

static void circ_flush_cb(struct paulis code_hi, const struct paulis *codes_lo,
	double *phis, size_t ncodes, void *data)
{
	qreg_paulirot((struct qreg *)data, code_hi, codes_lo, phis, ncodes);
}

static int circ_step_generic(struct circ *ct, const struct circ_hamil *hm,
	double omega, int reverse)
{
	for (size_t i = 0; i < hm->len; i++) {
		const size_t j = reverse ? hm->len - 1 - i : i;
		const double phi = omega * hm->terms[j].cf;
		const struct paulis code = hm->terms[j].op;
		if (circ_cache_insert(ct->cache, code, phi) == 0)
			continue;
		circ_cache_flush(ct->cache, circ_flush_cb, &ct->reg);
		if (circ_cache_insert(ct->cache, code, phi) < 0)
			return -1;
	}
	circ_cache_flush(ct->cache, circ_flush_cb, &ct->reg);
	return p2_qreg_error(&ct->reg);
}

int circ_step(struct circ *ct, const struct circ_hamil *hm, double omega)
{
	return circ_step_generic(ct, hm, omega, 0);
}

int circ_step_reverse(struct circ *ct, const struct circ_hamil *hm,
	double omega)
{
	return circ_step_generic(ct, hm, omega, 1);
}

_Complex double p2_circ_overlap(const struct circ_muldet *md,
	const _Complex double *a)
{
	_Complex double pr = 0.0;
	for (size_t d = 0; d < md->len; d++)
		pr += a[d] * conj(md->dets[d].cf);
	return pr;
}

/* <trial | evolved> of a coefficient-matrix trial state: the single block,
 * or the sum over blocks in order (reference: circ.c:315-336). */
static _Complex double measure_coeff(struct circ *ct)
{
	const struct data_coeff_matrix *cm = &ct->cm;
	_Complex double pr = 0.0, z;
	if (cm->n_components == 0) {
		if (state_prep_coeff_inner(&ct->reg, &ct->sp_scratch,
			    cm->C_alpha, cm->closed_shell ? NULL : cm->C_beta,
			    1.0, cm->tapered, &z) == 0)
			pr = z;
		return pr;
	}
	for (size_t k = 0; k < cm->n_components; k++) {
		const struct data_coeff_block *b = &cm->blocks[k];
		if (state_prep_coeff_inner(&ct->reg, &ct->sp_scratch,
			    b->C_alpha, cm->closed_shell ? NULL : b->C_beta,
			    b->cf, cm->tapered, &z) < 0)
			z = 0.0;
		pr += z;
	}
	return pr;
}

_Complex double circ_measure(struct circ *ct)
{
	if (ct->stprep_kind == STPREP_COEFF_MATRIX)
		return measure_coeff(ct);
	if (ct->stprep_kind != STPREP_MULTIDET)
		return 0.0;
	const struct circ_muldet *md = &ct->md;
	_Complex double pr = 0.0;
	if (md->len == 0)
		return pr;
	uint64_t *idx = malloc(sizeof *idx * md->len);
	_Complex double *a = malloc(sizeof *a * md->len);
	if (!idx || !a) {
		free(idx);
		free(a);
		log_error("circ_measure: allocation failed");
		return 0.0;
	}
	for (size_t d = 0; d < md->len; d++)
		idx[d] = md->dets[d].idx;
	if (qreg_getamps(&ct->reg, idx, a, md->len) < 0)
		log_error("circ_measure: gather failed");
	else
		pr = p2_circ_overlap(md, a);
	free(idx);
	free(a);
	return pr;
}
