/*
 * drivers.c -- trott, trott2, qdrift and cmpsit (include/circ/ headers).  Same
 * step loops as circ/trott.c, circ/trott2.c, circ/qdrift.c and
 * circ/cmpsit.c of Quantum-for-Life/phase2:
 *
 *   trott   per step: circ_step(delta), measure            (trott.c:44-65)
 *   trott2  per step: circ_step(delta/2), circ_step_reverse(delta/2),
 *           measure                                        (trott2.c:44-74)
 *   qdrift  per sample: prepst, depth draws from the |c| CDF with
 *           cf = sign(c), circ_step(asin(step_size)), measure
 *                                                          (qdrift.c:95-134)
 *           (FP32 registers: the same loop with draws, plans and passes
 *           on the GPU, qdrift_simul_device)
 *   cmpsit  split by |c| (top `length` lex-sorted, rest sampled); per
 *           sample: prepst, per step a forward half of one sample and a
 *           reverse half of a fresh one at omega 0.5; measure
 *                                                          (cmpsit.c:65-235)
 *
 * Sampling uses the same generator, CDF and sign rule, so draws are
 * identical to the reference for equal seeds.  The deterministic term
 * order follows phase2_get_term_order() (lexicographic by default).
 */
#define _POSIX_C_SOURCE 200809L /* clock_gettime */

#include <complex.h>
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define LOG_SUBSYS "circ"
#include "log.h"

#include "circ/cmpsit.h"
#include "circ/qdrift.h"
#include "circ/trott.h"
#include "circ/trott2.h"
#include "phase2_b200.h"

#include "p2_host.h"

/* |a| < DBL_EPSILON -> 0, else -1 or +1 (circ/internal.h:26-32). */
static double sign_dz(double a)
{
	const double f = fabs(a);
	if (f < DBL_EPSILON)
		return 0.0;
	return a < f ? -1.0 : 1.0;
}

static void order_terms(struct circ_hamil *hm)
{
	switch (p2_cfg.order) {
	case PHASE2_ORDER_LEX:
		circ_hamil_sort_lex(hm);
		break;
	case PHASE2_ORDER_FLIP:
		circ_hamil_sort_flip(hm);
		break;
	default:
		break;
	}
}

static int emit(struct phase2_step_writer *sw, size_t i, _Complex double z)
{
	return (sw && sw->write(sw->ctx, i, z) < 0) ? -1 : 0;
}

/* ---- trott -------------------------------------------------------------- */

int trott_init(struct trott *tt, const struct trott_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw)
{
	if (circ_init(&tt->ct, hm, sp_kind, sp_data, dt->steps) < 0) {
		log_error("trott_init: circ_init failed");
		return -1;
	}
	tt->dt = *dt;
	tt->sw = sw;
	order_terms(&tt->ct.hm);
	return 0;
}

void trott_free(struct trott *tt)
{
	circ_free(&tt->ct);
}

int trott_simul(struct trott *tt)
{
	struct circ *ct = &tt->ct;
	struct circ_values *vals = &ct->vals;
	if (circ_prepst(ct) < 0)
		return -1;
	for (size_t i = 0; i < vals->len; i++) {
		if (circ_step(ct, &ct->hm, tt->dt.delta) < 0) {
			log_error("trott_simul: step %zu failed", i);
			return -1;
		}
		vals->z[i] = circ_measure(ct);
		if (p2_qreg_error(&ct->reg) < 0 || emit(tt->sw, i, vals->z[i]) < 0) {
			log_error("trott_simul: step %zu output failed", i);
			return -1;
		}
	}
	return 0;
}

/* ---- trott2 ------------------------------------------------------------- */

int trott2_init(struct trott2 *t2, const struct trott2_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw)
{
	if (circ_init(&t2->ct, hm, sp_kind, sp_data, dt->steps) < 0) {
		log_error("trott2_init: circ_init failed");
		return -1;
	}
	t2->dt = *dt;
	t2->sw = sw;
	order_terms(&t2->ct.hm);
	return 0;
}

void trott2_free(struct trott2 *t2)
{
	circ_free(&t2->ct);
}

int trott2_simul(struct trott2 *t2)
{
	struct circ *ct = &t2->ct;
	struct circ_values *vals = &ct->vals;
	const double half = t2->dt.delta / 2.0;
	if (circ_prepst(ct) < 0)
		return -1;
	for (size_t i = 0; i < vals->len; i++) {
		if (circ_step(ct, &ct->hm, half) < 0 ||
			circ_step_reverse(ct, &ct->hm, half) < 0) {
			log_error("trott2_simul: step %zu failed", i);
			return -1;
		}
		vals->z[i] = circ_measure(ct);
		if (p2_qreg_error(&ct->reg) < 0 || emit(t2->sw, i, vals->z[i]) < 0) {
			log_error("trott2_simul: step %zu output failed", i);
			return -1;
		}
	}
	return 0;
}

/* ---- qdrift ------------------------------------------------------------- */

/* Default seed, replaced by the last non-zero seed seen (circ/qdrift.c:30,
 * 72-75). */
static uint64_t QDRIFT_SEED = UINT64_C(0xeccd9dcc749fcdca);

int qdrift_init(struct qdrift *qd, const struct qdrift_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw)
{
	memset(&qd->ranct, 0, sizeof qd->ranct);
	if (circ_init(&qd->ct, hm, sp_kind, sp_data, dt->samples) < 0)
		return -1;
	qd->dt = *dt;
	qd->sw = sw;
	if (prob_cdf_init(&qd->ranct.cdf, qd->ct.hm.len) < 0 ||
		circ_hamil_init(&qd->ranct.hm_ran, qd->ct.hm.qb, dt->depth) <
			0) {
		prob_cdf_free(&qd->ranct.cdf);
		circ_free(&qd->ct);
		return -1;
	}
	prob_cdf_from_array_strided(&qd->ranct.cdf, &qd->ct.hm.terms[0].cf,
		sizeof qd->ct.hm.terms[0], NULL);
	if (qd->dt.seed != 0)
		QDRIFT_SEED = qd->dt.seed;
	else
		qd->dt.seed = QDRIFT_SEED;
	xoshiro256ss_init(&qd->rng, qd->dt.seed);
	return 0;
}

void qdrift_free(struct qdrift *qd)
{
	circ_hamil_free(&qd->ranct.hm_ran);
	prob_cdf_free(&qd->ranct.cdf);
	circ_free(&qd->ct);
}

static void qdrift_draw(struct qdrift *qd)
{
	struct circ_hamil *ran = &qd->ranct.hm_ran;
	for (size_t i = 0; i < ran->len; i++) {
		const double x = xoshiro256ss_dbl01(&qd->rng);
		const size_t k = prob_cdf_inverse(&qd->ranct.cdf, x);
		ran->terms[i].cf = sign_dz(qd->ct.hm.terms[k].cf);
		ran->terms[i].op = qd->ct.hm.terms[k].op;
	}
}

/* A register the persistent kernel runs: FP64 (exact form) or FP32
 * (either FP32 form); at most 31 qubits. */
static int persistent_reg_ok(const struct qreg *reg)
{
	const struct p2_qreg *b = reg->backend;
	return b && p2d_batch_ok(b->dev);
}

/* Registers that device sampling (p2d_sampled_device) takes under the
 * current mode: those the persistent kernel runs (FP64, or FP32 in either
 * form; at most 31 qubits) with a multi-determinant trial state; AUTO
 * also caps the width. */
/* Whether a sampled driver runs on the device.  In AUTO mode a run with a
 * step writer keeps the host loop, so the writer sees each sample as soon
 * as it completes (a writer that flushes per step stays crash-consistent);
 * ON runs such a run on the device too and calls the writer for every
 * sample, in order, after the launch. */
static int device_sampling_ok(const struct circ *ct,
	const struct phase2_step_writer *sw)
{
	const struct p2_qreg *b = ct->reg.backend;
	if (p2_cfg.device_sampling == PHASE2_DEVICE_SAMPLING_OFF ||
		(p2_cfg.device_sampling == PHASE2_DEVICE_SAMPLING_AUTO &&
			(ct->reg.qb_lo > PHASE2_DEVICE_SAMPLING_AUTO_QB || sw)))
		return 0;
	return b && b->rec == NULL && persistent_reg_ok(&ct->reg) &&
		ct->stprep_kind == STPREP_MULTIDET && ct->md.len > 0;
}

/*
 * A sampled driver run with the draws, plans and passes on the GPU.  The
 * caller fills job's depth, length, halves, reverse_odd and rphi; pool and
 * cdf are the drawable terms, head/hphi the head terms and their angles.
 * The host steps *rng to the start of every (sample, half) (depth draws
 * each) and lets last_half(obj) draw the final half itself, so the
 * generator and the driver's drawn terms end as the host loop leaves them;
 * each overlap is the host loop's expression over the gathered amplitudes.
 */
static int sampled_device(struct circ *ct, struct p2_smp_job *job,
	const struct circ_hamil *pool, const struct prob_cdf *cdf,
	const struct circ_hamil *head, const double *hphi,
	struct xoshiro256ss *rng, void (*last_half)(void *), void *obj,
	struct phase2_step_writer *sw, const char *who)
{
	struct circ_values *vals = &ct->vals;
	struct p2_qreg *b = ct->reg.backend;
	const size_t ns = vals->len, nh = job->halves;
	const size_t nt = cdf->len, nd = ct->md.len, nl = job->length;
	if (ns == 0)
		return 0;
	struct p2_dev *dev = p2_qreg_direct(&ct->reg);
	if (!dev)
		return -1;
	for (size_t d = 0; d < nd; d++)
		if (ct->md.dets[d].idx >= ct->reg.namp) {
			log_error("%s: determinant %llu out of range", who,
				(unsigned long long)ct->md.dets[d].idx);
			return p2_qreg_fail(&ct->reg);
		}
	uint64_t *rng0 = malloc(sizeof *rng0 * 4 * ns * nh);
	uint64_t *tfl = malloc(sizeof *tfl * (nt ? nt : 1));
	uint64_t *tph = malloc(sizeof *tph * (nt ? nt : 1));
	double *tcf = malloc(sizeof *tcf * (nt ? nt : 1));
	uint64_t *hfl = malloc(sizeof *hfl * (nl ? nl : 1));
	uint64_t *hph = malloc(sizeof *hph * (nl ? nl : 1));
	double *hcs = malloc(sizeof *hcs * 2 * (nl ? nl : 1));
	uint64_t *didx = malloc(sizeof *didx * nd);
	double *dval = malloc(sizeof *dval * 2 * nd);
	_Complex double *g = malloc(sizeof *g * ns * nd);
	int rc = -1;
	if (!rng0 || !tfl || !tph || !tcf || !hfl || !hph || !hcs || !didx ||
		!dval || !g) {
		log_error("%s: allocation failed", who);
		goto out;
	}
	for (size_t i = 0; i < ns * nh; i++) {
		memcpy(&rng0[4 * i], rng->s, sizeof rng->s);
		if (i + 1 == ns * nh)
			last_half(obj);
		else
			for (size_t k = 0; k < job->depth; k++)
				(void)xoshiro256ss_next(rng);
	}
	for (size_t k = 0; k < nt; k++) {
		tfl[k] = pool->terms[k].op.pak[0];
		tph[k] = pool->terms[k].op.pak[1];
		tcf[k] = pool->terms[k].cf;
	}
	for (size_t k = 0; k < nl; k++) {
		hfl[k] = head->terms[k].op.pak[0];
		hph[k] = head->terms[k].op.pak[1];
		hcs[2 * k] = cos(hphi[k]);
		hcs[2 * k + 1] = sin(hphi[k]);
	}
	for (size_t d = 0; d < nd; d++) {
		didx[d] = ct->md.dets[d].idx;
		dval[2 * d] = creal(ct->md.dets[d].cf);
		dval[2 * d + 1] = cimag(ct->md.dets[d].cf);
	}
	job->nqb = ct->reg.qb_lo;
	job->ndet = (uint32_t)nd;
	job->nterms = nt;
	job->mask = ct->reg.qb_lo >= 64 ? ~UINT64_C(0)
					: (UINT64_C(1) << ct->reg.qb_lo) - 1;
	for (int sg = 0; sg < 3; sg++) {
		job->rcs[sg][0] = cos(job->rphi[sg]);
		job->rcs[sg][1] = sin(job->rphi[sg]);
	}
	job->max_span = b->max_span;
	job->max_rots = b->max_rots;
	job->form = p2_form_for(b->prec);
	p2_sweep_for(job->nqb, job->form, &job->sweep_k, &job->sweep_low);
	uint64_t npass = 0;
	if (p2d_sampled_device(dev, job, rng0, ns, cdf->y, tfl, tph, tcf, hfl,
		    hph, hphi, hcs, didx, dval, (double *)g, &npass) < 0) {
		p2_qreg_fail(&ct->reg);
		goto out;
	}
	for (size_t i = 0; i < ns; i++) {
		vals->z[i] = p2_circ_overlap(&ct->md, g + i * nd);
		if (emit(sw, i, vals->z[i]) < 0) {
			log_error("%s: sample %zu output failed", who, i);
			goto out;
		}
	}
	rc = 0;
out:
	free(rng0);
	free(tfl);
	free(tph);
	free(tcf);
	free(hfl);
	free(hph);
	free(hcs);
	free(didx);
	free(dval);
	free(g);
	return rc;
}

static void qdrift_last_half(void *obj)
{
	qdrift_draw(obj);
}

/* qdrift_simul on the GPU: one forward half of `depth` draws per sample
 * at angle asin(step_size) * sign_dz(c), as the host loop applies them. */
static int qdrift_simul_device(struct qdrift *qd)
{
	struct p2_smp_job job;
	memset(&job, 0, sizeof job);
	job.depth = (uint32_t)qd->ranct.hm_ran.len;
	job.halves = 1;
	const double omega = asin(qd->dt.step_size);
	for (int sg = 0; sg < 3; sg++)
		job.rphi[sg] = omega * (double)(sg - 1);
	return sampled_device(&qd->ct, &job, &qd->ct.hm, &qd->ranct.cdf, NULL,
		NULL, &qd->rng, qdrift_last_half, qd, qd->sw, "qdrift_simul");
}

static int qdrift_device_ok(const struct qdrift *qd)
{
	return device_sampling_ok(&qd->ct, qd->sw) && qd->ranct.cdf.len > 0 &&
		qd->ranct.hm_ran.len > 0 &&
		qd->ranct.hm_ran.len < (UINT64_C(1) << 31);
}

int qdrift_simul(struct qdrift *qd)
{
	struct circ *ct = &qd->ct;
	struct circ_values *vals = &ct->vals;
	const double omega = asin(qd->dt.step_size);
	if (qdrift_device_ok(qd))
		return qdrift_simul_device(qd);
	for (size_t i = 0; i < vals->len; i++) {
		if (circ_prepst(ct) < 0)
			return -1;
		qdrift_draw(qd);
		if (circ_step(ct, &qd->ranct.hm_ran, omega) < 0) {
			log_error("qdrift_simul: sample %zu failed", i);
			return -1;
		}
		vals->z[i] = circ_measure(ct);
		if (p2_qreg_error(&ct->reg) < 0 || emit(qd->sw, i, vals->z[i]) < 0) {
			log_error("qdrift_simul: sample %zu output failed", i);
			return -1;
		}
	}
	return 0;
}

/* ---- cmpsit ------------------------------------------------------------- */

static uint64_t CMPSIT_SEED = UINT64_C(0xafb424901446f21f);

static int cmp_abscf_desc(const void *a, const void *b)
{
	const double x = fabs(((const struct circ_hamil_term *)a)->cf);
	const double y = fabs(((const struct circ_hamil_term *)b)->cf);
	return x > y ? -1 : (x < y ? 1 : 0);
}

static int cmpsit_split(struct cmpsit_ranct *rc, const struct circ_hamil *hm,
	const struct cmpsit_data *dt)
{
	if (dt->length > hm->len)
		return -1;
	struct circ_hamil tmp;
	if (circ_hamil_init(&tmp, hm->qb, hm->len) < 0)
		return -1;
	memcpy(tmp.terms, hm->terms, sizeof *tmp.terms * hm->len);
	qsort(tmp.terms, tmp.len, sizeof *tmp.terms, cmp_abscf_desc);
	const size_t nran = hm->len - dt->length;
	if (circ_hamil_init(&rc->hm_det, hm->qb, dt->length) < 0)
		goto fail_tmp;
	memcpy(rc->hm_det.terms, tmp.terms, sizeof *tmp.terms * dt->length);
	order_terms(&rc->hm_det);
	if (circ_hamil_init(&rc->hm_ran, hm->qb, nran) < 0)
		goto fail_det;
	memcpy(rc->hm_ran.terms, tmp.terms + dt->length,
		sizeof *tmp.terms * nran);
	if (prob_cdf_init(&rc->cdf, nran) < 0)
		goto fail_ran;
	prob_cdf_from_array_strided(&rc->cdf, &rc->hm_ran.terms[0].cf,
		sizeof rc->hm_ran.terms[0], &rc->lambda_r);
	rc->depth = dt->depth;
	rc->angle_rand = dt->angle_rand;
	circ_hamil_free(&tmp);
	return 0;
fail_ran:
	circ_hamil_free(&rc->hm_ran);
fail_det:
	circ_hamil_free(&rc->hm_det);
fail_tmp:
	circ_hamil_free(&tmp);
	return -1;
}

int cmpsit_ranct_init(struct cmpsit_ranct *rc, const struct circ_hamil *hm,
	const struct cmpsit_data *dt)
{
	memset(rc, 0, sizeof *rc);
	if (!hm || !dt || !hm->terms || dt->length >= hm->len) {
		log_error("cmpsit_ranct_init: needs more terms than length");
		return -1;
	}
	return cmpsit_split(rc, hm, dt);
}

void cmpsit_ranct_free(struct cmpsit_ranct *rc)
{
	circ_hamil_free(&rc->hm_smpl);
	circ_hamil_free(&rc->hm_ran);
	circ_hamil_free(&rc->hm_det);
	prob_cdf_free(&rc->cdf);
}

int cmpsit_init(struct cmpsit *cp, const struct cmpsit_data *dt,
	struct circ_hamil hm, enum stprep_kind sp_kind, const void *sp_data,
	struct phase2_step_writer *sw)
{
	memset(&cp->ranct, 0, sizeof cp->ranct);
	if (circ_init(&cp->ct, hm, sp_kind, sp_data, dt->samples) < 0)
		return -1;
	cp->dt = *dt;
	cp->sw = sw;
	if (cmpsit_split(&cp->ranct, &cp->ct.hm, dt) < 0) {
		circ_free(&cp->ct);
		return -1;
	}
	if (cp->dt.seed != 0)
		CMPSIT_SEED = cp->dt.seed;
	else
		cp->dt.seed = CMPSIT_SEED;
	xoshiro256ss_init(&cp->rng, cp->dt.seed);
	return 0;
}

void cmpsit_free(struct cmpsit *cp)
{
	circ_hamil_free(&cp->ranct.hm_smpl);
	circ_hamil_free(&cp->ranct.hm_ran);
	circ_hamil_free(&cp->ranct.hm_det);
	prob_cdf_free(&cp->ranct.cdf);
	circ_free(&cp->ct);
}

/* One composite sample: deterministic head at angle_det * c, then `depth`
 * draws at sign(c) * angle_rand (circ/cmpsit.c:151-177). */
static int cmpsit_sample(struct cmpsit *cp)
{
	struct cmpsit_ranct *rc = &cp->ranct;
	const size_t len = cp->dt.length + rc->depth;
	if (!rc->hm_smpl.terms || rc->hm_smpl.len != len) {
		circ_hamil_free(&rc->hm_smpl);
		if (circ_hamil_init(&rc->hm_smpl, cp->ct.hm.qb, len) < 0)
			return -1;
	}
	for (size_t i = 0; i < cp->dt.length; i++) {
		rc->hm_smpl.terms[i].op = rc->hm_det.terms[i].op;
		rc->hm_smpl.terms[i].cf = rc->hm_det.terms[i].cf * cp->dt.angle_det;
	}
	const double tau = rc->angle_rand;
	for (size_t i = cp->dt.length; i < len; i++) {
		const double x = xoshiro256ss_dbl01(&cp->rng);
		const size_t k = prob_cdf_inverse(&rc->cdf, x);
		rc->hm_smpl.terms[i].op = rc->hm_ran.terms[k].op;
		rc->hm_smpl.terms[i].cf = sign_dz(rc->hm_ran.terms[k].cf) * tau;
	}
	return 0;
}

static void cmpsit_last_half(void *obj)
{
	(void)cmpsit_sample(obj);
}

/* cmpsit_simul on the GPU: per step a forward half (head at
 * 0.5 * (c * angle_det), then depth draws at 0.5 * (sign_dz(c) * tau))
 * and a reversed half of fresh draws, as the host loop applies them. */
static int cmpsit_simul_device(struct cmpsit *cp)
{
	struct cmpsit_ranct *rc = &cp->ranct;
	const size_t nl = cp->dt.length;
	double *hphi = malloc(sizeof *hphi * (nl ? nl : 1));
	if (!hphi)
		return -1;
	for (size_t k = 0; k < nl; k++)
		hphi[k] = 0.5 * (rc->hm_det.terms[k].cf * cp->dt.angle_det);
	struct p2_smp_job job;
	memset(&job, 0, sizeof job);
	job.depth = (uint32_t)rc->depth;
	job.length = (uint32_t)nl;
	job.halves = (uint32_t)(2 * cp->dt.steps);
	job.reverse_odd = 1;
	for (int sg = 0; sg < 3; sg++)
		job.rphi[sg] = 0.5 * ((double)(sg - 1) * rc->angle_rand);
	const int r = sampled_device(&cp->ct, &job, &rc->hm_ran, &rc->cdf,
		&rc->hm_det, hphi, &cp->rng, cmpsit_last_half, cp, cp->sw,
		"cmpsit_simul");
	free(hphi);
	return r;
}

static int cmpsit_device_ok(const struct cmpsit *cp)
{
	const uint64_t T = 2 * (uint64_t)cp->dt.steps *
		((uint64_t)cp->dt.length + cp->ranct.depth);
	return device_sampling_ok(&cp->ct, cp->sw) && cp->dt.steps > 0 &&
		cp->dt.steps < (UINT64_C(1) << 30) &&
		cp->ranct.depth < (UINT64_C(1) << 31) &&
		cp->dt.length < (UINT64_C(1) << 31) &&
		(cp->ranct.depth == 0 || cp->ranct.cdf.len > 0) &&
		T < (UINT64_C(1) << 31);
}

int cmpsit_simul(struct cmpsit *cp)
{
	struct circ *ct = &cp->ct;
	struct circ_values *vals = &ct->vals;
	if (cmpsit_device_ok(cp))
		return cmpsit_simul_device(cp);
	for (size_t i = 0; i < vals->len; i++) {
		if (circ_prepst(ct) < 0)
			return -1;
		for (size_t s = 0; s < cp->dt.steps; s++) {
			if (cmpsit_sample(cp) < 0 ||
				circ_step(ct, &cp->ranct.hm_smpl, 0.5) < 0)
				return -1;
			if (cmpsit_sample(cp) < 0 ||
				circ_step_reverse(ct, &cp->ranct.hm_smpl, 0.5) <
					0)
				return -1;
		}
		vals->z[i] = circ_measure(ct);
		if (p2_qreg_error(&ct->reg) < 0 || emit(cp->sw, i, vals->z[i]) < 0) {
			log_error("cmpsit_simul: sample %zu output failed", i);
			return -1;
		}
	}
	return 0;
}

/* ---- batched drivers (include/phase2_b200.h) ---------------------------- */

/* One instance of a batch: its circuit, writer, the next output slot, and
 * the function that queues the work producing output slot `idx`. */
struct batch_item {
	void *obj;
	struct circ *ct;
	struct phase2_step_writer *sw;
	int (*enqueue)(void *obj, size_t idx);
	size_t next;
	int failed;
};

static int trott_enqueue(void *obj, size_t idx)
{
	struct trott *tt = obj;
	if (idx == 0 && circ_prepst(&tt->ct) < 0)
		return -1;
	return circ_step(&tt->ct, &tt->ct.hm, tt->dt.delta);
}

static int trott2_enqueue(void *obj, size_t idx)
{
	struct trott2 *t2 = obj;
	const double half = t2->dt.delta / 2.0;
	if (idx == 0 && circ_prepst(&t2->ct) < 0)
		return -1;
	if (circ_step(&t2->ct, &t2->ct.hm, half) < 0)
		return -1;
	return circ_step_reverse(&t2->ct, &t2->ct.hm, half);
}

static int qdrift_enqueue(void *obj, size_t idx)
{
	struct qdrift *qd = obj;
	(void)idx;
	if (circ_prepst(&qd->ct) < 0)
		return -1;
	qdrift_draw(qd);
	return circ_step(&qd->ct, &qd->ranct.hm_ran, asin(qd->dt.step_size));
}

static int cmpsit_enqueue(void *obj, size_t idx)
{
	struct cmpsit *cp = obj;
	(void)idx;
	if (circ_prepst(&cp->ct) < 0)
		return -1;
	for (size_t s = 0; s < cp->dt.steps; s++) {
		if (cmpsit_sample(cp) < 0 ||
			circ_step(&cp->ct, &cp->ranct.hm_smpl, 0.5) < 0)
			return -1;
		if (cmpsit_sample(cp) < 0 ||
			circ_step_reverse(&cp->ct, &cp->ranct.hm_smpl, 0.5) < 0)
			return -1;
	}
	return 0;
}

static void batch_launch(struct batch_item *it)
{
	if (it->enqueue(it->obj, it->next) < 0 || qreg_flush(&it->ct->reg) < 0) {
		log_error("batch: instance failed at output %zu", it->next);
		it->failed = 1;
	}
}

/*
 * One persistent launch for the whole batch: each instance's work is
 * recorded as a program
 * (its enqueue calls, then a gather of its determinant amplitudes per
 * output), all programs run in p2d_batch_run, and every output is then
 * formed on the host from its gathered amplitudes with circ_measure's
 * expression.  Instances whose recording fails are left out and reported.
 */
/* Record instance i's program (all its outputs): its enqueue calls, then a
 * gather of the determinant amplitudes per output (gat[k]: output index of
 * output k's first amplitude).  Touches only the instance's own objects
 * and no device state, so instances record in parallel. */
static void record_one(struct batch_item *it, struct p2_prog *pg, long **gat)
{
	struct qreg *reg = &it->ct->reg;
	const struct circ_muldet *md = &it->ct->md;
	const size_t len = it->ct->vals.len;
	uint64_t *didx = malloc(sizeof *didx * (md->len ? md->len : 1));
	*gat = malloc(sizeof **gat * (len ? len : 1));
	if (!didx || !*gat || p2_qreg_record(reg, pg) < 0) {
		free(didx);
		it->failed = 1;
		return;
	}
	for (size_t d = 0; d < md->len; d++)
		didx[d] = md->dets[d].idx;
	for (size_t k = 0; k < len && !it->failed; k++) {
		if (it->enqueue(it->obj, k) < 0)
			it->failed = 1;
		else if (((*gat)[k] = p2_qreg_record_gather(reg, didx,
				  md->len)) < 0)
			it->failed = 1;
	}
	free(didx);
	if (p2_qreg_record_end(reg) < 0)
		it->failed = 1;
}

struct record_pool {
	struct batch_item *items;
	struct p2_prog *progs;
	long **gat;
	size_t n;
	size_t next; /* next instance to record (atomic) */
};

static void *record_worker(void *arg)
{
	struct record_pool *rp = arg;
	for (;;) {
		const size_t i = __atomic_fetch_add(&rp->next, 1,
			__ATOMIC_RELAXED);
		if (i >= rp->n)
			return NULL;
		record_one(&rp->items[i], &rp->progs[i], &rp->gat[i]);
	}
}

/* Host threads that record a batch: one per instance up to 16. */
#define P2_RECORD_THREADS 16

static void record_all(struct batch_item *items, struct p2_prog *progs,
	long **gat, size_t n)
{
	struct record_pool rp = { items, progs, gat, n, 0 };
	pthread_t th[P2_RECORD_THREADS];
	size_t nt = n < P2_RECORD_THREADS ? n : P2_RECORD_THREADS, started = 0;
	for (size_t k = 1; k < nt; k++)
		if (pthread_create(&th[started], NULL, record_worker, &rp) == 0)
			started++;
	record_worker(&rp);
	for (size_t k = 0; k < started; k++)
		pthread_join(th[k], NULL);
}

static double wall_s(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static int run_batch_persistent(struct batch_item *items, size_t n)
{
	const double t0 = wall_s();
	struct p2_prog *progs = calloc(n, sizeof *progs);
	const struct p2_prog **pp = calloc(n, sizeof *pp);
	struct p2_dev **devs = calloc(n, sizeof *devs);
	long **gat = calloc(n, sizeof *gat);
	size_t *who = calloc(n, sizeof *who);
	double *gout = NULL;
	int rc = -1;
	if (!progs || !pp || !devs || !gat || !who)
		goto out;
	record_all(items, progs, gat, n);
	const double t1 = wall_s();
	size_t m = 0, ng = 0;
	for (size_t i = 0; i < n; i++) {
		struct batch_item *it = &items[i];
		if (it->failed) {
			log_error("batch: instance %zu could not be recorded", i);
			continue;
		}
		devs[m] = p2_qreg_dev(&it->ct->reg);
		pp[m] = &progs[i];
		who[m++] = i;
		ng += progs[i].ng;
	}
	gout = malloc(sizeof(double) * 2 * (ng ? ng : 1));
	if (!gout)
		goto out;
	double kms = 0.0;
	if (p2d_batch_run(devs, pp, m, gout, &kms) < 0) {
		for (size_t j = 0; j < m; j++)
			items[who[j]].failed = 1;
		goto out;
	}
	(void)p2_batch_finish_map(who, m, n);
	if (getenv("PHASE2_BATCH_TIMING"))
		log_info("batch: %zu programs, record %.3f s, launch+copy %.3f s"
			 " (kernel %.3f s)",
			m, t1 - t0, wall_s() - t1, kms / 1e3);
	size_t base = 0;
	for (size_t j = 0; j < m; j++) {
		struct batch_item *it = &items[who[j]];
		struct circ_values *vals = &it->ct->vals;
		for (size_t k = 0; k < vals->len; k++) {
			const _Complex double *a = (const _Complex double *)(gout +
				2 * (base + (size_t)gat[who[j]][k]));
			vals->z[k] = p2_circ_overlap(&it->ct->md, a);
			if (emit(it->sw, k, vals->z[k]) < 0) {
				it->failed = 1;
				break;
			}
		}
		base += pp[j]->ng;
	}
	rc = 0;
out:
	for (size_t i = 0; i < n; i++) {
		if (progs)
			p2_prog_free(&progs[i]);
		if (gat)
			free(gat[i]);
		if (rc < 0)
			items[i].failed = 1;
	}
	free(progs);
	free(pp);
	free(devs);
	free(gat);
	free(who);
	free(gout);
	for (size_t i = 0; i < n; i++)
		if (items[i].failed)
			rc = -1;
	return rc;
}

/* Whether every instance can run in one persistent launch (registers of
 * one precision). */
static int batch_persistent_ok(const struct batch_item *items, size_t n)
{
	if (!p2_cfg.batch_persistent)
		return 0;
	for (size_t i = 0; i < n; i++) {
		const struct qreg *reg = &items[i].ct->reg;
		if (!persistent_reg_ok(reg) ||
			items[i].ct->stprep_kind != STPREP_MULTIDET ||
			((const struct p2_qreg *)reg->backend)->prec !=
				((const struct p2_qreg *)items[0].ct->reg.backend)
					->prec)
			return 0;
	}
	return 1;
}

/* Queue output 0 everywhere, then repeatedly read each instance's pending
 * output and immediately queue its next one. */
static int run_batch_streams(struct batch_item *items, size_t n)
{
	for (size_t i = 0; i < n; i++)
		if (items[i].ct->vals.len > 0)
			batch_launch(&items[i]);
	int active = 1;
	while (active) {
		active = 0;
		for (size_t i = 0; i < n; i++) {
			struct batch_item *it = &items[i];
			struct circ_values *vals = &it->ct->vals;
			if (it->failed || it->next >= vals->len)
				continue;
			active = 1;
			vals->z[it->next] = circ_measure(it->ct);
			if (p2_qreg_error(&it->ct->reg) < 0 ||
				emit(it->sw, it->next, vals->z[it->next]) < 0) {
				it->failed = 1;
				continue;
			}
			if (++it->next < vals->len)
				batch_launch(it);
		}
	}
	int rc = 0;
	for (size_t i = 0; i < n; i++)
		if (items[i].failed)
			rc = -1;
	return rc;
}

#define BATCH_ENTRY(NAME, TYPE, ENQ)                                           \
	int NAME(TYPE *const *objs, size_t n)                                  \
	{                                                                      \
		if (n == 0)                                                    \
			return 0;                                              \
		struct batch_item *items = calloc(n, sizeof *items);           \
		if (!items)                                                    \
			return -1;                                             \
		p2_batch_finish_reset();                                       \
		for (size_t i = 0; i < n; i++) {                               \
			items[i].obj = objs[i];                                \
			items[i].ct = &objs[i]->ct;                            \
			items[i].sw = objs[i]->sw;                             \
			items[i].enqueue = ENQ;                                \
		}                                                              \
		const int rc = batch_persistent_ok(items, n)                   \
			? run_batch_persistent(items, n)                       \
			: run_batch_streams(items, n);                         \
		free(items);                                                   \
		return rc;                                                     \
	}

BATCH_ENTRY(trott_simul_batch, struct trott, trott_enqueue)
BATCH_ENTRY(trott2_simul_batch, struct trott2, trott2_enqueue)
BATCH_ENTRY(qdrift_simul_batch, struct qdrift, qdrift_enqueue)
BATCH_ENTRY(cmpsit_simul_batch, struct cmpsit, cmpsit_enqueue)
