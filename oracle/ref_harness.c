/*
 * ref_harness.c -- flat entry points over the reference's own CPU path
 * (TEST INFRASTRUCTURE ONLY).
 *
 * Compiled against the reference headers and linked with the reference
 * objects into oracle/_ref/libphase2_ref.so.  Python (tests/golden/
 * make_golden.py and the not-gpu pin tests) calls these to obtain answers
 * from the unmodified reference code: qreg_paulirot (phase2/qreg.c:135-142),
 * trott_simul (circ/trott.c:44-65), trott2_simul (circ/trott2.c:44-74),
 * qdrift_simul (circ/qdrift.c:105-134), cmpsit_simul (circ/cmpsit.c:208-235),
 * and the coefficient-matrix state prep and overlap
 * (phase2/state_prep_coeff.c:156-325).
 *
 * Term records use the reference layout struct circ_hamil_term
 * {double cf; struct paulis op;} (include/phase2/circ.h:48-55).
 */
#include "c23_compat.h"
#include <complex.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "circ/cmpsit.h"
#include "circ/qdrift.h"
#include "circ/trott.h"
#include "circ/trott2.h"
#include "phase2.h"
#include "phase2/state_prep_coeff.h"

#include "circ_cache.h"

#define HARNESS_WORLD_SEED UINT64_C(0x5a17c0de2b9d4e61)

static int ensure_world(void)
{
	struct world_info wd;
	if (world_info(&wd) == WORLD_READY)
		return 0;
	return world_init(NULL, NULL, HARNESS_WORLD_SEED) == WORLD_READY ? 0
									 : -1;
}

/*
 * Amplitude capture: refh_capture arms it, and the next driver run
 * (refh_trott, refh_qdrift, refh_cmpsit) samples its register's final
 * state before freeing it, into caller buffers of `cap` entries:
 * stride > 0 takes indices 0, stride, 2 stride, ...; stride == 0 takes the
 * non-zero amplitudes in index order.  refh_captured returns the entries
 * written.  The reference keeps the whole state on one rank here.
 */
static struct {
	int on;
	uint64_t stride;
	size_t cap, got;
	uint64_t *idx;
	double *amp;
} CAP;

int refh_capture(uint64_t stride, size_t cap, uint64_t *idx, double *amp)
{
	CAP.on = 1;
	CAP.stride = stride;
	CAP.cap = cap;
	CAP.got = 0;
	CAP.idx = idx;
	CAP.amp = amp;
	return 0;
}

size_t refh_captured(void)
{
	return CAP.got;
}

static void capture(const struct qreg *reg)
{
	if (!CAP.on)
		return;
	CAP.on = 0;
	CAP.got = 0;
	for (uint64_t i = 0; i < reg->namp && CAP.got < CAP.cap;
		i += CAP.stride ? CAP.stride : 1) {
		const _Complex double z = reg->amp[i];
		if (!CAP.stride && z == 0)
			continue;
		CAP.idx[CAP.got] = i;
		CAP.amp[2 * CAP.got] = creal(z);
		CAP.amp[2 * CAP.got + 1] = cimag(z);
		CAP.got++;
	}
}

/* amp: 2*2^nqb doubles, in/out.  Applies the n rotations with one
 * qreg_paulirot call per 1024-term batch, as the batch cache would. */
int refh_paulirot(uint32_t nqb, double *amp, const uint64_t *flip,
	const uint64_t *phase, const double *phi, size_t n)
{
	if (ensure_world() < 0)
		return -1;
	struct qreg reg;
	if (qreg_init(&reg, nqb) < 0)
		return -1;
	const uint64_t namp = UINT64_C(1) << nqb;
	for (uint64_t i = 0; i < namp; i++)
		reg.amp[i] = CMPLX(amp[2 * i], amp[2 * i + 1]);
	struct paulis *lo = malloc(sizeof *lo * (n ? n : 1));
	if (!lo) {
		qreg_free(&reg);
		return -1;
	}
	for (size_t k = 0; k < n; k++) {
		lo[k].pak[0] = flip[k];
		lo[k].pak[1] = phase[k];
	}
	const struct paulis hi = paulis_new();
	for (size_t k = 0; k < n; k += 1024) {
		const size_t m = n - k < 1024 ? n - k : 1024;
		qreg_paulirot(&reg, hi, lo + k, phi + k, m);
	}
	for (uint64_t i = 0; i < namp; i++) {
		amp[2 * i] = creal(reg.amp[i]);
		amp[2 * i + 1] = cimag(reg.amp[i]);
	}
	free(lo);
	qreg_free(&reg);
	return 0;
}

static int load_hamil(struct circ_hamil *hm, uint32_t nqb, const void *terms,
	size_t nterms)
{
	if (circ_hamil_init(hm, nqb, nterms ? nterms : 1) < 0)
		return -1;
	hm->len = nterms;
	memcpy(hm->terms, terms, sizeof hm->terms[0] * nterms);
	return 0;
}

static int load_muldet(struct circ_muldet *md, size_t ndets,
	const uint64_t *idx, const double *cf)
{
	if (circ_muldet_init(md, ndets) < 0)
		return -1;
	for (size_t d = 0; d < ndets; d++) {
		md->dets[d].idx = idx[d];
		md->dets[d].cf = CMPLX(cf[2 * d], cf[2 * d + 1]);
	}
	return 0;
}

static void store_vals(const struct circ_values *v, double *out)
{
	for (size_t i = 0; i < v->len; i++) {
		out[2 * i] = creal(v->z[i]);
		out[2 * i + 1] = cimag(v->z[i]);
	}
}

/* order2 = 0: trott, 1: trott2.  sort_lex = 1 goes through *_init (which
 * lex-sorts); 0 builds the struct by hand in the given order, as
 * test/t-circ_trott.c:162-201 does. */
int refh_trott(int order2, uint32_t nqb, const void *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t steps, double delta, int sort_lex, double *out_z)
{
	if (ensure_world() < 0)
		return -1;
	struct circ_hamil hm;
	struct circ_muldet md;
	if (load_hamil(&hm, nqb, terms, nterms) < 0)
		return -1;
	if (load_muldet(&md, ndets, det_idx, det_cf) < 0)
		return -1;
	int rc;
	if (order2) {
		struct trott2 t2;
		memset(&t2, 0, sizeof t2);
		const struct trott2_data dt = { .steps = steps, .delta = delta };
		if (sort_lex) {
			if (trott2_init(&t2, &dt, hm, STPREP_MULTIDET, &md,
				    NULL) < 0)
				return -1;
		} else {
			t2.ct.hm = hm;
			t2.ct.md = md;
			t2.ct.stprep_kind = STPREP_MULTIDET;
			if (qreg_init(&t2.ct.reg, nqb) < 0)
				return -1;
			t2.ct.cache = circ_cache_init(t2.ct.reg.qb_hi,
				t2.ct.reg.qb_lo);
			circ_values_init(&t2.ct.vals, steps);
			t2.dt = dt;
		}
		rc = trott2_simul(&t2);
		store_vals(&t2.ct.vals, out_z);
		capture(&t2.ct.reg);
		trott2_free(&t2);
	} else {
		struct trott tt;
		memset(&tt, 0, sizeof tt);
		const struct trott_data dt = { .steps = steps, .delta = delta };
		if (sort_lex) {
			if (trott_init(&tt, &dt, hm, STPREP_MULTIDET, &md,
				    NULL) < 0)
				return -1;
		} else {
			tt.ct.hm = hm;
			tt.ct.md = md;
			tt.ct.stprep_kind = STPREP_MULTIDET;
			if (qreg_init(&tt.ct.reg, nqb) < 0)
				return -1;
			tt.ct.cache = circ_cache_init(tt.ct.reg.qb_hi,
				tt.ct.reg.qb_lo);
			circ_values_init(&tt.ct.vals, steps);
			tt.dt = dt;
		}
		rc = trott_simul(&tt);
		store_vals(&tt.ct.vals, out_z);
		capture(&tt.ct.reg);
		trott_free(&tt);
	}
	return rc;
}

int refh_qdrift(uint32_t nqb, const void *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t samples, size_t depth, double step_size, uint64_t seed,
	double *out_z)
{
	if (ensure_world() < 0)
		return -1;
	struct circ_hamil hm;
	struct circ_muldet md;
	if (load_hamil(&hm, nqb, terms, nterms) < 0)
		return -1;
	if (load_muldet(&md, ndets, det_idx, det_cf) < 0)
		return -1;
	struct qdrift qd;
	memset(&qd, 0, sizeof qd);
	const struct qdrift_data dt = { .samples = samples, .depth = depth,
		.step_size = step_size, .seed = seed };
	if (qdrift_init(&qd, &dt, hm, STPREP_MULTIDET, &md, NULL) < 0)
		return -1;
	const int rc = qdrift_simul(&qd);
	store_vals(&qd.ct.vals, out_z);
	capture(&qd.ct.reg);
	qdrift_free(&qd);
	return rc;
}

int refh_cmpsit(uint32_t nqb, const void *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t samples, size_t steps, size_t length, size_t depth,
	double angle_det, double angle_rand, uint64_t seed, double *out_z)
{
	if (ensure_world() < 0)
		return -1;
	struct circ_hamil hm;
	struct circ_muldet md;
	if (load_hamil(&hm, nqb, terms, nterms) < 0)
		return -1;
	if (load_muldet(&md, ndets, det_idx, det_cf) < 0)
		return -1;
	struct cmpsit cp;
	memset(&cp, 0, sizeof cp);
	const struct cmpsit_data dt = { .samples = samples, .steps = steps,
		.length = length, .depth = depth, .angle_det = angle_det,
		.angle_rand = angle_rand, .seed = seed };
	if (cmpsit_init(&cp, &dt, hm, STPREP_MULTIDET, &md, NULL) < 0)
		return -1;
	const int rc = cmpsit_simul(&cp);
	store_vals(&cp.ct.vals, out_z);
	capture(&cp.ct.reg);
	cmpsit_free(&cp);
	return rc;
}

/*
 * Coefficient-matrix trial state (phase2/state_prep_coeff.c:156-325) on an
 * nqb-qubit reference register.  Blocks: ncomp weights w and matrices
 * Ca[k*n_sites*na ...], Cb[k*n_sites*nb ...] (Cb NULL = closed shell).
 * ncomp == 0 means one block of weight 1.0 carried by Ca/Cb (the
 * single-block case of data_coeff_matrix).
 *
 * refh_coeff_expand_all: the state after state_prep_coeff_expand_all
 * (2*2^nqb doubles out).
 * refh_coeff_inner: amp (in) is loaded into the register, then the sum of
 * state_prep_coeff_inner over the blocks in order, as circ.c measure_coeff
 * does (out: 2 doubles).
 */
static void fill_cm(struct data_coeff_matrix *cm, struct data_coeff_block *bl,
	uint32_t nqb, uint32_t n_sites, uint32_t na, uint32_t nb, int tapered,
	size_t ncomp, const double *w, const double *Ca, const double *Cb)
{
	memset(cm, 0, sizeof *cm);
	cm->nqb = nqb;
	cm->n_sites = n_sites;
	cm->n_alpha = na;
	cm->n_beta = nb;
	cm->closed_shell = Cb == NULL;
	cm->tapered = tapered;
	cm->n_components = ncomp;
	if (ncomp == 0) {
		cm->C_alpha = Ca;
		cm->C_beta = Cb;
		return;
	}
	for (size_t k = 0; k < ncomp; k++) {
		bl[k].cf = w[k];
		bl[k].C_alpha = Ca + k * (size_t)n_sites * na;
		bl[k].C_beta = Cb ? Cb + k * (size_t)n_sites * nb : NULL;
	}
	cm->blocks = bl;
}

int refh_coeff_expand_all(uint32_t nqb, uint32_t n_sites, uint32_t na,
	uint32_t nb, int tapered, size_t ncomp, const double *w,
	const double *Ca, const double *Cb, double *amp)
{
	if (ensure_world() < 0)
		return -1;
	struct qreg reg;
	if (qreg_init(&reg, nqb) < 0)
		return -1;
	struct data_coeff_block *bl = calloc(ncomp ? ncomp : 1, sizeof *bl);
	struct data_coeff_matrix cm;
	struct state_prep_coeff_scratch sc;
	int rc = -1;
	if (bl && state_prep_coeff_scratch_init(&sc, n_sites, na, nb) == 0) {
		fill_cm(&cm, bl, nqb, n_sites, na, nb, tapered, ncomp, w, Ca,
			Cb);
		rc = state_prep_coeff_expand_all(&reg, &sc, &cm);
		for (uint64_t i = 0; i < reg.namp; i++) {
			amp[2 * i] = creal(reg.amp[i]);
			amp[2 * i + 1] = cimag(reg.amp[i]);
		}
		state_prep_coeff_scratch_free(&sc);
	}
	free(bl);
	qreg_free(&reg);
	return rc;
}

int refh_coeff_inner(uint32_t nqb, uint32_t n_sites, uint32_t na,
	uint32_t nb, int tapered, size_t ncomp, const double *w,
	const double *Ca, const double *Cb, const double *amp, double *out)
{
	if (ensure_world() < 0)
		return -1;
	struct qreg reg;
	if (qreg_init(&reg, nqb) < 0)
		return -1;
	for (uint64_t i = 0; i < reg.namp; i++)
		reg.amp[i] = CMPLX(amp[2 * i], amp[2 * i + 1]);
	struct data_coeff_block *bl = calloc(ncomp ? ncomp : 1, sizeof *bl);
	struct data_coeff_matrix cm;
	struct state_prep_coeff_scratch sc;
	int rc = -1;
	if (bl && state_prep_coeff_scratch_init(&sc, n_sites, na, nb) == 0) {
		fill_cm(&cm, bl, nqb, n_sites, na, nb, tapered, ncomp, w, Ca,
			Cb);
		_Complex double pr = 0.0, z = 0.0;
		rc = 0;
		if (ncomp == 0) {
			rc = state_prep_coeff_inner(&reg, &sc, Ca, Cb, 1.0,
				tapered, &z);
			pr = z;
		} else {
			for (size_t k = 0; k < ncomp && rc == 0; k++) {
				rc = state_prep_coeff_inner(&reg, &sc,
					bl[k].C_alpha, bl[k].C_beta, bl[k].cf,
					tapered, &z);
				pr += z;
			}
		}
		out[0] = creal(pr);
		out[1] = cimag(pr);
		state_prep_coeff_scratch_free(&sc);
	}
	free(bl);
	qreg_free(&reg);
	return rc;
}
