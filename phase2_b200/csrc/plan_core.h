/*
 * plan_core.h -- the pass planner (see plan.c for what it computes),
 * written once for the host (plan.c) and the device (engine.cu, the
 * device-side qDRIFT planner): both compile this code, so both produce the
 * same passes and records, bit for bit, for the same rotations and cos/sin
 * values.  The floating-point steps are single IEEE operations
 * (division, sum, product, conversion), rounded the same on both sides.
 */
#ifndef P2_PLAN_CORE_H
#define P2_PLAN_CORE_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "phase2_b200.h"

#include "p2_internal.h"

#if defined(__CUDACC__)
#define P2_HD static __host__ __device__ __forceinline__
#if defined(__CUDA_ARCH__)
#define P2_POPC64(x) __popcll(x)
#define P2_POPC32(x) __popc(x)
#define P2_CLZ64(x) __clzll(x)
#else
#define P2_POPC64(x) __builtin_popcountll(x)
#define P2_POPC32(x) __builtin_popcount(x)
#define P2_CLZ64(x) __builtin_clzll(x)
#endif
#else
#define P2_HD static inline
#define P2_POPC64(x) __builtin_popcountll(x)
#define P2_POPC32(x) __builtin_popcount(x)
#define P2_CLZ64(x) __builtin_clzll(x)
#endif

struct echelon {
	int rows;
	uint64_t v[PHASE2_MAX_SPAN];     /* reduced rows, pivots descending */
	uint32_t combo[PHASE2_MAX_SPAN]; /* row = xor of basis[k], k in combo */
	int piv[PHASE2_MAX_SPAN];
};

P2_HD int top_bit(uint64_t v)
{
	return 63 - P2_CLZ64(v);
}

/* Reduce v by the rows; returns the remainder, *combo = rows used. */
P2_HD uint64_t ech_reduce(const struct echelon *e, uint64_t v,
	uint32_t *combo)
{
	uint32_t c = 0;
	for (int r = 0; r < e->rows; r++)
		if (v >> e->piv[r] & 1) {
			v ^= e->v[r];
			c ^= e->combo[r];
		}
	*combo = c;
	return v;
}

/* Insert a non-zero remainder v (combination `combo`) keeping pivots in
 * descending order. */
P2_HD void ech_insert(struct echelon *e, uint64_t v, uint32_t combo)
{
	const int p = top_bit(v);
	int at = e->rows;
	while (at > 0 && e->piv[at - 1] < p) {
		e->v[at] = e->v[at - 1];
		e->combo[at] = e->combo[at - 1];
		e->piv[at] = e->piv[at - 1];
		at--;
	}
	e->v[at] = v;
	e->combo[at] = combo;
	e->piv[at] = p;
	e->rows++;
}

struct pass_builder {
	struct echelon ech;
	uint64_t basis[PHASE2_MAX_SPAN];
	int m;
	/* rotations of the open pass (indices into the caller's arrays) */
	size_t first_rec;
	uint32_t nrot;
};

P2_HD void builder_reset(struct pass_builder *b, size_t first_rec)
{
	memset(b, 0, sizeof *b);
	b->first_rec = first_rec;
}

/* Add basis vector f (not in the span); returns its slot bit. */
P2_HD uint32_t builder_add(struct pass_builder *b, uint64_t f)
{
	uint32_t combo;
	const uint64_t v = ech_reduce(&b->ech, f, &combo);
	const int k = b->m++;
	b->basis[k] = f;
	ech_insert(&b->ech, v, combo ^ (UINT32_C(1) << k));
	return UINT32_C(1) << k;
}

P2_HD int parity64(uint64_t v)
{
	return P2_POPC64(v) & 1;
}

/*
 * Coefficients of a lifted rotation applied with FP32 arithmetic (c >= 0):
 * s is rounded to FP32 and t = (1 - c) / fl32(s) is kept in FP64, so the
 * product t * fl32(s), which fixes the rotation angle (the three shears
 * have trace 2 (1 - t s)), equals 1 - cos(phi) to FP64 accuracy; the
 * kernel's rounding of t to FP32 is then the only error in the angle
 * (relative, at most 2^-25).  1 - c is formed as s^2 / (1 + c).
 */
P2_HD void lift_f32(double c, double s, double *t_out, double *s_out)
{
	const float s32 = (float)s;
	*s_out = s32;
	*t_out = s32 == 0.0f ? 0.0 : s * s / (1.0 + c) / (double)s32;
}

/* Header of the open pass: pad the basis with unit vectors (more
 * amplitudes per thread, contiguous along low qubits), pivots ascending,
 * basis, sizes; scale 1 (the records' signs set it, p2_rec_fill); head:
 * the pass starts a sweep. */
P2_HD void builder_header(struct pass_builder *b, uint32_t nqb, int pad_to,
	int form, int head, struct phase2_pass *pass)
{
	for (uint32_t q = 0; b->m < pad_to && q < nqb; q++) {
		uint32_t combo;
		if (ech_reduce(&b->ech, UINT64_C(1) << q, &combo) != 0)
			(void)builder_add(b, UINT64_C(1) << q);
	}
	memset(pass, 0, sizeof *pass);
	pass->span = (uint32_t)b->m;
	pass->nrot = b->nrot;
	pass->rot_off = (uint32_t)b->first_rec;
	/* pivots ascending (the echelon keeps them descending) */
	for (int k = 0; k < b->m; k++) {
		pass->piv[k] = (uint8_t)b->ech.piv[b->m - 1 - k];
		pass->basis[k] = b->basis[k];
	}
	pass->scale = 1.0;
	pass->form = (uint8_t)form;
	pass->sweep = (uint8_t)(head != 0);
}

/* Echelon of a sweep's flip masks modulo the low qubits (rows with
 * distinct top bits, kept in descending order). */
#define P2_SWEEP_ROWS 16
struct sweep_ech {
	int rows;
	uint64_t v[P2_SWEEP_ROWS];
	int piv[P2_SWEEP_ROWS];
};

P2_HD uint64_t swe_reduce(const struct sweep_ech *e, uint64_t v)
{
	for (int r = 0; r < e->rows; r++)
		if (v >> e->piv[r] & 1)
			v ^= e->v[r];
	return v;
}

P2_HD void swe_insert(struct sweep_ech *e, uint64_t v)
{
	const int p = top_bit(v);
	int at = e->rows;
	while (at > 0 && e->piv[at - 1] < p) {
		e->v[at] = e->v[at - 1];
		e->piv[at] = e->piv[at - 1];
		at--;
	}
	e->v[at] = v;
	e->piv[at] = p;
	e->rows++;
}

/*
 * The record of one rotation (flip, phase, cos c, sin s, slot combination
 * U) of a pass: slot masks, W, odd and, in the lifted forms, the lifted
 * coefficients.  Returns 1 when the record's -1 goes to the pass scale (a
 * lifted rotation with c < 0), else 0.
 */
P2_HD int p2_rec_fill(const struct phase2_pass *pass, uint64_t flip,
	uint64_t phase, double c, double s, uint32_t U,
	struct phase2_rot_rec *rec)
{
	const int m = (int)pass->span;
	const uint32_t nslot = UINT32_C(1) << m;
	uint32_t W = 0;
	for (int k = 0; k < m; k++)
		W |= (uint32_t)parity64(pass->basis[k] & phase) << k;
	const int kbase = (1 - P2_POPC64(flip & phase)) & 3;
	uint32_t smask = 0;
	for (uint32_t u = 0; u < nslot; u++)
		smask |= (uint32_t)((P2_POPC32(u & W) & 1) ^ (kbase >> 1)) << u;
	rec->z = phase;
	rec->smask = smask;
	rec->U = (uint8_t)U;
	rec->W = (uint8_t)W;
	rec->odd = (uint8_t)(kbase & 1);
	rec->form = 0;
	rec->c = c;
	rec->s = s;
	const int form = pass->form;
	int neg = 0;
	if (form == PHASE2_FORM_LIFTED || form == PHASE2_FORM_LIFTED_F32 ||
		form == PHASE2_FORM_LIFTED_MIXED) {
		/* Three shears per pair (no temporaries, no pass-wide factor):
		 * t = tan(phi/2) = s / (1 + c), computed with c >= 0 so it
		 * stays in [-1, 1]; for c < 0 the rotation is
		 * exp(i(phi -+ pi)P) times -1, and the -1 goes to the pass. */
		if (c < 0) {
			c = -c;
			s = -s;
			neg = 1;
		}
		rec->form = 1;
		if (form == PHASE2_FORM_LIFTED_F32 ||
			form == PHASE2_FORM_LIFTED_MIXED) {
			lift_f32(c, s, &rec->c, &rec->s);
		} else {
			rec->c = s / (1.0 + c);
			rec->s = s;
		}
	}
	return neg;
}

/*
 * Pass boundaries (the sequential half of the planner): greedy passes in
 * input order, a pass closing when the next flip mask would widen its
 * span beyond max_span or its rotations reach max_rots.  With sweep_k > 0,
 * passes also group into sweeps: a sweep closes (and with it the pass)
 * when the next flip mask, taken modulo the low sweep_low qubits, would
 * widen the sweep's span beyond sweep_k; a pass that starts a sweep has
 * its sweep flag set.  flip i is flips[i * fstride]; writes the pass
 * headers, each rotation's slot combination U to U_out[i * ustride] and,
 * when pidx is not NULL, its pass index to pidx[i].  Returns the number of
 * passes or -1.
 */
P2_HD long p2_plan_scan(uint32_t nqb, const uint64_t *flips, size_t fstride,
	size_t n, int max_span, int max_rots, int pad_span, int form,
	int sweep_k, int sweep_low, struct phase2_pass *passes,
	uint8_t *U_out, size_t ustride, uint16_t *pidx)
{
	if (nqb == 0 || nqb > QREG_MAX_WIDTH)
		return -1;
	if (max_span < 1)
		max_span = 1;
	if (max_span > PHASE2_MAX_SPAN)
		max_span = PHASE2_MAX_SPAN;
	if ((uint32_t)max_span > nqb)
		max_span = (int)nqb;
	if (pad_span > max_span)
		pad_span = max_span;
	if (pad_span < 0)
		pad_span = 0;
	const uint32_t cap = (max_rots > 0 && max_rots < P2_MAX_ROTS_PER_PASS)
		? (uint32_t)max_rots
		: P2_MAX_ROTS_PER_PASS;

	if (sweep_k < 0 || sweep_k > P2_SWEEP_ROWS || sweep_low < 0 ||
		sweep_low > 31)
		return -1;
	const uint64_t lowm = (UINT64_C(1) << sweep_low) - 1;
	long npass = 0;
	struct pass_builder b;
	builder_reset(&b, 0);
	struct sweep_ech sw;
	sw.rows = 0;
	int head = 1; /* the open pass starts a sweep */
	for (size_t i = 0; i < n; i++) {
		const uint64_t f = flips[i * fstride];
		uint32_t U = 0;
		int fits = b.nrot < cap;
		if (fits && f != 0) {
			uint32_t combo;
			const uint64_t v = ech_reduce(&b.ech, f, &combo);
			if (v == 0)
				U = combo;
			else if (b.m < max_span)
				U = 0xffffffffu; /* new basis vector */
			else
				fits = 0;
		}
		uint64_t vs = 0;
		int new_sweep = 0;
		if (sweep_k > 0 && (f & ~lowm) != 0) {
			vs = swe_reduce(&sw, f & ~lowm);
			new_sweep = vs != 0 && sw.rows >= sweep_k;
		}
		if (!fits || new_sweep) {
			builder_header(&b, nqb, pad_span, form, head,
				&passes[npass]);
			npass++;
			builder_reset(&b, i);
			head = new_sweep;
			if (new_sweep) {
				sw.rows = 0;
				vs = f & ~lowm;
			}
			U = f != 0 ? 0xffffffffu : 0;
		}
		if (U == 0xffffffffu)
			U = builder_add(&b, f);
		if (vs != 0)
			swe_insert(&sw, vs);
		U_out[i * ustride] = (uint8_t)U;
		if (pidx)
			pidx[i] = (uint16_t)npass;
		b.nrot++;
	}
	if (b.nrot > 0) {
		builder_header(&b, nqb, pad_span, form, head, &passes[npass]);
		npass++;
	}
	return npass;
}

/* Records are emitted in input order: recs[i] describes rots[i].  cs
 * holds cos(phi), sin(phi) per rotation, or is NULL (computed here). */
P2_HD long p2_plan_core(uint32_t nqb, const struct phase2_rot_in *rots,
	const double *cs, size_t n, int max_span, int max_rots, int pad_span,
	int form, int sweep_k, int sweep_low, struct phase2_pass *passes,
	struct phase2_rot_rec *recs)
{
	const long np = p2_plan_scan(nqb, &rots[0].flip,
		sizeof *rots / sizeof(uint64_t), n, max_span, max_rots,
		pad_span, form, sweep_k, sweep_low, passes, &recs[0].U,
		sizeof *recs, NULL);
	for (long p = 0; p < np; p++) {
		struct phase2_pass *ps = &passes[p];
		int neg = 0;
		for (uint32_t r = 0; r < ps->nrot; r++) {
			const size_t i = ps->rot_off + (size_t)r;
			const double c = cs ? cs[2 * i] : cos(rots[i].phi);
			const double s = cs ? cs[2 * i + 1] : sin(rots[i].phi);
			neg ^= p2_rec_fill(ps, rots[i].flip, rots[i].phase, c, s,
				recs[i].U, &recs[i]);
		}
		ps->scale = neg ? -1.0 : 1.0;
	}
	return np;
}

#endif /* P2_PLAN_CORE_H */
