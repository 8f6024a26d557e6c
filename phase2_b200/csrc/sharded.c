/*
 * sharded.c -- registers sharded by their high qubits, with qubit-swap
 * exchange, for C hosts (include/phase2_sharded.h).
 *
 * One struct qreg per rank this process holds (its 2^L local amplitudes);
 * a layout maps global qubits to physical positions and back, the same on
 * every rank.  A rotation whose flip reaches a high position first swaps
 * that position with a local one (Belady's choice over the rotations that
 * follow), then every run of rotations whose flips are local goes to the
 * engine's rotation queue (qreg_paulirot) with the sign of its high Z
 * bits folded into the angle.  This replaces the reference's per-flush
 * slab exchange (phase2/qreg.c:124-142).
 */
#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "sharded"
#include "log.h"

#include "phase2/circ.h"
#include "phase2/qreg.h"
#include "phase2_b200.h"
#include "phase2_sharded.h"
#include "prob.h"
#include "xoshiro256ss.h"

#include "p2_internal.h"

/* rotations searched for the next use of a local qubit */
#define SH_LOOKAHEAD 4096
/* rotations handed to qreg_paulirot per call */
#define SH_BATCH 1024
#define SH_CHUNK (UINT64_C(1) << 26)

struct phase2_sharded {
	uint32_t nqb, nloc, world, nranks;
	int prec;
	uint32_t *ranks;     /* ranks held here */
	struct qreg *slab;   /* one register per rank held */
	int *held;           /* world entries: index into slab, or -1 */
	uint8_t pos[64];     /* global qubit -> physical position */
	uint8_t at[64];      /* physical position -> global qubit */
	struct phase2_shard_io io;
	uint64_t chunk;
	size_t elem;
	void *sbuf, *rbuf;   /* exchange buffers, chunk * elem bytes */
	uint64_t swaps, exchanged;
	/* scratch of one batch: local codes and angles */
	struct paulis codes[SH_BATCH];
	double phis[SH_BATCH];
};

static uint64_t phys_mask(const struct phase2_sharded *s, uint64_t m)
{
	uint64_t out = 0;
	while (m) {
		const int q = __builtin_ctzll(m);
		out |= UINT64_C(1) << s->pos[q];
		m &= m - 1;
	}
	return out;
}

void phase2_sharded_free(struct phase2_sharded *s)
{
	if (!s)
		return;
	for (uint32_t k = 0; k < s->nranks && s->slab; k++)
		qreg_free(&s->slab[k]);
	p2d_buffer_free(s->sbuf);
	p2d_buffer_free(s->rbuf);
	free(s->slab);
	free(s->ranks);
	free(s->held);
	free(s);
}

struct phase2_sharded *phase2_sharded_new(uint32_t nqb, uint32_t world,
	const uint32_t *ranks, uint32_t nranks, int prec,
	const struct phase2_shard_io *io, uint64_t chunk)
{
	uint32_t g = 0;
	while (g < 32 && (UINT32_C(1) << g) < world)
		g++;
	if (world == 0 || (UINT32_C(1) << g) != world || nqb > 63 ||
		nqb <= g || !ranks || nranks == 0 || nranks > world ||
		(prec != PHASE2_PREC_FP32 && prec != PHASE2_PREC_FP64)) {
		log_error("sharded register: bad shape (nqb %u, world %u, %u "
			  "ranks held)", nqb, world, nranks);
		return NULL;
	}
	struct phase2_sharded *s = calloc(1, sizeof *s);
	if (!s)
		return NULL;
	s->nqb = nqb;
	s->nloc = nqb - g;
	s->world = world;
	s->prec = prec;
	s->elem = prec == PHASE2_PREC_FP64 ? 16 : 8;
	s->chunk = chunk ? chunk : SH_CHUNK;
	s->ranks = malloc(nranks * sizeof *s->ranks);
	s->slab = calloc(nranks, sizeof *s->slab);
	s->held = malloc(world * sizeof *s->held);
	if (!s->ranks || !s->slab || !s->held) {
		phase2_sharded_free(s);
		return NULL;
	}
	for (uint32_t r = 0; r < world; r++)
		s->held[r] = -1;
	for (uint32_t k = 0; k < nranks; k++) {
		if (ranks[k] >= world || s->held[ranks[k]] >= 0) {
			log_error("sharded register: rank %u held twice or "
				  "outside the world", ranks[k]);
			phase2_sharded_free(s);
			return NULL;
		}
		s->held[ranks[k]] = 0;
	}
	/* Ranks held in increasing order, whatever the caller's order: a swap
	 * of rank bit b then runs its exchanges in increasing order of the
	 * pair (r with bit b cleared) on every process, one total order, so a
	 * blocking pairwise transport cannot deadlock. */
	uint32_t nh = 0;
	for (uint32_t r = 0; r < world; r++)
		if (s->held[r] >= 0) {
			s->held[r] = (int)nh;
			s->ranks[nh++] = r;
		}
	for (uint32_t k = 0; k < nranks; k++) {
		if (qreg_init_prec(&s->slab[k], s->nloc, prec) != 0) {
			s->nranks = k;
			phase2_sharded_free(s);
			return NULL;
		}
		s->nranks = k + 1;
	}
	if (io)
		s->io = *io;
	if (nranks < world && (!io || !io->exchange || !io->sum)) {
		log_error("sharded register: %u of %u ranks held and no "
			  "transport", nranks, world);
		phase2_sharded_free(s);
		return NULL;
	}
	for (uint32_t q = 0; q < 64; q++)
		s->pos[q] = s->at[q] = (uint8_t)q;
	return s;
}

int phase2_sharded_synchronize(struct phase2_sharded *s)
{
	if (!s)
		return -1;
	int rc = 0;
	for (uint32_t k = 0; k < s->nranks; k++)
		if (qreg_synchronize(&s->slab[k]) != 0)
			rc = -1;
	return rc;
}

int phase2_sharded_layout(const struct phase2_sharded *s, uint32_t *pos)
{
	if (!s || !pos)
		return -1;
	for (uint32_t q = 0; q < s->nqb; q++)
		pos[q] = s->pos[q];
	return 0;
}

void phase2_sharded_counters(const struct phase2_sharded *s,
	uint64_t *swaps, uint64_t *exchanged)
{
	if (swaps)
		*swaps = s ? s->swaps : 0;
	if (exchanged)
		*exchanged = s ? s->exchanged : 0;
}

/* ---- the qubit swap ------------------------------------------------------ */

/*
 * Trade the qubits at high position h and local position l: rank r swaps
 * the half of its slab whose bit l differs from its rank bit b = h - L
 * (val = 1 - bit b of r) with the partner r ^ 2^b.  Held pairs trade in
 * place; others through the transport, chunk by chunk, in increasing rank
 * order (s->ranks is sorted).
 */
static int swap_positions(struct phase2_sharded *s, uint32_t h, uint32_t l)
{
	const uint32_t b = h - s->nloc, mask = UINT32_C(1) << b;
	const uint64_t nhalf = UINT64_C(1) << (s->nloc - 1);
	for (uint32_t k = 0; k < s->nranks; k++) {
		const uint32_t r = s->ranks[k], partner = r ^ mask;
		const uint32_t val = 1u - (r >> b & 1u);
		const int pk = s->held[partner];
		if (pk >= 0) {
			if (r < partner) {
				if (qreg_slab_swap(&s->slab[k], &s->slab[pk], l,
					    val, 1u - val) != 0)
					return -1;
				s->exchanged += 2 * nhalf;
			}
			continue;
		}
		const uint64_t cnt0 = nhalf < s->chunk ? nhalf : s->chunk;
		if (!s->sbuf) {
			s->sbuf = p2d_buffer_alloc(cnt0 * s->elem);
			s->rbuf = p2d_buffer_alloc(cnt0 * s->elem);
			if (!s->sbuf || !s->rbuf)
				return -1;
		}
		for (uint64_t first = 0; first < nhalf; first += cnt0) {
			const uint64_t cnt =
				nhalf - first < cnt0 ? nhalf - first : cnt0;
			if (qreg_slab_get(&s->slab[k], l, val, first, cnt,
				    s->sbuf) != 0 ||
				s->io.exchange(s->io.ctx, r, partner, s->sbuf,
					s->rbuf, cnt * s->elem) != 0 ||
				qreg_slab_put(&s->slab[k], l, val, first, cnt,
					s->rbuf) != 0) {
				log_error("sharded register: exchange of rank "
					  "%u with %u failed", r, partner);
				return -1;
			}
			s->exchanged += cnt;
		}
	}
	const uint8_t qh = s->at[h], ql = s->at[l];
	s->at[h] = ql;
	s->at[l] = qh;
	s->pos[qh] = (uint8_t)l;
	s->pos[ql] = (uint8_t)h;
	s->swaps++;
	return 0;
}

/*
 * Make the flip of rotation k local: every high position of its physical
 * flip trades places with a local position outside the flip, the one
 * whose global qubit the next SH_LOOKAHEAD rotations flip again farthest
 * ahead (never: farthest of all; ties to the higher position).
 */
static int make_local(struct phase2_sharded *s, const uint64_t *flip,
	size_t k, size_t n)
{
	const uint64_t lomask = (UINT64_C(1) << s->nloc) - 1;
	const uint64_t pf = phys_mask(s, flip[k]);
	uint64_t need = pf & ~lomask;
	uint64_t taken = pf & lomask;
	if ((uint32_t)__builtin_popcountll(pf) > s->nloc) {
		log_error("sharded register: a flip over %d qubits does not fit "
			  "the %u local qubits of a rank",
			  __builtin_popcountll(pf), s->nloc);
		return -1;
	}
	while (need) {
		const uint32_t h = (uint32_t)__builtin_ctzll(need);
		need &= need - 1;
		/* next use, in rotations ahead, of each free local position */
		size_t next[64];
		const uint64_t free_pos = lomask & ~taken;
		uint64_t open = free_pos;
		for (uint32_t p = 0; p < s->nloc; p++)
			next[p] = SH_LOOKAHEAD + 1;
		const size_t end = n - k - 1 < SH_LOOKAHEAD ? n - k - 1
							     : SH_LOOKAHEAD;
		for (size_t i = 0; i < end && open; i++) {
			uint64_t hit = phys_mask(s, flip[k + 1 + i]) & open;
			open &= ~hit;
			while (hit) {
				next[__builtin_ctzll(hit)] = i;
				hit &= hit - 1;
			}
		}
		uint32_t best = 64;
		for (uint32_t p = 0; p < s->nloc; p++)
			if ((free_pos >> p & 1) &&
				(best == 64 || next[p] >= next[best]))
				best = p;
		if (best == 64) {
			log_error("sharded register: no free local position");
			return -1;
		}
		if (swap_positions(s, h, best) != 0)
			return -1;
		taken |= UINT64_C(1) << best;
	}
	return 0;
}

/* Rotations [k0, k1) whose physical flips are local: each rank held
 * applies exp(i sigma phi P_lo), sigma = (-1)^popc(r & z_hi). */
static void apply_local(struct phase2_sharded *s, const uint64_t *flip,
	const uint64_t *phase, const double *phi, size_t k0, size_t k1)
{
	const uint64_t lomask = (UINT64_C(1) << s->nloc) - 1;
	const struct paulis id = paulis_new();
	for (uint32_t j = 0; j < s->nranks; j++) {
		const uint64_t r = s->ranks[j];
		for (size_t k = k0; k < k1; k += SH_BATCH) {
			const size_t m = k1 - k < SH_BATCH ? k1 - k : SH_BATCH;
			for (size_t i = 0; i < m; i++) {
				const uint64_t pf = phys_mask(s, flip[k + i]);
				const uint64_t pp = phys_mask(s, phase[k + i]);
				const int odd = __builtin_popcountll(
						(pp >> s->nloc) & r) & 1;
				s->codes[i].pak[0] = pf;
				s->codes[i].pak[1] = pp & lomask;
				s->phis[i] = odd ? -phi[k + i] : phi[k + i];
			}
			qreg_paulirot(&s->slab[j], id, s->codes, s->phis, m);
		}
	}
}

int phase2_sharded_paulirot(struct phase2_sharded *s, const uint64_t *flip,
	const uint64_t *phase, const double *phi, size_t n)
{
	if (!s || (n && (!flip || !phase || !phi)))
		return -1;
	const uint64_t lomask = (UINT64_C(1) << s->nloc) - 1;
	const uint64_t wide = s->nqb < 64 ? ~((UINT64_C(1) << s->nqb) - 1) : 0;
	for (size_t k = 0; k < n; k++)
		if ((flip[k] | phase[k]) & wide) {
			log_error("sharded register: Pauli string acts beyond "
				  "the register");
			return -1;
		}
	size_t k = 0;
	while (k < n) {
		size_t j = k;
		while (j < n && !(phys_mask(s, flip[j]) & ~lomask))
			j++;
		if (j > k)
			apply_local(s, flip, phase, phi, k, j);
		if (j < n && make_local(s, flip, j, n) != 0)
			return -1;
		k = j;
	}
	return 0;
}

/* ---- state preparation and overlaps -------------------------------------- */

int phase2_sharded_prepst(struct phase2_sharded *s, const uint64_t *idx,
	const _Complex double *cf, size_t ndet)
{
	if (!s || (ndet && (!idx || !cf)))
		return -1;
	const uint64_t lomask = (UINT64_C(1) << s->nloc) - 1;
	for (uint32_t j = 0; j < s->nranks; j++) {
		qreg_zero(&s->slab[j]);
		for (size_t d = 0; d < ndet; d++) {
			const uint64_t p = phys_mask(s, idx[d]);
			if ((p >> s->nloc) != s->ranks[j])
				continue;
			const uint64_t loc = p & lomask;
			if (qreg_setamps(&s->slab[j], &loc, &cf[d], 1) != 0)
				return -1;
		}
	}
	return 0;
}

int phase2_sharded_getamps(struct phase2_sharded *s, const uint64_t *idx,
	_Complex double *out, size_t n)
{
	if (!s || (n && (!idx || !out)))
		return -1;
	const uint64_t lomask = (UINT64_C(1) << s->nloc) - 1;
	/* one read per rank held: its indices gathered, then scattered back */
	uint64_t *loc = malloc((n ? n : 1) * sizeof *loc);
	size_t *at = malloc((n ? n : 1) * sizeof *at);
	_Complex double *val = malloc((n ? n : 1) * sizeof *val);
	int rc = loc && at && val ? 0 : -1;
	for (size_t i = 0; i < n; i++)
		out[i] = 0;
	for (uint32_t j = 0; j < s->nranks && rc == 0; j++) {
		size_t m = 0;
		for (size_t i = 0; i < n; i++) {
			const uint64_t p = phys_mask(s, idx[i]);
			if ((p >> s->nloc) != s->ranks[j])
				continue;
			loc[m] = p & lomask;
			at[m++] = i;
		}
		if (m && qreg_getamps(&s->slab[j], loc, val, m) != 0)
			rc = -1;
		for (size_t k = 0; k < m && rc == 0; k++)
			out[at[k]] = val[k];
	}
	free(loc);
	free(at);
	free(val);
	if (rc != 0)
		return -1;
	if (s->nranks < s->world &&
		s->io.sum(s->io.ctx, (double *)out, 2 * n) != 0) {
		log_error("sharded register: sum over ranks failed");
		return -1;
	}
	return 0;
}

int phase2_sharded_measure(struct phase2_sharded *s, const uint64_t *idx,
	const _Complex double *cf, size_t ndet, _Complex double *z)
{
	if (!z || (ndet && !cf))
		return -1;
	_Complex double *a = malloc((ndet ? ndet : 1) * sizeof *a);
	if (!a || phase2_sharded_getamps(s, idx, a, ndet) != 0) {
		free(a);
		return -1;
	}
	double pr = 0.0, pi = 0.0;
	for (size_t d = 0; d < ndet; d++) {
		const double ar = creal(a[d]), ai = cimag(a[d]);
		const double cr = creal(cf[d]), ci = -cimag(cf[d]);
		pr += ar * cr - ai * ci;
		pi += ar * ci + ai * cr;
	}
	free(a);
	*z = CMPLX(pr, pi);
	return 0;
}

int phase2_sharded_norm2(struct phase2_sharded *s, double *out)
{
	if (!s || !out)
		return -1;
	double *part = calloc(s->world, sizeof *part);
	if (!part)
		return -1;
	for (uint32_t j = 0; j < s->nranks; j++)
		if (qreg_norm2(&s->slab[j], &part[s->ranks[j]]) != 0) {
			free(part);
			return -1;
		}
	if (s->nranks < s->world && s->io.sum(s->io.ctx, part, s->world)) {
		free(part);
		return -1;
	}
	double tot = 0.0;
	for (uint32_t r = 0; r < s->world; r++)
		tot += part[r];
	free(part);
	*out = tot;
	return 0;
}

/* ---- drivers --------------------------------------------------------------- */

/* Terms of a Hamiltonian as flip / phase / coefficient arrays. */
struct sh_terms {
	uint64_t *flip, *phase;
	double *cf, *phi;
	size_t n;
};

static void terms_free(struct sh_terms *t)
{
	free(t->flip);
	free(t->phase);
	free(t->cf);
	free(t->phi);
	memset(t, 0, sizeof *t);
}

static int terms_of(struct sh_terms *t, const struct circ_hamil *hm,
	size_t extra)
{
	memset(t, 0, sizeof *t);
	const size_t n = hm->len + extra;
	t->flip = malloc((n ? n : 1) * sizeof *t->flip);
	t->phase = malloc((n ? n : 1) * sizeof *t->phase);
	t->cf = malloc((n ? n : 1) * sizeof *t->cf);
	t->phi = malloc((n ? n : 1) * sizeof *t->phi);
	if (!t->flip || !t->phase || !t->cf || !t->phi) {
		terms_free(t);
		return -1;
	}
	for (size_t k = 0; k < hm->len; k++) {
		t->flip[k] = hm->terms[k].op.pak[0];
		t->phase[k] = hm->terms[k].op.pak[1];
		t->cf[k] = hm->terms[k].cf;
	}
	t->n = hm->len;
	return 0;
}

static void reverse_u64(uint64_t *a, size_t n)
{
	for (size_t i = 0, j = n ? n - 1 : 0; i < j; i++, j--) {
		const uint64_t t = a[i];
		a[i] = a[j];
		a[j] = t;
	}
}

static void reverse_f64(double *a, size_t n)
{
	for (size_t i = 0, j = n ? n - 1 : 0; i < j; i++, j--) {
		const double t = a[i];
		a[i] = a[j];
		a[j] = t;
	}
}

static uint64_t *det_idx(const struct circ_muldet *md)
{
	uint64_t *idx = malloc((md->len ? md->len : 1) * sizeof *idx);
	if (idx)
		for (size_t d = 0; d < md->len; d++)
			idx[d] = md->dets[d].idx;
	return idx;
}

static _Complex double *det_cf(const struct circ_muldet *md)
{
	_Complex double *cf = malloc((md->len ? md->len : 1) * sizeof *cf);
	if (cf)
		for (size_t d = 0; d < md->len; d++)
			cf[d] = md->dets[d].cf;
	return cf;
}

int phase2_sharded_trott(struct phase2_sharded *s,
	const struct circ_hamil *hm, const struct circ_muldet *md, size_t steps,
	double delta, int order2, _Complex double *out)
{
	if (!s || !hm || !md || (steps && !out))
		return -1;
	struct circ_hamil sorted;
	if (circ_hamil_init(&sorted, hm->qb, hm->len) != 0)
		return -1;
	if (hm->len)
		memcpy(sorted.terms, hm->terms, hm->len * sizeof *hm->terms);
	circ_hamil_sort_lex(&sorted);
	struct sh_terms f, r;
	uint64_t *idx = det_idx(md);
	_Complex double *cf = det_cf(md);
	int rc = -1;
	if (terms_of(&f, &sorted, 0) != 0) {
		circ_hamil_free(&sorted);
		free(idx);
		free(cf);
		return -1;
	}
	if (terms_of(&r, &sorted, 0) != 0) {
		terms_free(&f);
		circ_hamil_free(&sorted);
		free(idx);
		free(cf);
		return -1;
	}
	circ_hamil_free(&sorted);
	if (!idx || !cf)
		goto done;
	/* angles: c delta (first order), c delta/2 forward and reversed */
	const double half = delta / 2.0;
	for (size_t k = 0; k < f.n; k++) {
		f.phi[k] = order2 ? f.cf[k] * half : f.cf[k] * delta;
		r.phi[k] = f.phi[k];
	}
	reverse_u64(r.flip, r.n);
	reverse_u64(r.phase, r.n);
	reverse_f64(r.phi, r.n);
	if (phase2_sharded_prepst(s, idx, cf, md->len) != 0)
		goto done;
	for (size_t st = 0; st < steps; st++) {
		if (phase2_sharded_paulirot(s, f.flip, f.phase, f.phi, f.n))
			goto done;
		if (order2 && phase2_sharded_paulirot(s, r.flip, r.phase,
				      r.phi, r.n))
			goto done;
		if (phase2_sharded_measure(s, idx, cf, md->len, &out[st]))
			goto done;
	}
	rc = 0;
done:
	terms_free(&f);
	terms_free(&r);
	free(idx);
	free(cf);
	return rc;
}

/* -1, 0 or +1 with a dead zone of DBL_EPSILON (the drivers' sign of a
 * drawn coefficient). */
static double sign_dz(double a)
{
	const double f = fabs(a);
	return f < DBL_EPSILON ? 0.0 : (a < f ? -1.0 : 1.0);
}

int phase2_sharded_qdrift(struct phase2_sharded *s,
	const struct circ_hamil *hm, const struct circ_muldet *md,
	size_t samples, size_t depth, double step_size, uint64_t seed,
	_Complex double *out)
{
	if (!s || !hm || !md || hm->len == 0 || seed == 0 ||
		(samples && !out)) {
		log_error("sharded qdrift: bad arguments (no terms, or seed 0)");
		return -1;
	}
	struct prob_cdf cdf;
	if (prob_cdf_init(&cdf, hm->len) != 0)
		return -1;
	prob_cdf_from_array_strided(&cdf, &hm->terms[0].cf,
		sizeof hm->terms[0], NULL);
	struct xoshiro256ss rng;
	xoshiro256ss_init(&rng, seed);
	const double omega = asin(step_size);
	uint64_t *fl = malloc((depth ? depth : 1) * sizeof *fl);
	uint64_t *ph = malloc((depth ? depth : 1) * sizeof *ph);
	double *phi = malloc((depth ? depth : 1) * sizeof *phi);
	uint64_t *idx = det_idx(md);
	_Complex double *cf = det_cf(md);
	int rc = -1;
	if (!fl || !ph || !phi || !idx || !cf)
		goto done;
	for (size_t smp = 0; smp < samples; smp++) {
		if (phase2_sharded_prepst(s, idx, cf, md->len) != 0)
			goto done;
		for (size_t i = 0; i < depth; i++) {
			const double x = xoshiro256ss_dbl01(&rng);
			const size_t k = prob_cdf_inverse(&cdf, x);
			fl[i] = hm->terms[k].op.pak[0];
			ph[i] = hm->terms[k].op.pak[1];
			phi[i] = omega * sign_dz(hm->terms[k].cf);
		}
		if (phase2_sharded_paulirot(s, fl, ph, phi, depth) != 0 ||
			phase2_sharded_measure(s, idx, cf, md->len, &out[smp]))
			goto done;
	}
	rc = 0;
done:
	prob_cdf_free(&cdf);
	free(fl);
	free(ph);
	free(phi);
	free(idx);
	free(cf);
	return rc;
}

/* One cmpsit sample: the head terms at c angle_det, then `depth` draws
 * from the tail's CDF at sign_dz(c) angle_rand, all times 0.5; reversed
 * for a backward half. */
static void cmpsit_sample(const struct cmpsit_ranct *rc,
	const struct cmpsit_data *dt, struct xoshiro256ss *rng,
	struct sh_terms *t, int reverse)
{
	const size_t nd = rc->hm_det.len;
	for (size_t k = 0; k < nd; k++) {
		t->flip[k] = rc->hm_det.terms[k].op.pak[0];
		t->phase[k] = rc->hm_det.terms[k].op.pak[1];
		t->phi[k] = 0.5 * (rc->hm_det.terms[k].cf * dt->angle_det);
	}
	for (size_t i = 0; i < dt->depth; i++) {
		const double x = xoshiro256ss_dbl01(rng);
		const size_t k = prob_cdf_inverse(&rc->cdf, x);
		t->flip[nd + i] = rc->hm_ran.terms[k].op.pak[0];
		t->phase[nd + i] = rc->hm_ran.terms[k].op.pak[1];
		t->phi[nd + i] = 0.5 * (sign_dz(rc->hm_ran.terms[k].cf) *
			dt->angle_rand);
	}
	t->n = nd + dt->depth;
	if (reverse) {
		reverse_u64(t->flip, t->n);
		reverse_u64(t->phase, t->n);
		reverse_f64(t->phi, t->n);
	}
}

int phase2_sharded_cmpsit(struct phase2_sharded *s,
	const struct circ_hamil *hm, const struct circ_muldet *md,
	const struct cmpsit_data *dt, _Complex double *out)
{
	if (!s || !hm || !md || !dt || dt->seed == 0 ||
		(dt->samples && !out)) {
		log_error("sharded cmpsit: bad arguments (seed 0?)");
		return -1;
	}
	struct cmpsit_ranct rc;
	memset(&rc, 0, sizeof rc);
	if (cmpsit_ranct_init(&rc, hm, dt) != 0) {
		log_error("sharded cmpsit: term split failed");
		return -1;
	}
	struct circ_hamil none;
	memset(&none, 0, sizeof none);
	struct sh_terms t;
	uint64_t *idx = det_idx(md);
	_Complex double *cf = det_cf(md);
	int ret = -1;
	if (terms_of(&t, &none, rc.hm_det.len + dt->depth) != 0) {
		cmpsit_ranct_free(&rc);
		free(idx);
		free(cf);
		return -1;
	}
	struct xoshiro256ss rng;
	xoshiro256ss_init(&rng, dt->seed);
	if (!idx || !cf)
		goto done;
	for (size_t smp = 0; smp < dt->samples; smp++) {
		if (phase2_sharded_prepst(s, idx, cf, md->len) != 0)
			goto done;
		for (size_t st = 0; st < dt->steps; st++) {
			for (int half = 0; half < 2; half++) {
				cmpsit_sample(&rc, dt, &rng, &t, half);
				if (phase2_sharded_paulirot(s, t.flip, t.phase,
					    t.phi, t.n) != 0)
					goto done;
			}
		}
		if (phase2_sharded_measure(s, idx, cf, md->len, &out[smp]))
			goto done;
	}
	ret = 0;
done:
	terms_free(&t);
	cmpsit_ranct_free(&rc);
	free(idx);
	free(cf);
	return ret;
}
