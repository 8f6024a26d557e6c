/*
 * oracle.c -- CPU restatement of the phase2 hot path (TEST INFRASTRUCTURE
 * ONLY; see oracle.h).  Plain, single-threaded C on a dense FP64 state.
 */
#define _POSIX_C_SOURCE 200809L

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* ---- xoshiro256** (lib/xoshiro256ss.c:34-85) ---------------------------- */

static uint64_t splitmix_next(uint64_t *x)
{
	uint64_t z = (*x += UINT64_C(0x9e3779b97f4a7c15));
	z = (z ^ (z >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
	z = (z ^ (z >> 27)) * UINT64_C(0x94d049bb133111eb);
	return z ^ (z >> 31);
}

static inline uint64_t rotl64(uint64_t x, int k)
{
	return (x << k) | (x >> (64 - k));
}

uint64_t orc_rng_next(uint64_t s[4])
{
	const uint64_t out = rotl64(s[1] * 5, 7) * 9;
	const uint64_t t = s[1] << 17;
	s[2] ^= s[0];
	s[3] ^= s[1];
	s[1] ^= s[2];
	s[0] ^= s[3];
	s[2] ^= t;
	s[3] = rotl64(s[3], 45);
	return out;
}

void orc_rng_init(uint64_t s[4], uint64_t seed)
{
	uint64_t x = seed;
	for (int k = 0; k < 4; k++)
		s[k] = splitmix_next(&x);
	for (int k = 0; k < 128; k++)
		(void)orc_rng_next(s);
}

double orc_rng_dbl01(uint64_t s[4])
{
	/* include/xoshiro256ss.h:58-59: top 53 bits scaled by 2^-53. */
	return (double)(orc_rng_next(s) >> 11) * 0x1.0p-53;
}

/* ---- Pauli algebra (include/phase2/paulis.h:137-144, paulis.c) ---------- */

uint64_t orc_effect(uint64_t flip, uint64_t phase, uint64_t i, int *r4)
{
	const int ny = __builtin_popcountll(flip & phase);
	const int nm = __builtin_popcountll(i & phase);
	*r4 = (ny + 2 * nm) & 3;
	return i ^ flip;
}

/* Per-qubit code in enum pauli_op order: I=0, X=1, Y=2, Z=3. */
static int op_code(uint64_t flip, uint64_t phase, int q)
{
	const int f = (int)(flip >> q & 1), p = (int)(phase >> q & 1);
	if (!f && !p)
		return 0;
	if (f && !p)
		return 1;
	if (f && p)
		return 2;
	return 3;
}

int orc_pauli_cmp(uint64_t f1, uint64_t p1, uint64_t f2, uint64_t p2)
{
	/* The first qubit (from 63 down) where the operators differ decides. */
	const uint64_t diff = (f1 ^ f2) | (p1 ^ p2);
	if (!diff)
		return 0;
	const int q = 63 - __builtin_clzll(diff);
	const int a = op_code(f1, p1, q), b = op_code(f2, p2, q);
	return a < b ? -1 : 1;
}

static int term_cmp_lex(const void *a, const void *b)
{
	const struct orc_term *x = a, *y = b;
	return orc_pauli_cmp(x->flip, x->phase, y->flip, y->phase);
}

void orc_sort_lex(struct orc_term *t, size_t n)
{
	qsort(t, n, sizeof *t, term_cmp_lex);
}

/* ---- sampling (lib/prob.c:39-78, circ/internal.h:26-32) ----------------- */

int orc_cdf_build(const double *w, size_t stride_bytes, size_t n, double *cdf,
	double *lambda)
{
	double sum = 0.0;
	for (size_t i = 0; i < n; i++) {
		const double v = fabs(*(const double *)((const char *)w +
			i * stride_bytes));
		cdf[i] = v;
		sum += v;
	}
	if (sum < DBL_EPSILON)
		return -1;
	double run = 0.0;
	for (size_t i = 0; i < n; i++) {
		run += cdf[i] / sum;
		cdf[i] = run;
	}
	if (lambda)
		*lambda = sum;
	return 0;
}

size_t orc_cdf_inverse(const double *cdf, size_t n, double y)
{
	/* Smallest i with cdf[i] > y; n-1 if there is none. */
	size_t lo = 0, hi = n;
	while (lo < hi) {
		const size_t mid = lo + (hi - lo) / 2;
		if (cdf[mid] <= y)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo < n ? lo : n - 1;
}

double orc_signof(double a)
{
	const double f = fabs(a);
	if (f < DBL_EPSILON)
		return 0.0;
	return a < f ? -1.0 : 1.0;
}

/* ---- the rotation (phase2/qreg_qreg.c:149-160, 181-198) ----------------- */

/* (s * i^k) * (pr + i pi), each component a single rounded product. */
static inline void mul_ipow(double s, int k, double pr, double pi,
	double *or_, double *oi)
{
	switch (k & 3) {
	case 0:
		*or_ = s * pr;
		*oi = s * pi;
		break;
	case 1:
		*or_ = -(s * pi);
		*oi = s * pr;
		break;
	case 2:
		*or_ = -(s * pr);
		*oi = -(s * pi);
		break;
	default:
		*or_ = s * pi;
		*oi = -(s * pr);
		break;
	}
}

static void rotate_cs(double *amp, uint64_t n, uint64_t flip, uint64_t phase,
	double c, double s)
{
	for (uint64_t i = 0; i < n; i++) {
		int r4;
		const uint64_t j = orc_effect(flip, phase, i, &r4);
		if (j < i)
			continue;
		const double xr = amp[2 * i], xi = amp[2 * i + 1];
		const double yr = amp[2 * j], yi = amp[2 * j + 1];
		double tr, ti, ur, ui;
		/* a_i <- c a_i + i conj(s z) a_j ; a_j <- c a_j + i (s z) a_i,
		 * with z = i^r4, i.e. multipliers s i^(1-r4) and s i^(1+r4). */
		mul_ipow(s, 1 - r4, yr, yi, &tr, &ti);
		mul_ipow(s, 1 + r4, xr, xi, &ur, &ui);
		const double ar = c * xr, ai = c * xi;
		const double br = c * yr, bi = c * yi;
		amp[2 * i] = ar + tr;
		amp[2 * i + 1] = ai + ti;
		if (j != i) {
			amp[2 * j] = br + ur;
			amp[2 * j + 1] = bi + ui;
		}
	}
}

void orc_rotate(double *amp, uint32_t nqb, uint64_t flip, uint64_t phase,
	double phi)
{
	rotate_cs(amp, UINT64_C(1) << nqb, flip, phase, cos(phi), sin(phi));
}

void orc_rotate_many(double *amp, uint32_t nqb, const uint64_t *flip,
	const uint64_t *phase, const double *phi, size_t n)
{
	for (size_t k = 0; k < n; k++)
		orc_rotate(amp, nqb, flip[k], phase[k], phi[k]);
}

/* ---- multidet state prep and overlap (phase2/circ.c:215-224, 338-350) --- */

void orc_prepst(double *amp, uint32_t nqb, size_t ndets,
	const uint64_t *det_idx, const double *det_cf)
{
	memset(amp, 0, sizeof(double) * 2 * (UINT64_C(1) << nqb));
	for (size_t d = 0; d < ndets; d++) {
		amp[2 * det_idx[d]] = det_cf[2 * d];
		amp[2 * det_idx[d] + 1] = det_cf[2 * d + 1];
	}
}

void orc_measure(const double *amp, size_t ndets, const uint64_t *det_idx,
	const double *det_cf, double out[2])
{
	double pr = 0.0, pi = 0.0;
	for (size_t d = 0; d < ndets; d++) {
		const double ar = amp[2 * det_idx[d]];
		const double ai = amp[2 * det_idx[d] + 1];
		const double cr = det_cf[2 * d], ci = -det_cf[2 * d + 1];
		/* a * conj(cf) as the C complex product (ac - bd, ad + bc). */
		pr += ar * cr - ai * ci;
		pi += ar * ci + ai * cr;
	}
	out[0] = pr;
	out[1] = pi;
}

/* ---- drivers (circ/trott.c, trott2.c, qdrift.c, cmpsit.c) --------------- */

static double *state_alloc(uint32_t nqb)
{
	if (nqb == 0 || nqb > 40)
		return NULL;
	return malloc(sizeof(double) * 2 * (UINT64_C(1) << nqb));
}

/* One sweep of circ_step_generic (phase2/circ.c:256-280): phi = omega*cf,
 * forward or reverse term order.  On one rank the batch cache only groups
 * consecutive terms, so the rotations apply one by one in sweep order. */
static void sweep(double *amp, uint32_t nqb, const struct orc_term *t,
	size_t n, double omega, int reverse)
{
	for (size_t k = 0; k < n; k++) {
		const struct orc_term *x = &t[reverse ? n - 1 - k : k];
		orc_rotate(amp, nqb, x->flip, x->phase, omega * x->cf);
	}
}

static struct orc_term *terms_copy(const struct orc_term *t, size_t n)
{
	struct orc_term *c = malloc(sizeof *c * (n ? n : 1));
	if (c && n)
		memcpy(c, t, sizeof *c * n);
	return c;
}

static int trott_any(int order2, uint32_t nqb, const struct orc_term *terms,
	size_t nterms, size_t ndets, const uint64_t *det_idx,
	const double *det_cf, size_t steps, double delta, int sort_lex,
	double *out_z)
{
	double *amp = state_alloc(nqb);
	struct orc_term *t = terms_copy(terms, nterms);
	if (!amp || !t) {
		free(amp);
		free(t);
		return -1;
	}
	if (sort_lex)
		orc_sort_lex(t, nterms);
	orc_prepst(amp, nqb, ndets, det_idx, det_cf);
	const double half = delta / 2.0;
	for (size_t s = 0; s < steps; s++) {
		if (order2) {
			sweep(amp, nqb, t, nterms, half, 0);
			sweep(amp, nqb, t, nterms, half, 1);
		} else {
			sweep(amp, nqb, t, nterms, delta, 0);
		}
		orc_measure(amp, ndets, det_idx, det_cf, out_z + 2 * s);
	}
	free(t);
	free(amp);
	return 0;
}

int orc_trott(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t steps, double delta, int sort_lex, double *out_z)
{
	return trott_any(0, nqb, terms, nterms, ndets, det_idx, det_cf, steps,
		delta, sort_lex, out_z);
}

int orc_trott2(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t steps, double delta, int sort_lex, double *out_z)
{
	return trott_any(1, nqb, terms, nterms, ndets, det_idx, det_cf, steps,
		delta, sort_lex, out_z);
}

/* Seed handling of qdrift_init (circ/qdrift.c:30,72-75): a zero seed falls
 * back to the driver's default.  The reference keeps the last non-zero seed
 * in a file-static variable; the oracle is stateless and always uses the
 * initial default for a zero seed. */
#define ORC_QDRIFT_SEED UINT64_C(0xeccd9dcc749fcdca)
#define ORC_CMPSIT_SEED UINT64_C(0xafb424901446f21f)

int orc_qdrift_draws(const struct orc_term *terms, size_t nterms,
	size_t samples, size_t depth, uint64_t seed, struct orc_term *out)
{
	if (nterms == 0)
		return -1;
	double *cdf = malloc(sizeof *cdf * nterms);
	if (!cdf)
		return -1;
	orc_cdf_build(&terms[0].cf, sizeof terms[0], nterms, cdf, NULL);
	uint64_t rng[4];
	orc_rng_init(rng, seed ? seed : ORC_QDRIFT_SEED);
	for (size_t s = 0; s < samples; s++)
		for (size_t k = 0; k < depth; k++) {
			const double x = orc_rng_dbl01(rng);
			const size_t idx = orc_cdf_inverse(cdf, nterms, x);
			struct orc_term *o = &out[s * depth + k];
			o->cf = orc_signof(terms[idx].cf);
			o->flip = terms[idx].flip;
			o->phase = terms[idx].phase;
		}
	free(cdf);
	return 0;
}

int orc_qdrift(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t samples, size_t depth, double step_size, uint64_t seed,
	double *out_z)
{
	double *amp = state_alloc(nqb);
	struct orc_term *draws = malloc(sizeof *draws * (depth ? depth : 1));
	double *cdf = malloc(sizeof *cdf * (nterms ? nterms : 1));
	int rc = -1;
	if (!amp || !draws || !cdf || nterms == 0)
		goto out;
	orc_cdf_build(&terms[0].cf, sizeof terms[0], nterms, cdf, NULL);
	uint64_t rng[4];
	orc_rng_init(rng, seed ? seed : ORC_QDRIFT_SEED);
	const double omega = asin(step_size);
	for (size_t s = 0; s < samples; s++) {
		orc_prepst(amp, nqb, ndets, det_idx, det_cf);
		for (size_t k = 0; k < depth; k++) {
			const double x = orc_rng_dbl01(rng);
			const size_t idx = orc_cdf_inverse(cdf, nterms, x);
			draws[k].cf = orc_signof(terms[idx].cf);
			draws[k].flip = terms[idx].flip;
			draws[k].phase = terms[idx].phase;
		}
		sweep(amp, nqb, draws, depth, omega, 0);
		orc_measure(amp, ndets, det_idx, det_cf, out_z + 2 * s);
	}
	rc = 0;
out:
	free(cdf);
	free(draws);
	free(amp);
	return rc;
}

static int cmp_abscf_desc(const void *a, const void *b)
{
	const double x = fabs(((const struct orc_term *)a)->cf);
	const double y = fabs(((const struct orc_term *)b)->cf);
	if (x > y)
		return -1;
	if (x < y)
		return 1;
	return 0;
}

int orc_cmpsit(uint32_t nqb, const struct orc_term *terms, size_t nterms,
	size_t ndets, const uint64_t *det_idx, const double *det_cf,
	size_t samples, size_t steps, size_t length, size_t depth,
	double angle_det, double angle_rand, uint64_t seed, double *out_z)
{
	/* circ/cmpsit.c:65-111: split by |c| descending into a deterministic
	 * head (then lex-sorted) and a sampled tail with its own CDF. */
	if (length > nterms || nterms - length == 0)
		return -1;
	double *amp = state_alloc(nqb);
	struct orc_term *tmp = terms_copy(terms, nterms);
	const size_t nran = nterms - length;
	double *cdf = malloc(sizeof *cdf * nran);
	struct orc_term *smpl = malloc(sizeof *smpl * (length + depth + 1));
	int rc = -1;
	if (!amp || !tmp || !cdf || !smpl)
		goto out;
	qsort(tmp, nterms, sizeof *tmp, cmp_abscf_desc);
	struct orc_term *det = terms_copy(tmp, length);
	if (!det)
		goto out;
	orc_sort_lex(det, length);
	const struct orc_term *ran = tmp + length;
	double lambda_r = 0.0;
	orc_cdf_build(&ran[0].cf, sizeof ran[0], nran, cdf, &lambda_r);
	uint64_t rng[4];
	orc_rng_init(rng, seed ? seed : ORC_CMPSIT_SEED);
	for (size_t smp = 0; smp < samples; smp++) {
		orc_prepst(amp, nqb, ndets, det_idx, det_cf);
		for (size_t st = 0; st < steps; st++) {
			for (int half = 0; half < 2; half++) {
				/* hm_sample (circ/cmpsit.c:151-177), fresh per half. */
				for (size_t i = 0; i < length; i++) {
					smpl[i].flip = det[i].flip;
					smpl[i].phase = det[i].phase;
					smpl[i].cf = det[i].cf * angle_det;
				}
				for (size_t i = length; i < length + depth; i++) {
					const double x = orc_rng_dbl01(rng);
					const size_t idx =
						orc_cdf_inverse(cdf, nran, x);
					smpl[i].flip = ran[idx].flip;
					smpl[i].phase = ran[idx].phase;
					smpl[i].cf = orc_signof(ran[idx].cf) *
						angle_rand;
				}
				sweep(amp, nqb, smpl, length + depth, 0.5, half);
			}
		}
		orc_measure(amp, ndets, det_idx, det_cf, out_z + 2 * smp);
	}
	free(det);
	rc = 0;
out:
	free(smpl);
	free(cdf);
	free(tmp);
	free(amp);
	return rc;
}

/* ---- one-shot entry (phase2/phase2_run.c:43-174) ------------------------ */

static int parse_basis(const char *s, uint32_t nqb, uint64_t *out)
{
	*out = 0;
	for (uint32_t k = 0; k < nqb; k++) {
		if (s[k] == '1')
			*out |= UINT64_C(1) << k;
		else if (s[k] != '0')
			return -1;
	}
	return 0;
}

static int parse_pauli(const char *s, uint32_t nqb, uint64_t *flip,
	uint64_t *phase)
{
	char buf[4096];
	const size_t len = strlen(s);
	if (len >= sizeof buf)
		return -1;
	memcpy(buf, s, len + 1);
	*flip = *phase = 0;
	char *save = NULL;
	for (char *tok = strtok_r(buf, " \t\n", &save); tok;
		tok = strtok_r(NULL, " \t\n", &save)) {
		int f, p;
		switch (tok[0]) {
		case 'I':
			f = 0, p = 0;
			break;
		case 'X':
			f = 1, p = 0;
			break;
		case 'Y':
			f = 1, p = 1;
			break;
		case 'Z':
			f = 0, p = 1;
			break;
		default:
			return -1;
		}
		char *end;
		const unsigned long q = strtoul(tok + 1, &end, 10);
		if (end == tok + 1 || *end != '\0' || q >= nqb)
			return -1;
		const uint64_t m = UINT64_C(1) << q;
		*flip = f ? (*flip | m) : (*flip & ~m);
		*phase = p ? (*phase | m) : (*phase & ~m);
	}
	return 0;
}

int orc_phase2_run(const char **pauli_strs, const double *coeffs,
	size_t nterms, double delta, const char *psi_str, double *out_re,
	double *out_im)
{
	if (!psi_str)
		return -1;
	const size_t nqb = strlen(psi_str);
	if (nqb == 0 || nqb > 30)
		return -1;
	uint64_t idx;
	if (parse_basis(psi_str, (uint32_t)nqb, &idx) < 0)
		return -1;
	double *amp = state_alloc((uint32_t)nqb);
	if (!amp)
		return -1;
	memset(amp, 0, sizeof(double) * 2 * (UINT64_C(1) << nqb));
	amp[2 * idx] = 1.0;
	for (size_t k = 0; k < nterms; k++) {
		uint64_t f, p;
		if (parse_pauli(pauli_strs[k], (uint32_t)nqb, &f, &p) < 0) {
			free(amp);
			return -1;
		}
		orc_rotate(amp, (uint32_t)nqb, f, p, delta * coeffs[k]);
	}
	*out_re = amp[2 * idx];
	*out_im = amp[2 * idx + 1];
	free(amp);
	return 0;
}

double orc_norm2(const double *amp, uint32_t nqb)
{
	double s = 0.0;
	const uint64_t n = UINT64_C(1) << nqb;
	for (uint64_t i = 0; i < 2 * n; i++)
		s += amp[i] * amp[i];
	return s;
}

/* ---- coefficient-matrix trial state ------------------------------------ */

#define ORC_CM_MAX_K 32

/* k-subsets of {0..n-1} in lex order (lib/combinations.c:45-98); returns
 * the count, tuples of k entries in out (NULL: count only). */
static size_t orc_subsets(uint32_t n, uint32_t k, uint32_t *out)
{
	uint32_t c[ORC_CM_MAX_K];
	if (k > n || k > ORC_CM_MAX_K)
		return 0;
	for (uint32_t i = 0; i < k; i++)
		c[i] = i;
	size_t m = 0;
	for (;;) {
		if (out)
			memcpy(out + m * (k ? k : 1), c, sizeof(uint32_t) * k);
		m++;
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

/* LU with partial pivoting (lib/det_small.c:27-71); a is overwritten. */
static double orc_det(double *a, uint32_t n)
{
	if (n == 0)
		return 1.0;
	double det = 1.0;
	for (uint32_t k = 0; k < n; k++) {
		uint32_t piv = k;
		double mx = fabs(a[k * n + k]);
		for (uint32_t i = k + 1; i < n; i++)
			if (fabs(a[i * n + k]) > mx) {
				mx = fabs(a[i * n + k]);
				piv = i;
			}
		if (mx == 0.0)
			return 0.0;
		if (piv != k) {
			for (uint32_t j = k; j < n; j++) {
				const double t = a[k * n + j];
				a[k * n + j] = a[piv * n + j];
				a[piv * n + j] = t;
			}
			det = -det;
		}
		const double p = a[k * n + k];
		det *= p;
		const double ip = 1.0 / p;
		for (uint32_t i = k + 1; i < n; i++) {
			const double f = a[i * n + k] * ip;
			if (f == 0.0)
				continue;
			for (uint32_t j = k + 1; j < n; j++)
				a[i * n + j] -= f * a[k * n + j];
		}
	}
	return det;
}

/* det(C[tuple, :]) for each tuple (state_prep_coeff.c:102-122). */
static void orc_tuple_dets(const double *C, uint32_t k, const uint32_t *tup,
	size_t m, double *out)
{
	double a[ORC_CM_MAX_K * ORC_CM_MAX_K];
	for (size_t i = 0; i < m; i++) {
		for (uint32_t r = 0; r < k; r++)
			for (uint32_t c = 0; c < k; c++)
				a[r * k + c] = C[tup[i * k + r] * k + c];
		out[i] = orc_det(a, k);
	}
}

struct orc_cm {
	uint32_t n_sites, na, nb;
	size_t Ma, Mb;
	uint32_t *ta, *tb;
	double *da, *db;
};

static int orc_cm_init(struct orc_cm *s, uint32_t nqb, uint32_t n_sites,
	uint32_t na, uint32_t nb, int tapered)
{
	memset(s, 0, sizeof *s);
	if (na > n_sites || nb > n_sites || n_sites == 0 || n_sites > 32 ||
		(tapered ? 2 * n_sites - 2 : 2 * n_sites) > nqb)
		return -1;
	s->n_sites = n_sites;
	s->na = na;
	s->nb = nb;
	s->Ma = orc_subsets(n_sites, na, NULL);
	s->Mb = orc_subsets(n_sites, nb, NULL);
	s->ta = malloc(sizeof *s->ta * s->Ma * (na ? na : 1));
	s->tb = malloc(sizeof *s->tb * s->Mb * (nb ? nb : 1));
	s->da = malloc(sizeof *s->da * s->Ma);
	s->db = malloc(sizeof *s->db * s->Mb);
	if (!s->ta || !s->tb || !s->da || !s->db)
		return -1;
	orc_subsets(n_sites, na, s->ta);
	orc_subsets(n_sites, nb, s->tb);
	return 0;
}

static void orc_cm_free(struct orc_cm *s)
{
	free(s->ta);
	free(s->tb);
	free(s->da);
	free(s->db);
}

/* Index of tuple pair (i, j): alpha bits, beta bits above n_sites, and
 * for tapered states bits 0 and n_sites dropped (state_prep_coeff.c:34-54). */
static uint64_t orc_cm_index(const struct orc_cm *s, size_t i, size_t j,
	int tapered)
{
	uint64_t idx = 0;
	for (uint32_t r = 0; r < s->na; r++)
		idx |= UINT64_C(1) << s->ta[i * s->na + r];
	for (uint32_t r = 0; r < s->nb; r++)
		idx |= UINT64_C(1) << (s->n_sites + s->tb[j * s->nb + r]);
	if (tapered) {
		const uint64_t lo =
			(idx >> 1) & ((UINT64_C(1) << (s->n_sites - 1)) - 1);
		idx = lo | ((idx >> (s->n_sites + 1)) << (s->n_sites - 1));
	}
	return idx;
}

/* One block: write (accumulate 0) or add the products weight * da * db
 * not below 1e-12 in magnitude (state_prep_coeff.c:156-196). */
static void orc_cm_block(struct orc_cm *s, const double *Ca, const double *Cb,
	double weight, int tapered, int accumulate, double *amp)
{
	orc_tuple_dets(Ca, s->na, s->ta, s->Ma, s->da);
	orc_tuple_dets(Cb ? Cb : Ca, s->nb, s->tb, s->Mb, s->db);
	for (size_t i = 0; i < s->Ma; i++)
		for (size_t j = 0; j < s->Mb; j++) {
			const double cf = weight * s->da[i] * s->db[j];
			if (fabs(cf) < 1.0e-12)
				continue;
			const uint64_t idx = orc_cm_index(s, i, j, tapered);
			if (accumulate) {
				amp[2 * idx] += cf;
			} else {
				amp[2 * idx] = cf;
				amp[2 * idx + 1] = 0.0;
			}
		}
}

int orc_coeff_expand_all(uint32_t nqb, uint32_t n_sites, uint32_t na,
	uint32_t nb, int tapered, size_t ncomp, const double *w,
	const double *Ca, const double *Cb, double *amp)
{
	struct orc_cm s;
	if (orc_cm_init(&s, nqb, n_sites, na, nb, tapered) < 0) {
		orc_cm_free(&s);
		return -1;
	}
	memset(amp, 0, sizeof(double) * 2 * (UINT64_C(1) << nqb));
	if (ncomp == 0)
		orc_cm_block(&s, Ca, Cb, 1.0, tapered, 0, amp);
	for (size_t k = 0; k < ncomp; k++)
		orc_cm_block(&s, Ca + k * (size_t)n_sites * na,
			Cb ? Cb + k * (size_t)n_sites * nb : NULL, w[k], tapered,
			1, amp);
	orc_cm_free(&s);
	return 0;
}

/* Sequential sum of cf * a over one block (state_prep_coeff.c:199-244). */
static void orc_cm_inner_block(struct orc_cm *s, const double *Ca,
	const double *Cb, double weight, int tapered, const double *amp,
	double *re, double *im)
{
	orc_tuple_dets(Ca, s->na, s->ta, s->Ma, s->da);
	orc_tuple_dets(Cb ? Cb : Ca, s->nb, s->tb, s->Mb, s->db);
	double ar = 0.0, ai = 0.0;
	for (size_t i = 0; i < s->Ma; i++)
		for (size_t j = 0; j < s->Mb; j++) {
			const double cf = weight * s->da[i] * s->db[j];
			if (fabs(cf) < 1.0e-12)
				continue;
			const uint64_t idx = orc_cm_index(s, i, j, tapered);
			ar += cf * amp[2 * idx];
			ai += cf * amp[2 * idx + 1];
		}
	*re = ar;
	*im = ai;
}

int orc_coeff_inner(uint32_t nqb, uint32_t n_sites, uint32_t na, uint32_t nb,
	int tapered, size_t ncomp, const double *w, const double *Ca,
	const double *Cb, const double *amp, double *out)
{
	struct orc_cm s;
	if (orc_cm_init(&s, nqb, n_sites, na, nb, tapered) < 0) {
		orc_cm_free(&s);
		return -1;
	}
	double pr = 0.0, pi = 0.0, zr, zi;
	if (ncomp == 0) {
		orc_cm_inner_block(&s, Ca, Cb, 1.0, tapered, amp, &pr, &pi);
	}
	for (size_t k = 0; k < ncomp; k++) {
		orc_cm_inner_block(&s, Ca + k * (size_t)n_sites * na,
			Cb ? Cb + k * (size_t)n_sites * nb : NULL, w[k], tapered,
			amp, &zr, &zi);
		pr += zr;
		pi += zi;
	}
	out[0] = pr;
	out[1] = pi;
	orc_cm_free(&s);
	return 0;
}
