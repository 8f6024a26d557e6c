#ifndef PROB_H
#define PROB_H

/*
 * Discrete CDF of |w| and inverse-CDF sampling, as used by the qDRIFT and
 * composite samplers.  Replaces include/prob.h of Quantum-for-Life/phase2
 * (lines 11-33) with the same contract; results are bit-identical (same
 * summation order), which keeps the sampled term sequences identical.
 */

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

struct prob_cdf {
	double *y;
	size_t len;
};

/* Allocate y for len > 0 entries; -1 on len == 0 or allocation failure
 * (reference: prob.h:20). */
int prob_cdf_init(struct prob_cdf *cdf, size_t len);

/* Free y and zero the struct; repeat calls are safe (reference: prob.h:24). */
void prob_cdf_free(struct prob_cdf *cdf);

/* y[i] = running sum of |w[k]| / lambda over cdf->len weights read at byte
 * stride `stride` from base; *out_lambda = lambda if non-NULL.  -1 if
 * lambda < DBL_EPSILON (reference: prob.h:30-31). */
int prob_cdf_from_array_strided(struct prob_cdf *cdf, const double *base,
	size_t stride, double *out_lambda);

/* Smallest i with y[i] > y, or len-1 (reference: prob.h:34). */
size_t prob_cdf_inverse(const struct prob_cdf *cdf, double y);

#ifdef __cplusplus
}
#endif

#endif /* PROB_H */
