/*
 * prob.c -- |w| CDF and inverse-CDF sampling.  Same results as lib/prob.c
 * of Quantum-for-Life/phase2 (lines 16-78): the CDF is the running sum of
 * |w_i| / lambda in index order, and the inverse returns the smallest i with
 * y[i] > y (clamped to len-1); here the inverse is a plain upper-bound
 * binary search, which returns the same index on any non-decreasing y.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>

#include "prob.h"

int prob_cdf_init(struct prob_cdf *cdf, size_t len)
{
	if (len == 0)
		return -1;
	double *y = malloc(sizeof *y * len);
	if (!y)
		return -1;
	cdf->y = y;
	cdf->len = len;
	return 0;
}

void prob_cdf_free(struct prob_cdf *cdf)
{
	free(cdf->y);
	cdf->y = NULL;
	cdf->len = 0;
}

int prob_cdf_from_array_strided(struct prob_cdf *cdf, const double *base,
	size_t stride, double *out_lambda)
{
	double lambda = 0.0;
	for (size_t i = 0; i < cdf->len; i++) {
		const double w =
			fabs(*(const double *)((const char *)base + i * stride));
		cdf->y[i] = w;
		lambda += w;
	}
	if (lambda < DBL_EPSILON)
		return -1;
	double acc = 0.0;
	for (size_t i = 0; i < cdf->len; i++) {
		acc += cdf->y[i] / lambda;
		cdf->y[i] = acc;
	}
	if (out_lambda)
		*out_lambda = lambda;
	return 0;
}

size_t prob_cdf_inverse(const struct prob_cdf *cdf, double y)
{
	size_t lo = 0, hi = cdf->len;
	while (lo < hi) {
		const size_t mid = lo + (hi - lo) / 2;
		if (cdf->y[mid] <= y)
			lo = mid + 1;
		else
			hi = mid;
	}
	return lo < cdf->len ? lo : cdf->len - 1;
}
