/*
 * circ_cache.c -- rotation batch cache with the contract of
 * phase2/circ_cache.c of Quantum-for-Life/phase2 (lines 30-95): up to
 * CACHE_MAX = 1024 consecutive terms sharing one hi code; insert returns -1
 * when the batch is full or the hi code changes, flush hands the batch to
 * a callback and empties the cache.
 */
#include <stdlib.h>

#include "circ_cache.h"

#define CACHE_MAX 1024

struct circ_cache {
	int qb_hi, qb_lo;
	size_t len;
	struct paulis hi;
	struct paulis lo[CACHE_MAX];
	double phis[CACHE_MAX];
};

struct circ_cache *circ_cache_init(int hi, int lo)
{
	struct circ_cache *c = calloc(1, sizeof *c);
	if (!c)
		return NULL;
	c->qb_hi = hi;
	c->qb_lo = lo;
	return c;
}

void circ_cache_free(struct circ_cache *c)
{
	free(c);
}

int circ_cache_insert(struct circ_cache *c, struct paulis pa, double phi)
{
	struct paulis lo, hi;
	paulis_split(pa, (uint32_t)c->qb_lo, (uint32_t)c->qb_hi, &lo, &hi);
	if (c->len > 0 && (c->len == CACHE_MAX || !paulis_eq(c->hi, hi)))
		return -1;
	if (c->len == 0)
		c->hi = hi;
	c->lo[c->len] = lo;
	c->phis[c->len] = phi;
	c->len++;
	return 0;
}

void circ_cache_flush(struct circ_cache *c,
	void (*fn)(struct paulis hi, const struct paulis *lo, double *phis,
		size_t n, void *data),
	void *data)
{
	if (c->len > 0 && fn)
		fn(c->hi, c->lo, c->phis, c->len, data);
	c->len = 0;
}

size_t circ_cache_len(const struct circ_cache *c)
{
	return c->len;
}
