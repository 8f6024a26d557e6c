#ifndef CIRC_CACHE
#define CIRC_CACHE

/*
 * Rotation batch cache: collects up to 1024 consecutive (Pauli, angle)
 * terms that share one hi-qubit code and hands them to a flush callback.
 * Replaces phase2/circ_cache.h of Quantum-for-Life/phase2 (lines 21-41),
 * exported so that code built against the reference's private header links
 * unchanged.  With one rank every term has the identity hi code, so the
 * cache only bounds batches to 1024 terms.
 */

#include <stddef.h>

#include "phase2/paulis.h"

#ifdef __cplusplus
extern "C" {
#endif

struct circ_cache;

/* NULL on allocation failure (reference: circ_cache.h:21). */
struct circ_cache *circ_cache_init(int hi, int lo);

void circ_cache_free(struct circ_cache *c);

/* 0 on insert; -1 if full or the hi code differs (flush, then retry)
 * (reference: circ_cache.h:28-29). */
int circ_cache_insert(struct circ_cache *c, struct paulis pa, double phi);

/* Call fn with the batch (if non-empty) and empty the cache
 * (reference: circ_cache.h:35-38). */
void circ_cache_flush(struct circ_cache *c,
	void (*fn)(struct paulis hi, const struct paulis *lo, double *phis,
		size_t n, void *data),
	void *data);

size_t circ_cache_len(const struct circ_cache *c);

#ifdef __cplusplus
}
#endif

#endif /* CIRC_CACHE */
