#ifndef XOSHIRO256SS_H
#define XOSHIRO256SS_H

/*
 * xoshiro256** pseudo-random generator (Blackman and Vigna, "Scrambled
 * Linear Pseudorandom Number Generators", ACM TOMS 47(4), 2021), with
 * explicit state.  Replaces include/xoshiro256ss.h of Quantum-for-Life/
 * phase2 (lines 44-59): same seeding (four splitmix64 outputs, then 128
 * discarded draws) and the same [0,1) double map, so sampled sequences are
 * identical for equal seeds.
 */

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct xoshiro256ss {
	uint64_t s[4];
};

void xoshiro256ss_init(struct xoshiro256ss *rng, uint64_t seed);

uint64_t xoshiro256ss_next(struct xoshiro256ss *rng);

/* Advance by 2^128 / 2^192 draws (reference: xoshiro256ss.h:50-52). */
void xoshiro256ss_jump(struct xoshiro256ss *rng);

void xoshiro256ss_longjump(struct xoshiro256ss *rng);

/* Uniform double in [0,1): top 53 bits times 2^-53. */
#define xoshiro256ss_dbl01(rng)                                                \
	((double)(xoshiro256ss_next(rng) >> 11) * 0x1.0p-53)

#ifdef __cplusplus
}
#endif

#endif /* XOSHIRO256SS_H */
