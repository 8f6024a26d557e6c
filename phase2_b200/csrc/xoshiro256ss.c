/*
 * xoshiro256ss.c -- xoshiro256** 1.0 (Blackman and Vigna, ACM TOMS 47(4),
 * 2021; published reference algorithm, public domain), with explicit state,
 * splitmix64 seeding and 128 discarded draws as lib/xoshiro256ss.c of
 * Quantum-for-Life/phase2 (lines 34-54) does, so equal seeds give equal
 * sequences.  The jump polynomials are the published constants of the
 * algorithm.
 */
#include <stddef.h>
#include <stdint.h>

#include "xoshiro256ss.h"

static uint64_t splitmix64_next(uint64_t *x)
{
	uint64_t z = (*x += UINT64_C(0x9e3779b97f4a7c15));
	z = (z ^ (z >> 30)) * UINT64_C(0xbf58476d1ce4e5b9);
	z = (z ^ (z >> 27)) * UINT64_C(0x94d049bb133111eb);
	return z ^ (z >> 31);
}

static inline uint64_t rol64(uint64_t x, int k)
{
	return (x << k) | (x >> (64 - k));
}

uint64_t xoshiro256ss_next(struct xoshiro256ss *rng)
{
	uint64_t *s = rng->s;
	const uint64_t out = rol64(s[1] * 5, 7) * 9;
	const uint64_t t = s[1] << 17;
	s[2] ^= s[0];
	s[3] ^= s[1];
	s[1] ^= s[2];
	s[0] ^= s[3];
	s[2] ^= t;
	s[3] = rol64(s[3], 45);
	return out;
}

void xoshiro256ss_init(struct xoshiro256ss *rng, uint64_t seed)
{
	uint64_t x = seed;
	for (int k = 0; k < 4; k++)
		rng->s[k] = splitmix64_next(&x);
	for (int k = 0; k < 128; k++)
		(void)xoshiro256ss_next(rng);
}

static void jump_by(struct xoshiro256ss *rng, const uint64_t poly[4])
{
	uint64_t acc[4] = { 0, 0, 0, 0 };
	for (int w = 0; w < 4; w++)
		for (int b = 0; b < 64; b++) {
			if (poly[w] >> b & 1)
				for (int k = 0; k < 4; k++)
					acc[k] ^= rng->s[k];
			(void)xoshiro256ss_next(rng);
		}
	for (int k = 0; k < 4; k++)
		rng->s[k] = acc[k];
}

void xoshiro256ss_jump(struct xoshiro256ss *rng)
{
	static const uint64_t poly[4] = { UINT64_C(0x180ec6d33cfd0aba),
		UINT64_C(0xd5a61266f0c9392c), UINT64_C(0xa9582618e03fc9aa),
		UINT64_C(0x39abdc4529b1661c) };
	jump_by(rng, poly);
}

void xoshiro256ss_longjump(struct xoshiro256ss *rng)
{
	static const uint64_t poly[4] = { UINT64_C(0x76e15d3efefdcbbf),
		UINT64_C(0xc5004e441c522fb3), UINT64_C(0x77710069854ee241),
		UINT64_C(0x39109bb02acbe635) };
	jump_by(rng, poly);
}
