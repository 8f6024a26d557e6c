/*
 * paulis.c -- Pauli strings in (flip, phase) form.  Same semantics as
 * phase2/paulis.c of Quantum-for-Life/phase2 (lines 9-205).
 */
#include <complex.h>
#include <stdint.h>

#include "phase2/paulis.h"
#include "phase2/qreg.h"

struct paulis paulis_new(void)
{
	struct paulis p = { { 0, 0 } };
	return p;
}

/* Two-bit code (phase << 1 | flip): 0 I, 1 X, 2 Z, 3 Y. */
enum pauli_op paulis_get(struct paulis code, uint32_t n)
{
	static const enum pauli_op by_bits[4] = { PAULI_I, PAULI_X, PAULI_Z,
		PAULI_Y };
	const unsigned bits = (unsigned)(code.pak[0] >> n & 1) |
		(unsigned)(code.pak[1] >> n & 1) << 1;
	return by_bits[bits];
}

void paulis_set(struct paulis *code, enum pauli_op op, uint32_t n)
{
	const uint64_t m = UINT64_C(1) << n;
	int f, p;
	switch (op) {
	case PAULI_I:
		f = 0, p = 0;
		break;
	case PAULI_X:
		f = 1, p = 0;
		break;
	case PAULI_Y:
		f = 1, p = 1;
		break;
	case PAULI_Z:
		f = 0, p = 1;
		break;
	default:
		return;
	}
	code->pak[0] = f ? code->pak[0] | m : code->pak[0] & ~m;
	code->pak[1] = p ? code->pak[1] | m : code->pak[1] & ~m;
}

int paulis_eq(struct paulis a, struct paulis b)
{
	return a.pak[0] == b.pak[0] && a.pak[1] == b.pak[1];
}

void paulis_shl(struct paulis *code, uint32_t n)
{
	code->pak[0] <<= n;
	code->pak[1] <<= n;
}

void paulis_shr(struct paulis *code, uint32_t n)
{
	code->pak[0] >>= n;
	code->pak[1] >>= n;
}

uint64_t paulis_effect(struct paulis code, uint64_t i, _Complex double *z)
{
	int r;
	const uint64_t j = paulis_effect_raw(code, i, &r);
	if (!z)
		return j;
	/* multiply by i^r; r = 0 leaves *z untouched */
	if (r == 1)
		*z *= I;
	else if (r == 2)
		*z *= -1.0;
	else if (r == 3)
		*z *= -I;
	return j;
}

void paulis_split(struct paulis code, uint32_t qb_lo, uint32_t qb_hi,
	struct paulis *lo, struct paulis *hi)
{
	const uint64_t lo_m = qb_lo >= 64 ? ~UINT64_C(0)
					  : (UINT64_C(1) << qb_lo) - 1;
	const uint32_t top = qb_lo + qb_hi;
	const uint64_t all_m = top >= 64 ? ~UINT64_C(0)
					 : (UINT64_C(1) << top) - 1;
	const uint64_t hi_m = all_m & ~lo_m;
	lo->pak[0] = code.pak[0] & lo_m;
	lo->pak[1] = code.pak[1] & lo_m;
	hi->pak[0] = code.pak[0] & hi_m;
	hi->pak[1] = code.pak[1] & hi_m;
}

int paulis_cmp(struct paulis a, struct paulis b)
{
	const uint64_t diff = (a.pak[0] ^ b.pak[0]) | (a.pak[1] ^ b.pak[1]);
	if (!diff)
		return 0;
	/* the highest differing qubit decides, by enum pauli_op value */
	const uint32_t q = (uint32_t)(63 - __builtin_clzll(diff));
	return paulis_get(a, q) < paulis_get(b, q) ? -1 : 1;
}
