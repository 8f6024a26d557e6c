#ifndef PAULIS_H
#define PAULIS_H

/*
 * Pauli strings on up to 64 qubits in symplectic (flip, phase) form.
 *
 * Replaces include/phase2/paulis.h of Quantum-for-Life/phase2 (lines
 * 30-169) with the same types, values and semantics:
 *
 *   pak[0]  flip mask:  bit k set iff qubit k carries X or Y
 *   pak[1]  phase mask: bit k set iff qubit k carries Z or Y
 *
 * so that P|i> = i^r |i ^ pak[0]> with
 * r = (popcount(pak[0] & pak[1]) + 2 popcount(i & pak[1])) mod 4.
 * Qubit indices are in [0, 64).
 */

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Operator codes; the integer values are part of the ABI
 * (reference: include/phase2/paulis.h:38-43). */
enum pauli_op {
	PAULI_I = 0,
	PAULI_X = 1,
	PAULI_Y = 2,
	PAULI_Z = 3,
};

/* Reference: include/phase2/paulis.h:56-58. */
struct paulis {
	uint64_t pak[2];
};

/* All-identity string (reference: paulis.h:61). */
struct paulis paulis_new(void);

/* Operator on qubit n (reference: paulis.h:67). */
enum pauli_op paulis_get(struct paulis code, uint32_t n);

/* Set the operator on qubit n; an unknown op leaves the string unchanged
 * (reference: paulis.h:76). */
void paulis_set(struct paulis *code, enum pauli_op op, uint32_t n);

/* 1 iff both masks are equal (reference: paulis.h:83). */
int paulis_eq(struct paulis code1, struct paulis code2);

/* Shift both masks by n qubits (reference: paulis.h:94-95). */
void paulis_shl(struct paulis *code, uint32_t n);
void paulis_shr(struct paulis *code, uint32_t n);

/* P|i> = z |j>: returns j and multiplies *z by the phase i^r; z may be
 * NULL (reference: paulis.h:110). */
uint64_t paulis_effect(struct paulis code, uint64_t i, _Complex double *z);

/*
 * Integer core shared by host and device code: returns j = i ^ flip and
 * stores r in [0,4) such that P|i> = i^r |j> (reference: paulis.h:137-144).
 */
#if defined(__CUDACC__)
#define PHASE2_HD __host__ __device__
#else
#define PHASE2_HD
#endif
PHASE2_HD static inline uint64_t paulis_effect_raw(struct paulis code,
	uint64_t i, int *r4_out)
{
	const int ny = __builtin_popcountll(code.pak[0] & code.pak[1]);
	const int nm = __builtin_popcountll(i & code.pak[1]);
	*r4_out = (ny + 2 * nm) & 3;
	return i ^ code.pak[0];
}
#undef PHASE2_HD

/* Keep qubits [0,qb_lo) in *lo and [qb_lo, qb_lo+qb_hi) in *hi
 * (reference: paulis.h:157-158). */
void paulis_split(struct paulis code, uint32_t qb_lo, uint32_t qb_hi,
	struct paulis *lo, struct paulis *hi);

/* Lexicographic order from qubit 63 down, I < X < Y < Z; returns -1, 0,
 * +1 (reference: paulis.h:167). */
int paulis_cmp(struct paulis a, struct paulis b);

#ifdef __cplusplus
}
#endif

#endif /* PAULIS_H */
