#ifndef PHASE2_RUN_H
#define PHASE2_RUN_H

/*
 * One-shot entry point used by the Python binding.  Replaces
 * include/phase2/phase2_run.h of Quantum-for-Life/phase2 (lines 38-40):
 *
 *   <psi| prod_k exp(i delta coeffs[k] P_k) |psi>
 *
 * pauli_strs[k] are space-separated tokens such as "X0 Z3 Y7" (other qubits
 * identity); psi_str is a bitstring, character k giving qubit k, and its
 * length (1..30) is the qubit count.  Returns 0, or -1 on an invalid token,
 * a qubit index >= strlen(psi_str), a character other than '0'/'1', a bad
 * length, or a failed allocation.  The world is initialised on first use.
 */

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

int phase2_run(const char **pauli_strs, const double *coeffs, size_t nterms,
	double delta, const char *psi_str, double *out_re, double *out_im);

#ifdef __cplusplus
}
#endif

#endif /* PHASE2_RUN_H */
