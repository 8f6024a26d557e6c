/*
 * phase2_run.c -- the one-shot call behind the Python binding
 * (include/phase2/phase2_run.h):
 *
 *   <psi| prod_k exp(i delta coeffs[k] P_k) |psi>,  psi a basis state.
 *
 * Contract (the reference's phase2/phase2_run.c:115-174): the qubit count
 * is strlen(psi_str), 1..30; psi_str holds '0'/'1', character k giving
 * qubit k; each Pauli string is a list of tokens "<op><index>" (op one of
 * I X Y Z, index a decimal qubit number below the qubit count) separated
 * by spaces, tabs or newlines, later tokens for the same qubit replacing
 * earlier ones; rotation k has angle delta * coeffs[k] and the rotations
 * apply in input order.  Any violation returns -1.  The world is brought
 * up on first use and released at process exit.
 *
 * Design: each string is scanned once, in place, straight into the
 * rotation's flip and phase masks, and the rotation goes directly into
 * the register's rotation queue (qreg_paulirot), which plans and fuses
 * the whole sequence; one GPU holds the register, so there is no hi/lo
 * split to group by and no batch cache in between.  The index grammar is
 * what the reference's strtoul(..., 10) accepts inside a token: optional
 * white space of the kinds that do not separate tokens (\v \f \r), an
 * optional sign, at least one digit, then the end of the token; "-0" is 0
 * and any other negative or too large value is out of range.  Unlike the
 * reference, a string is not copied into a 4096-byte buffer, so strings
 * of any length are accepted.
 */
#include <complex.h>
#include <stdint.h>
#include <stdlib.h>

#include "phase2/phase2_run.h"
#include "phase2/qreg.h"
#include "phase2/world.h"
#include "phase2_b200.h"

#define RUN_MAX_QUBITS 30
#define RUN_WORLD_SEED UINT64_C(0x3c6ef372fe94f82b)

static int run_world_owned;

static void run_world_release(void)
{
	if (run_world_owned)
		world_free();
}

static int run_world(void)
{
	if (world_info(NULL) == WORLD_READY)
		return 0;
	if (world_init(NULL, NULL, RUN_WORLD_SEED) != WORLD_READY)
		return -1;
	if (!run_world_owned) {
		run_world_owned = 1;
		atexit(run_world_release);
	}
	return 0;
}

static int is_separator(char c)
{
	return c == ' ' || c == '\t' || c == '\n';
}

/* Qubit index at *pp, up to the end of the token; advances *pp.  -1 when
 * the token's tail is not an index below nqb. */
static long scan_index(const char **pp, uint32_t nqb)
{
	const char *p = *pp;
	while (*p == '\v' || *p == '\f' || *p == '\r')
		p++;
	int negative = 0;
	if (*p == '+' || *p == '-')
		negative = *p++ == '-';
	uint64_t v = 0;
	const char *digits = p;
	for (; *p >= '0' && *p <= '9'; p++)
		if (v <= UINT32_MAX) /* saturates well above any qubit count */
			v = v * 10 + (uint64_t)(*p - '0');
	if (p == digits || (*p != '\0' && !is_separator(*p)))
		return -1;
	if ((negative && v != 0) || v >= nqb)
		return -1;
	*pp = p;
	return (long)v;
}

/* Flip and phase masks of one Pauli string (I: 0/0, X: 1/0, Y: 1/1,
 * Z: 0/1 at the qubit), or -1. */
static int scan_string(const char *s, uint32_t nqb, struct paulis *out)
{
	uint64_t flip = 0, phase = 0;
	const char *p = s;
	for (;;) {
		while (is_separator(*p))
			p++;
		if (*p == '\0')
			break;
		const char op = *p++;
		if (op != 'I' && op != 'X' && op != 'Y' && op != 'Z')
			return -1;
		const long q = scan_index(&p, nqb);
		if (q < 0)
			return -1;
		const uint64_t bit = UINT64_C(1) << q;
		flip &= ~bit;
		phase &= ~bit;
		if (op == 'X' || op == 'Y')
			flip |= bit;
		if (op == 'Y' || op == 'Z')
			phase |= bit;
	}
	*out = paulis_new();
	out->pak[0] = flip;
	out->pak[1] = phase;
	return 0;
}

/* Basis index of psi (character k = qubit k), or -1. */
static int scan_basis(const char *psi, uint32_t nqb, uint64_t *out)
{
	uint64_t v = 0;
	for (uint32_t k = 0; k < nqb; k++) {
		if (psi[k] != '0' && psi[k] != '1')
			return -1;
		v |= (uint64_t)(psi[k] - '0') << k;
	}
	*out = v;
	return 0;
}

int phase2_run(const char **pauli_strs, const double *coeffs, size_t nterms,
	double delta, const char *psi_str, double *out_re, double *out_im)
{
	if (!psi_str || (nterms && (!pauli_strs || !coeffs)))
		return -1;
	size_t len = 0;
	while (len <= RUN_MAX_QUBITS && psi_str[len])
		len++;
	if (len == 0 || len > RUN_MAX_QUBITS)
		return -1;
	const uint32_t nqb = (uint32_t)len;
	if (run_world() < 0)
		return -1;
	uint64_t basis;
	if (scan_basis(psi_str, nqb, &basis) < 0)
		return -1;

	struct qreg reg;
	if (qreg_init(&reg, nqb) < 0)
		return -1;
	int rc = -1;
	qreg_zero(&reg);
	qreg_setamp(&reg, basis, 1.0);
	const struct paulis none = paulis_new();
	size_t k = 0;
	for (; k < nterms; k++) {
		struct paulis code;
		if (!pauli_strs[k] || scan_string(pauli_strs[k], nqb, &code) < 0)
			break;
		const double phi = delta * coeffs[k];
		qreg_paulirot(&reg, none, &code, &phi, 1);
	}
	_Complex double z = 0.0;
	if (k == nterms && qreg_getamps(&reg, &basis, &z, 1) == 0) {
		*out_re = creal(z);
		*out_im = cimag(z);
		rc = 0;
	}
	qreg_free(&reg);
	return rc;
}
