/*
 * phase2_run.c -- one-shot entry (include/phase2/phase2_run.h), the call
 * behind the Python binding.  Same input rules and errors as
 * phase2/phase2_run.c of Quantum-for-Life/phase2 (lines 16-174): nqb =
 * strlen(psi_str) in [1,30]; tokens "<op><qubit>" with op in IXYZ separated
 * by blanks; qubit < nqb; psi characters '0'/'1' (character k = qubit k);
 * phi_k = delta * coeffs[k], applied in order through the batch cache.
 */
#define _POSIX_C_SOURCE 200809L

#include <complex.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "circ_cache.h"
#include "phase2/phase2_run.h"
#include "phase2/qreg.h"
#include "phase2/world.h"
#include "phase2_b200.h"

#define PH2RUN_SEED UINT64_C(0xa7c3e1b9d4f20586)
#define PH2RUN_MAX_QB 30

static int world_owned;

static void world_release(void)
{
	if (world_owned)
		world_free();
}

static int world_ensure(void)
{
	if (world_info(NULL) == WORLD_READY)
		return 0;
	if (world_init(NULL, NULL, PH2RUN_SEED) != WORLD_READY)
		return -1;
	if (!world_owned) {
		world_owned = 1;
		atexit(world_release);
	}
	return 0;
}

static int basis_index(const char *s, uint32_t nqb, uint64_t *out)
{
	uint64_t v = 0;
	for (uint32_t k = 0; k < nqb; k++) {
		if (s[k] == '1')
			v |= UINT64_C(1) << k;
		else if (s[k] != '0')
			return -1;
	}
	*out = v;
	return 0;
}

static int pauli_parse(const char *s, uint32_t nqb, struct paulis *out)
{
	char buf[4096];
	const size_t len = strlen(s);
	if (len >= sizeof buf)
		return -1;
	memcpy(buf, s, len + 1);
	*out = paulis_new();
	char *save = NULL;
	for (char *tok = strtok_r(buf, " \t\n", &save); tok;
		tok = strtok_r(NULL, " \t\n", &save)) {
		enum pauli_op op;
		switch (tok[0]) {
		case 'I':
			op = PAULI_I;
			break;
		case 'X':
			op = PAULI_X;
			break;
		case 'Y':
			op = PAULI_Y;
			break;
		case 'Z':
			op = PAULI_Z;
			break;
		default:
			return -1;
		}
		char *end;
		const unsigned long q = strtoul(tok + 1, &end, 10);
		if (end == tok + 1 || *end != '\0' || q >= nqb)
			return -1;
		paulis_set(out, op, (uint32_t)q);
	}
	return 0;
}

static void flush_cb(struct paulis hi, const struct paulis *lo, double *phis,
	size_t n, void *data)
{
	qreg_paulirot((struct qreg *)data, hi, lo, phis, n);
}

int phase2_run(const char **pauli_strs, const double *coeffs, size_t nterms,
	double delta, const char *psi_str, double *out_re, double *out_im)
{
	if (!psi_str)
		return -1;
	const size_t nqb = strlen(psi_str);
	if (nqb == 0 || nqb > PH2RUN_MAX_QB)
		return -1;
	if (world_ensure() < 0)
		return -1;
	uint64_t idx;
	if (basis_index(psi_str, (uint32_t)nqb, &idx) < 0)
		return -1;
	struct qreg reg;
	if (qreg_init(&reg, (uint32_t)nqb) < 0)
		return -1;
	qreg_zero(&reg);
	qreg_setamp(&reg, idx, 1.0);
	struct circ_cache *cache = circ_cache_init((int)reg.qb_hi,
		(int)reg.qb_lo);
	if (!cache)
		goto fail_reg;
	for (size_t k = 0; k < nterms; k++) {
		struct paulis code;
		if (pauli_parse(pauli_strs[k], (uint32_t)nqb, &code) < 0)
			goto fail_cache;
		const double phi = delta * coeffs[k];
		if (circ_cache_insert(cache, code, phi) != 0) {
			circ_cache_flush(cache, flush_cb, &reg);
			if (circ_cache_insert(cache, code, phi) < 0)
				goto fail_cache;
		}
	}
	circ_cache_flush(cache, flush_cb, &reg);
	_Complex double z = 0.0;
	if (qreg_getamps(&reg, &idx, &z, 1) < 0)
		goto fail_cache;
	*out_re = creal(z);
	*out_im = cimag(z);
	circ_cache_free(cache);
	qreg_free(&reg);
	return 0;

fail_cache:
	circ_cache_free(cache);
fail_reg:
	qreg_free(&reg);
	return -1;
}
