/*
 * qreg.c -- the register API (include/phase2/qreg.h) over the device
 * engine.  Replaces phase2/qreg.c + phase2/qreg_cuda.c of
 * Quantum-for-Life/phase2 for one rank.
 *
 * The reference applies a batch with a partner exchange, a projector split
 * into two buffers, two rotation launches per term and a recombination
 * (phase2/qreg_cuda_lo.cu:111-131).  With one rank the exchange is a self
 * copy and the second buffer is identically zero, so all of that reduces
 * to applying the rotations in order to the one state; this file queues
 * them and hands planned passes to the engine.  Observing calls drain the
 * queue first, so the state seen by any caller is the one the reference
 * would produce.
 */
#include <complex.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "qreg"
#include "log.h"

#include "phase2/qreg.h"
#include "phase2_b200.h"

#include "p2_host.h"
#include "p2_internal.h"

/* Host shadow reg->amp is allocated eagerly up to this width. */
#define QREG_EAGER_SHADOW_QB 24

static struct p2_qreg *B(const struct qreg *reg)
{
	return (struct p2_qreg *)reg->backend;
}

int p2_qreg_error(const struct qreg *reg)
{
	const struct p2_qreg *b = B(reg);
	return (!b || b->error) ? -1 : 0;
}

int qreg_init_prec(struct qreg *reg, uint32_t nqb, int prec)
{
	memset(reg, 0, sizeof *reg);
	if (world_info(&reg->wd) != WORLD_READY) {
		log_error("qreg_init: world not ready");
		return -1;
	}
	if (nqb == 0 || nqb > QREG_MAX_WIDTH) {
		log_error("qreg_init: nqb=%u out of range", nqb);
		return -1;
	}
	struct p2_qreg *b = calloc(1, sizeof *b);
	if (!b)
		return -1;
	b->prec = prec;
	b->max_span = p2_cfg.max_span;
	b->max_rots = p2_cfg.max_rots;
	b->dev = p2d_create(nqb, prec);
	if (!b->dev) {
		log_error("qreg_init: device state for %u qubits failed", nqb);
		free(b);
		return -1;
	}
	reg->qb_lo = nqb;
	reg->qb_hi = 0;
	reg->namp = UINT64_C(1) << nqb;
	reg->backend = b;
	if (nqb <= QREG_EAGER_SHADOW_QB) {
		reg->amp = calloc(reg->namp, sizeof *reg->amp);
		if (!reg->amp) {
			qreg_free(reg);
			return -1;
		}
	}
	log_debug("qreg_init: nqb=%u prec=%d", nqb, prec);
	return 0;
}

int qreg_init(struct qreg *reg, uint32_t nqb)
{
	return qreg_init_prec(reg, nqb, p2_cfg.prec);
}

void qreg_free(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (b) {
		p2d_destroy(b->dev);
		free(b->q);
		free(b->passes);
		free(b->recs);
		free(b);
	}
	free(reg->amp);
	reg->amp = NULL;
	reg->backend = NULL;
}

int qreg_precision(const struct qreg *reg)
{
	const struct p2_qreg *b = B(reg);
	return b ? b->prec : -1;
}

int qreg_set_fusion(struct qreg *reg, int max_span, int max_rots)
{
	struct p2_qreg *b = B(reg);
	if (!b || max_span < 1 || max_span > PHASE2_MAX_SPAN || max_rots < 0)
		return -1;
	if (qreg_flush(reg) < 0)
		return -1;
	b->max_span = max_span;
	b->max_rots = max_rots;
	return 0;
}

int qreg_flush(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (!b)
		return -1;
	if (b->qlen == 0)
		return b->error;
	if (b->plan_cap < b->qlen) {
		free(b->passes);
		free(b->recs);
		b->passes = malloc(sizeof *b->passes * b->qlen);
		b->recs = malloc(sizeof *b->recs * b->qlen);
		if (!b->passes || !b->recs) {
			free(b->passes);
			free(b->recs);
			b->passes = NULL;
			b->recs = NULL;
			b->plan_cap = 0;
			b->error = -1;
			return -1;
		}
		b->plan_cap = b->qlen;
	}
	const long np = p2_plan(reg->qb_lo, b->q, b->qlen, b->max_span,
		b->max_rots, P2_DEFAULT_PAD_SPAN, b->passes, b->recs);
	if (np < 0 || p2d_run(b->dev, b->passes, (size_t)np, b->recs,
			      b->qlen) < 0) {
		log_error("qreg_flush: %zu rotations failed", b->qlen);
		b->error = -1;
	}
	b->qlen = 0;
	return b->error;
}

int qreg_synchronize(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	if (p2d_sync(b->dev) < 0)
		b->error = -1;
	return b->error;
}

void qreg_paulirot(struct qreg *reg, struct paulis code_hi,
	const struct paulis *codes_lo, const double *phis, size_t ncodes)
{
	struct p2_qreg *b = B(reg);
	if (!b)
		return;
	/* Operators beyond the register's qubits are dropped, as the
	 * reference's hi/lo split does (phase2/paulis.c:165-180). */
	const uint64_t m = reg->qb_lo >= 64 ? ~UINT64_C(0)
					    : (UINT64_C(1) << reg->qb_lo) - 1;
	for (size_t k = 0; k < ncodes; k++) {
		if (b->qlen == b->qcap) {
			const size_t cap = b->qcap ? 2 * b->qcap : 1024;
			struct phase2_rot_in *q =
				realloc(b->q, sizeof *q * cap);
			if (!q) {
				log_error("qreg_paulirot: queue growth failed");
				b->error = -1;
				return;
			}
			b->q = q;
			b->qcap = cap;
		}
		struct phase2_rot_in *r = &b->q[b->qlen++];
		r->flip = (code_hi.pak[0] | codes_lo[k].pak[0]) & m;
		r->phase = (code_hi.pak[1] | codes_lo[k].pak[1]) & m;
		r->phi = phis[k];
		if (b->qlen >= P2_QUEUE_FLUSH)
			qreg_flush(reg);
	}
}

int qreg_getamps(struct qreg *reg, const uint64_t *idx, _Complex double *z,
	size_t n)
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	/* _Complex double is laid out as two doubles (re, im) */
	if (p2d_get(b->dev, idx, (double *)z, n) < 0) {
		b->error = -1;
		return -1;
	}
	return 0;
}

int qreg_setamps(struct qreg *reg, const uint64_t *idx,
	const _Complex double *z, size_t n)
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	if (p2d_set(b->dev, idx, (const double *)z, n) < 0) {
		b->error = -1;
		return -1;
	}
	return 0;
}

void qreg_getamp(struct qreg *reg, uint64_t i, _Complex double *z)
{
	if (qreg_getamps(reg, &i, z, 1) < 0)
		log_error("qreg_getamp: index %llu failed",
			(unsigned long long)i);
}

void qreg_setamp(struct qreg *reg, uint64_t i, _Complex double z)
{
	if (qreg_setamps(reg, &i, &z, 1) < 0)
		log_error("qreg_setamp: index %llu failed",
			(unsigned long long)i);
}

void qreg_zero(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (!b)
		return;
	/* queued rotations act on a state about to be overwritten */
	b->qlen = 0;
	if (p2d_zero(b->dev) < 0)
		b->error = -1;
}

int qreg_get_state(struct qreg *reg, double *out)
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	return p2d_get_state(b->dev, out);
}

int qreg_set_state(struct qreg *reg, const double *in)
{
	struct p2_qreg *b = B(reg);
	if (!b)
		return -1;
	b->qlen = 0;
	return p2d_set_state(b->dev, in);
}

void qreg_sync_host_to_device(struct qreg *reg)
{
	if (!reg->amp) {
		log_error("qreg_sync_host_to_device: no host shadow (call"
			  " qreg_sync_device_to_host first above %d qubits)",
			QREG_EAGER_SHADOW_QB);
		return;
	}
	if (qreg_set_state(reg, (const double *)reg->amp) < 0)
		log_error("qreg_sync_host_to_device failed");
}

void qreg_sync_device_to_host(struct qreg *reg)
{
	if (!reg->amp) {
		reg->amp = malloc(sizeof *reg->amp * reg->namp);
		if (!reg->amp) {
			log_error("qreg_sync_device_to_host: host shadow"
				  " allocation failed");
			return;
		}
	}
	if (qreg_get_state(reg, (double *)reg->amp) < 0)
		log_error("qreg_sync_device_to_host failed");
}

int qreg_norm2(struct qreg *reg, double *out)
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	return p2d_norm2(b->dev, out);
}

int qreg_inner_dense(struct qreg *reg, const double *trial, double out[2])
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	return p2d_inner_dense(b->dev, trial, out);
}

int qreg_get_stats(const struct qreg *reg, struct phase2_stats *st)
{
	const struct p2_qreg *b = B(reg);
	if (!b || !st)
		return -1;
	p2d_stats(b->dev, st);
	return 0;
}

void qreg_reset_stats(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (b)
		p2d_stats_reset(b->dev);
}

int qreg_set_timing(struct qreg *reg, int on)
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	p2d_set_timing(b->dev, on);
	return 0;
}

void *qreg_stream(const struct qreg *reg)
{
	const struct p2_qreg *b = B(reg);
	return b ? p2d_stream(b->dev) : NULL;
}
