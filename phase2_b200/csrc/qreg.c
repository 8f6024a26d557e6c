/*
 * qreg.c -- the register API (include/phase2/qreg.h) over the device
 * engine.  Replaces phase2/qreg.c + phase2/qreg_cuda.c of
 * Quantum-for-Life/phase2 for one rank.
 *
 * The reference applies a batch with a partner exchange, a projector split
 * into two buffers, two rotation launches per term and a recombination
 * (phase2/qreg_cuda_lo.cu:111-131).  With one rank the exchange is a self
 * copy and the second buffer is identically zero, so all of that reduces
 * to applying the rotations in order to the one state.
 *
 * Execution model: rotations and amplitude writes are queued on the host
 * in program order and executed in batches -- rotations as planned passes
 * (plan.c), writes as one scatter launch.  Every call that observes the
 * state (getamp, sync, norms, stats) drains the queues first, so callers
 * see exactly the state the reference would hold at that point.  Small
 * registers keep a host copy after a read so that runs of single-amplitude
 * reads (the reference's tests read whole states one amplitude at a time)
 * cost one download.
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
	if (nqb <= P2_HOST_COPY_QB) {
		b->host_copy = calloc(2 * reg->namp, sizeof(double));
		if (!b->host_copy) {
			qreg_free(reg);
			return -1;
		}
	}
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
		free(b->plan_q);
		free(b->widx);
		free(b->wval);
		free(b->host_copy);
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

/* Reads of the state are not possible while the register records. */
static int recording(const struct p2_qreg *b, const char *what)
{
	if (!b->rec)
		return 0;
	log_error("%s: register is recording a batch program", what);
	return 1;
}

/* Launch the queued amplitude writes (one scatter, later writes win). */
static int drain_writes(struct p2_qreg *b)
{
	if (b->wlen == 0)
		return b->error;
	if (b->rec) {
		if (p2_prog_write(b->rec, b->widx, b->wval, b->wlen) < 0)
			b->error = -1;
		b->wlen = 0;
		return b->error;
	}
	if (p2d_set(b->dev, b->widx, b->wval, b->wlen) < 0) {
		log_error("qreg: %zu amplitude writes failed", b->wlen);
		b->error = -1;
	}
	b->wlen = 0;
	return b->error;
}

/* Keep a copy of the queue just planned (the plan cache's key). */
static void remember_plan(struct p2_qreg *b, long np, int form, int sweep)
{
	b->plan_qlen = 0;
	if (np < 0)
		return;
	if (b->plan_qcap < b->qlen) {
		free(b->plan_q);
		b->plan_q = malloc(sizeof *b->plan_q * b->qlen);
		b->plan_qcap = b->plan_q ? b->qlen : 0;
		if (!b->plan_q)
			return;
	}
	memcpy(b->plan_q, b->q, sizeof *b->q * b->qlen);
	b->plan_qlen = b->qlen;
	b->plan_np = np;
	b->plan_span = b->max_span;
	b->plan_rots = b->max_rots;
	b->plan_form = form;
	b->plan_sweep = sweep;
}

/* Plan and launch the queued rotations (asynchronously). */
static int drain_rotations(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
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
		b->plan_qlen = 0; /* the held plan is gone */
	}
	const int form = p2_form_for(b->prec);
	int swk, swl;
	p2_sweep_for(reg->qb_lo, form, &swk, &swl);
	const int sweep = swk << 8 | swl;
	/* the same queue under the same settings plans to the same passes:
	 * reuse the plan still held in passes/recs */
	const int same = b->plan_q && b->plan_qlen == b->qlen &&
		b->plan_span == b->max_span && b->plan_rots == b->max_rots &&
		b->plan_form == form && b->plan_sweep == sweep &&
		memcmp(b->plan_q, b->q, sizeof *b->q * b->qlen) == 0;
	long np = b->plan_np;
	if (!same) {
		np = p2_plan(reg->qb_lo, b->q, b->qlen, b->max_span,
			b->max_rots, P2_DEFAULT_PAD_SPAN, form, swk, swl,
			b->passes, b->recs);
		remember_plan(b, np, form, sweep);
	}
	if (np >= 0 && b->rec) {
		if (p2_prog_plan(b->rec, b->passes, (size_t)np, b->recs,
			    b->qlen, same) < 0)
			b->error = -1;
	} else if (np < 0 || p2d_run(b->dev, b->passes, (size_t)np, b->recs,
				    b->qlen) < 0) {
		log_error("qreg: %zu rotations failed", b->qlen);
		b->error = -1;
	}
	b->qlen = 0;
	return b->error;
}

int qreg_flush(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (!b)
		return -1;
	/* at most one queue is non-empty; order does not matter here */
	drain_writes(b);
	drain_rotations(reg);
	return b->error;
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

int qreg_synchronize(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (!b || qreg_flush(reg) < 0)
		return -1;
	if (!b->rec && p2d_sync(b->dev) < 0)
		b->error = -1;
	return b->error;
}

void qreg_paulirot(struct qreg *reg, struct paulis code_hi,
	const struct paulis *codes_lo, const double *phis, size_t ncodes)
{
	struct p2_qreg *b = B(reg);
	if (!b || ncodes == 0)
		return;
	if (drain_writes(b) < 0)
		return;
	b->host_copy_valid = 0;
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
			drain_rotations(reg);
	}
}

int qreg_setamps(struct qreg *reg, const uint64_t *idx,
	const _Complex double *z, size_t n)
{
	struct p2_qreg *b = B(reg);
	if (!b)
		return -1;
	for (size_t i = 0; i < n; i++)
		if (idx[i] >= reg->namp) {
			log_error("qreg_setamps: index %llu out of range",
				(unsigned long long)idx[i]);
			return -1;
		}
	if (drain_rotations(reg) < 0)
		return -1;
	if (b->wlen + n > b->wcap) {
		size_t cap = b->wcap ? b->wcap : 256;
		while (cap < b->wlen + n)
			cap *= 2;
		uint64_t *wi = realloc(b->widx, sizeof *wi * cap);
		if (wi)
			b->widx = wi;
		double *wv = realloc(b->wval, sizeof *wv * 2 * cap);
		if (wv)
			b->wval = wv;
		if (!wi || !wv) {
			b->error = -1;
			return -1;
		}
		b->wcap = cap;
	}
	memcpy(b->widx + b->wlen, idx, sizeof *idx * n);
	memcpy(b->wval + 2 * b->wlen, z, sizeof(double) * 2 * n);
	b->wlen += n;
	b->host_copy_valid = 0;
	return 0;
}

int qreg_getamps(struct qreg *reg, const uint64_t *idx, _Complex double *z,
	size_t n)
{
	struct p2_qreg *b = B(reg);
	if (!b || recording(b, "qreg_getamps"))
		return -1;
	for (size_t i = 0; i < n; i++)
		if (idx[i] >= reg->namp) {
			log_error("qreg_getamps: index %llu out of range",
				(unsigned long long)idx[i]);
			return -1;
		}
	if (qreg_flush(reg) < 0)
		return -1;
	double *out = (double *)z; /* _Complex double = (re, im) */
	if (b->host_copy) {
		if (!b->host_copy_valid) {
			if (p2d_get_state(b->dev, b->host_copy) < 0) {
				b->error = -1;
				return -1;
			}
			b->host_copy_valid = 1;
		}
		for (size_t i = 0; i < n; i++) {
			out[2 * i] = b->host_copy[2 * idx[i]];
			out[2 * i + 1] = b->host_copy[2 * idx[i] + 1];
		}
		return 0;
	}
	if (p2d_get(b->dev, idx, out, n) < 0) {
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
	/* queued work acts on a state about to be overwritten */
	b->qlen = 0;
	b->wlen = 0;
	if (b->rec) {
		if (p2_prog_zero(b->rec) < 0)
			b->error = -1;
		return;
	}
	if (p2d_zero(b->dev) < 0) {
		b->error = -1;
		b->host_copy_valid = 0;
		return;
	}
	if (b->host_copy) {
		memset(b->host_copy, 0, sizeof(double) * 2 * reg->namp);
		b->host_copy_valid = 1;
	}
}

int qreg_get_state(struct qreg *reg, double *out)
{
	struct p2_qreg *b = B(reg);
	if (!b || recording(b, "qreg_get_state") || qreg_flush(reg) < 0)
		return -1;
	if (b->host_copy && b->host_copy_valid) {
		memcpy(out, b->host_copy, sizeof(double) * 2 * reg->namp);
		return 0;
	}
	return p2d_get_state(b->dev, out);
}

int qreg_set_state(struct qreg *reg, const double *in)
{
	struct p2_qreg *b = B(reg);
	if (!b || recording(b, "qreg_set_state"))
		return -1;
	b->qlen = 0;
	b->wlen = 0;
	b->host_copy_valid = 0;
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
	if (!b || recording(b, "qreg_norm2") || qreg_flush(reg) < 0)
		return -1;
	return p2d_norm2(b->dev, out);
}

int qreg_inner_dense(struct qreg *reg, const double *trial, double out[2])
{
	struct p2_qreg *b = B(reg);
	if (!b || recording(b, "qreg_inner_dense") || qreg_flush(reg) < 0)
		return -1;
	return p2d_inner_dense(b->dev, trial, out);
}

static int slab_copy(struct qreg *reg, uint32_t bit, uint32_t val,
	uint64_t first, uint64_t count, void *buf, int put)
{
	struct p2_qreg *b = B(reg);
	if (!b || recording(b, put ? "qreg_slab_put" : "qreg_slab_get") ||
		qreg_flush(reg) < 0)
		return -1;
	if (put)
		b->host_copy_valid = 0;
	return p2d_slab_copy(b->dev, bit, val, first, count, buf, put);
}

int qreg_slab_get(struct qreg *reg, uint32_t bit, uint32_t val,
	uint64_t first, uint64_t count, void *d_buf)
{
	return slab_copy(reg, bit, val, first, count, d_buf, 0);
}

int qreg_slab_put(struct qreg *reg, uint32_t bit, uint32_t val,
	uint64_t first, uint64_t count, const void *d_buf)
{
	return slab_copy(reg, bit, val, first, count, (void *)d_buf, 1);
}

int qreg_slab_swap(struct qreg *a, struct qreg *b, uint32_t bit,
	uint32_t val_a, uint32_t val_b)
{
	struct p2_qreg *ba = B(a), *bb = B(b);
	if (!ba || !bb || recording(ba, "qreg_slab_swap") ||
		recording(bb, "qreg_slab_swap") || qreg_flush(a) < 0 ||
		qreg_flush(b) < 0)
		return -1;
	ba->host_copy_valid = 0;
	bb->host_copy_valid = 0;
	return p2d_slab_swap(ba->dev, bb->dev, bit, val_a, val_b);
}

int p2_qreg_record(struct qreg *reg, struct p2_prog *pg)
{
	struct p2_qreg *b = B(reg);
	if (!b || b->rec || qreg_flush(reg) < 0)
		return -1;
	b->rec = pg;
	b->host_copy_valid = 0;
	return 0;
}

long p2_qreg_record_gather(struct qreg *reg, const uint64_t *idx, size_t n)
{
	struct p2_qreg *b = B(reg);
	if (!b || !b->rec || qreg_flush(reg) < 0)
		return -1;
	for (size_t i = 0; i < n; i++)
		if (idx[i] >= reg->namp) {
			log_error("gather: index %llu out of range",
				(unsigned long long)idx[i]);
			return -1;
		}
	const long at = p2_prog_gather(b->rec, idx, n);
	if (at < 0)
		b->error = -1;
	return at;
}

int p2_qreg_record_end(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (!b || !b->rec)
		return -1;
	qreg_flush(reg);
	if (b->rec->error)
		b->error = -1;
	b->rec = NULL;
	return b->error;
}

struct p2_dev *p2_qreg_dev(const struct qreg *reg)
{
	const struct p2_qreg *b = B(reg);
	return b ? b->dev : NULL;
}

struct p2_dev *p2_qreg_direct(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (!b || recording(b, "coefficient-matrix state") ||
		qreg_flush(reg) < 0)
		return NULL;
	b->host_copy_valid = 0;
	return b->dev;
}

int p2_qreg_fail(struct qreg *reg)
{
	struct p2_qreg *b = B(reg);
	if (b)
		b->error = -1;
	return -1;
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
