/*
 * prog.c -- recorded register programs (p2_internal.h): the ops a register
 * would have executed, kept for one persistent launch over many registers.
 *
 * Flush plans are deduplicated by content: a Trotter step produces the same
 * passes and records every time, so a program of S steps holds one copy of
 * the step's plan and S runs of PASS ops pointing at it.
 */
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "prog"
#include "log.h"

#include "p2_internal.h"

void p2_prog_free(struct p2_prog *pg)
{
	free(pg->ops);
	free(pg->passes);
	free(pg->recs);
	free(pg->widx);
	free(pg->wval);
	free(pg->gidx);
	free(pg->plans);
	memset(pg, 0, sizeof *pg);
}

/* Grow *p (elements of size sz, capacity *cap) to hold `need`. */
static int grow(void **p, size_t *cap, size_t need, size_t sz)
{
	if (need <= *cap)
		return 0;
	size_t c = *cap ? *cap : 64;
	while (c < need)
		c *= 2;
	void *q = realloc(*p, c * sz);
	if (!q)
		return -1;
	*p = q;
	*cap = c;
	return 0;
}

static int push_op(struct p2_prog *pg, uint32_t kind, uint32_t a, uint32_t b)
{
	if (pg->error)
		return -1;
	if (grow((void **)&pg->ops, &pg->ops_cap, pg->nops + 1,
		    sizeof *pg->ops) < 0 ||
		pg->nops >= UINT32_MAX) {
		pg->error = -1;
		return -1;
	}
	struct p2_op *op = &pg->ops[pg->nops++];
	op->kind = kind;
	op->a = a;
	op->b = b;
	op->ntiles = 0;
	return 0;
}

int p2_prog_zero(struct p2_prog *pg)
{
	return push_op(pg, P2_OP_ZERO, 0, 0);
}

int p2_prog_write(struct p2_prog *pg, const uint64_t *idx, const double *val,
	size_t n)
{
	if (pg->error || n == 0)
		return pg->error;
	const size_t at = pg->nw;
	size_t cw = pg->w_cap;
	if (grow((void **)&pg->widx, &pg->w_cap, at + n, sizeof *pg->widx) <
			0 ||
		grow((void **)&pg->wval, &cw, at + n, 2 * sizeof *pg->wval) <
			0 ||
		at + n > UINT32_MAX) {
		pg->error = -1;
		return -1;
	}
	memcpy(pg->widx + at, idx, n * sizeof *idx);
	memcpy(pg->wval + 2 * at, val, 2 * n * sizeof *val);
	pg->nw = at + n;
	return push_op(pg, P2_OP_WRITE, (uint32_t)at, (uint32_t)n);
}

static uint64_t fnv1a(uint64_t h, const void *p, size_t n)
{
	const unsigned char *c = p;
	for (size_t i = 0; i < n; i++) {
		h ^= c[i];
		h *= UINT64_C(0x100000001b3);
	}
	return h;
}

static int same_plan(const struct p2_prog *pg, const struct p2_plan_ref *r,
	const struct phase2_pass *passes, size_t npass,
	const struct phase2_rot_rec *recs, size_t nrec)
{
	if (r->npass != npass || r->nrec != nrec)
		return 0;
	for (size_t i = 0; i < npass; i++) {
		struct phase2_pass a = pg->passes[r->pass_off + i];
		a.rot_off -= r->rec_off;
		if (memcmp(&a, &passes[i], sizeof a) != 0)
			return 0;
	}
	return memcmp(pg->recs + r->rec_off, recs, nrec * sizeof *recs) == 0;
}

int p2_prog_plan(struct p2_prog *pg, const struct phase2_pass *passes,
	size_t npass, const struct phase2_rot_rec *recs, size_t nrec,
	int same_as_last)
{
	if (pg->error || npass == 0)
		return pg->error;
	const struct p2_plan_ref *hit = NULL;
	if (same_as_last && pg->last_plan >= 0 && pg->nplans > 0 &&
		pg->plans[pg->last_plan].npass == npass &&
		pg->plans[pg->last_plan].nrec == nrec)
		hit = &pg->plans[pg->last_plan];
	uint64_t h = 0;
	if (!hit) {
		h = fnv1a(UINT64_C(0xcbf29ce484222325), passes,
			npass * sizeof *passes);
		h = fnv1a(h, recs, nrec * sizeof *recs);
	}
	for (size_t k = 0; k < pg->nplans && !hit; k++)
		if (pg->plans[k].hash == h &&
			same_plan(pg, &pg->plans[k], passes, npass, recs, nrec))
			hit = &pg->plans[k];
	if (!hit) {
		if (grow((void **)&pg->passes, &pg->pass_cap, pg->npass + npass,
			    sizeof *pg->passes) < 0 ||
			grow((void **)&pg->recs, &pg->rec_cap, pg->nrec + nrec,
				sizeof *pg->recs) < 0 ||
			grow((void **)&pg->plans, &pg->plans_cap,
				pg->nplans + 1, sizeof *pg->plans) < 0 ||
			pg->nrec + nrec > UINT32_MAX ||
			pg->npass + npass > UINT32_MAX) {
			pg->error = -1;
			return -1;
		}
		struct p2_plan_ref *r = &pg->plans[pg->nplans++];
		r->hash = h;
		r->pass_off = (uint32_t)pg->npass;
		r->npass = (uint32_t)npass;
		r->rec_off = (uint32_t)pg->nrec;
		r->nrec = (uint32_t)nrec;
		memcpy(pg->recs + pg->nrec, recs, nrec * sizeof *recs);
		for (size_t i = 0; i < npass; i++) {
			pg->passes[pg->npass + i] = passes[i];
			pg->passes[pg->npass + i].rot_off += r->rec_off;
		}
		pg->npass += npass;
		pg->nrec += nrec;
		hit = r;
	}
	pg->last_plan = hit - pg->plans;
	for (size_t i = 0; i < npass; i++) {
		if (push_op(pg, P2_OP_PASS, hit->pass_off + (uint32_t)i, 0) < 0)
			return -1;
		pg->rotations += passes[i].nrot;
	}
	return 0;
}

long p2_prog_gather(struct p2_prog *pg, const uint64_t *idx, size_t n)
{
	if (pg->error)
		return -1;
	const size_t at = pg->ng;
	if (grow((void **)&pg->gidx, &pg->g_cap, at + n, sizeof *pg->gidx) <
			0 ||
		at + n > UINT32_MAX) {
		pg->error = -1;
		return -1;
	}
	if (n)
		memcpy(pg->gidx + at, idx, n * sizeof *idx);
	pg->ng = at + n;
	if (push_op(pg, P2_OP_GATHER, (uint32_t)at, (uint32_t)n) < 0)
		return -1;
	return (long)at;
}
