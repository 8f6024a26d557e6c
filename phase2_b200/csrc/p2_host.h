/*
 * p2_host.h -- host-side internals shared by the C sources of
 * libphase2.so: process settings and the register backend record.
 */
#ifndef P2_HOST_H
#define P2_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "phase2/qreg.h"
#include "phase2_b200.h"

#include "p2_internal.h"

/* Process-wide defaults (phase2_set_*; PHASE2_PRECISION env). */
struct p2_settings {
	int prec;
	int max_span;
	int max_rots;
	int order;
};
extern struct p2_settings p2_cfg;
void p2_settings_from_env(void);

/* reg->backend */
struct p2_qreg {
	struct p2_dev *dev;
	int prec;
	int max_span, max_rots;
	int error; /* sticky: a launch or copy failed */
	struct phase2_rot_in *q;
	size_t qlen, qcap;
	struct phase2_pass *passes;
	struct phase2_rot_rec *recs;
	size_t plan_cap;
};

/* Sticky error of a register (0 ok, -1 failed). */
int p2_qreg_error(const struct qreg *reg);

#endif /* P2_HOST_H */
