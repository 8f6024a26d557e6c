/*
 * p2_host.h -- host-side internals shared by the C sources of
 * libphase2.so: process settings and the register backend record.
 */
#ifndef P2_HOST_H
#define P2_HOST_H

#include <stddef.h>
#include <stdint.h>

#include "phase2/circ.h"
#include "phase2/qreg.h"
#include "phase2_b200.h"

#include "p2_internal.h"

/* Process-wide defaults (phase2_set_*; PHASE2_PRECISION env). */
struct p2_settings {
	int prec;
	int max_span;
	int max_rots;
	int order;
	int fp32_form; /* enum phase2_form used for FP32 registers */
	int batch_persistent; /* batched drivers: one persistent launch */
	int device_sampling; /* qdrift on the GPU: PHASE2_DEVICE_SAMPLING_* */
};
extern struct p2_settings p2_cfg;
void p2_settings_from_env(void);

/* reg->backend */
/*
 * Work on a register is kept in program order with two host queues:
 * rotations (q) and amplitude writes (w*).  At most one of them is
 * non-empty: queuing into one drains the other first.  Reads drain both.
 * Registers of up to P2_HOST_COPY_QB qubits keep a host copy of the state
 * (host_copy) after a read, valid until the next change, so that long runs
 * of single-amplitude reads cost one download.
 */
#define P2_HOST_COPY_QB 16

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
	uint64_t *widx;
	double *wval;
	size_t wlen, wcap;
	double *host_copy;
	int host_copy_valid;
	struct p2_prog *rec; /* recording instead of executing, or NULL */
	/* input of the plan held in passes/recs (a flush whose queue is
	 * byte-identical, with the same settings, reuses it: every Trotter
	 * step after the first) */
	struct phase2_rot_in *plan_q;
	size_t plan_qlen, plan_qcap;
	long plan_np;
	int plan_span, plan_rots, plan_form, plan_sweep;
};

/* Sticky error of a register (0 ok, -1 failed). */
int p2_qreg_error(const struct qreg *reg);

/*
 * Recording (batched persistent execution, drivers.c): between
 * p2_qreg_record and p2_qreg_record_end, zero, writes and rotation flushes
 * of the register are appended to *pg instead of running; reads of the
 * state are errors except p2_qreg_record_gather, which records a gather
 * and returns the output index of its first amplitude (or -1).
 */
int p2_qreg_record(struct qreg *reg, struct p2_prog *pg);
long p2_qreg_record_gather(struct qreg *reg, const uint64_t *idx, size_t n);
int p2_qreg_record_end(struct qreg *reg);
struct p2_dev *p2_qreg_dev(const struct qreg *reg);

/* For work on the device state outside the queues (coefficient-matrix
 * state prep and overlap): drain the queues, drop the host copy, and
 * return the device state (NULL on a register error or while recording).
 * p2_qreg_fail marks the register failed and returns -1. */
struct p2_dev *p2_qreg_direct(struct qreg *reg);
int p2_qreg_fail(struct qreg *reg);

/* sum_d a[d] * conj(cf_d) over the circuit's determinants, the expression
 * of circ_measure (a: the determinant amplitudes in order). */
_Complex double p2_circ_overlap(const struct circ_muldet *md,
	const _Complex double *a);

#endif /* P2_HOST_H */
