/*
 * p2_engine.h -- internals shared by the CUDA sources of the engine:
 * engine.cu (registers, pass kernels, state I/O, reductions), batch.cu
 * (the persistent kernel), sampling.cu (device sampling) and sweep.cu
 * (sweeps).  Include after log.h.
 */
#ifndef P2_ENGINE_H
#define P2_ENGINE_H

#include <cuda_runtime.h>
#include <stdint.h>

#include "phase2_b200.h"

#include "p2_internal.h"

#define P2_TPB 128
#define P2_RED_TPB 256

/* Replay of repeated flushes: registers up to this width keep a small LRU
 * of captured pass sequences (launch overhead matters only there). */
#define P2_GRAPH_SLOTS 8
#define P2_GRAPH_MAX_QB 24

struct p2_graph {
	uint64_t hash;
	size_t npass, nrec;
	struct phase2_pass *passes;    /* host copies: exact comparison */
	struct phase2_rot_rec *recs;
	struct phase2_rot_rec *d_recs; /* records read by the graph */
	cudaGraphExec_t exec;
	size_t nlaunch; /* kernel launches in the graph */
	int status;     /* the graph holds kernels that write d_status */
	uint64_t used;
};

struct p2_dev {
	uint32_t nqb;
	int prec;
	size_t elem;
	uint64_t namp;
	void *state;
	cudaStream_t stream;
	int sm_count;

	struct phase2_rot_rec *d_recs;
	size_t d_recs_cap;
	struct phase2_rot_rec *h_recs[2];
	size_t h_recs_cap[2];
	cudaEvent_t h_ev[2];
	int h_ev_live[2];
	int ring;

	/* error word of kernels with bounded waits (lift_bulk.cu): set on
	 * the device, read at the next synchronisation (p2_status_check) */
	unsigned int *d_status;
	unsigned int *h_status;
	int status_pending;

	uint64_t *d_idx;
	double *d_val;
	uint64_t *h_idx;
	double *h_val;
	size_t io_cap;

	double *d_part;
	size_t part_cap;

	unsigned char *d_cm; /* coefficient-matrix tables */
	size_t cm_cap;

	int timing;
	cudaEvent_t t0, t1;

	uint64_t rotations, passes, launches, timed_passes;
	uint64_t sweeps, timed_sweeps; /* state round trips (pass or sweep
					* kernels) */
	uint64_t h2d_bytes, d2h_bytes;
	double pass_ms;

	struct p2_graph graphs[P2_GRAPH_SLOTS];
	uint64_t graph_clock;
	uint64_t graph_replays;
	int graphs_on;
};

#define CUDA_OK(call, what)                                                    \
	do {                                                                   \
		cudaError_t e_ = (call);                                       \
		if (e_ != cudaSuccess) {                                       \
			log_error("%s: %s", (what), cudaGetErrorString(e_));  \
			return -1;                                             \
		}                                                              \
	} while (0)


static inline unsigned grid_for(const struct p2_dev *d, uint64_t work, unsigned tpb,
	unsigned per_sm)
{
	uint64_t b = (work + tpb - 1) / tpb;
	const uint64_t cap = (uint64_t)d->sm_count * per_sm;
	if (b > cap)
		b = cap;
	return b ? (unsigned)b : 1u;
}

/* ---- cross-file entry points -------------------------------------------- */

/* engine.cu: transient device buffers of one call (a batch program, the
 * scratch of device sampling), stream-ordered from the device's default
 * memory pool, which keeps up to 1 GiB of freed memory for the next call
 * instead of unmapping it at every synchronisation (a cudaFree of such a
 * buffer could take hundreds of milliseconds).  The pool is configured on
 * the first call, for the current device (one device per process). */
cudaError_t p2_scratch_alloc(void **p, size_t bytes, cudaStream_t stream);
void p2_scratch_free(void *p, cudaStream_t stream);

struct p2_binst;
struct p2_bctl;

/* Idle scheduling rounds (each sleeps ~1 us, and counting restarts
 * whenever any ticket moves) before a block of the persistent kernel gives
 * up. */
#define P2_BATCH_IDLE_LIMIT 2000000u

/* batch.cu: the persistent kernel for FP32 registers (FP32 arithmetic,
 * P2_BK_F32, or FP64 arithmetic, P2_BK_F32X) or FP64 registers
 * (P2_BK_F64): the instance for a precision and FP32 form, its function
 * (occupancy queries) and its launch.  status points to 16
 * zeroed bytes: status[0] is raised when a wait gives up, status[2..3]
 * receive the complement of the launch's start time (global timer).  cum
 * (device, one double per program, or NULL for round robin): running
 * totals of the programs' work, which spread the warps' home programs. */
enum { P2_BK_F32 = 0, P2_BK_F32X = 1, P2_BK_F64 = 2 };
int p2_batch_kind(int prec, int form);
const void *p2_batch_kernel(int kind);
void p2_batch_launch(int kind, unsigned grid, cudaStream_t stream,
	const struct p2_binst *inst, uint32_t ninst, const struct p2_op *ops,
	const struct phase2_pass *passes, const struct phase2_rot_rec *recs,
	const uint64_t *widx, const double *wval, const uint64_t *gidx,
	double2 *gout, struct p2_bctl *ctl, unsigned int *status,
	const double *cum);

/* lift_bulk.cu: one FP32 pass of the FP64-arithmetic form on a kernel
 * whose next cosets are staged in shared memory, by bulk copies (variant
 * 1) or cp.async (variant 2); returns 1 when launched, 0 when the pass
 * does not qualify (the caller runs the direct kernel), -1 on error.
 * per_sm_cap: resident blocks per SM at most (0: occupancy). */
extern "C" int p2_lift_staged_launch(struct p2_dev *d,
	const struct phase2_pass *p, const struct phase2_rot_rec *recs,
	int variant, unsigned per_sm_cap);

/* engine.cu: read the error word of kernels with bounded waits if one ran
 * since the last check (synchronises the register's stream); -1 and a
 * logged error when a wait gave up. */
int p2_status_check(struct p2_dev *d);

/* slab.cu: 0 if [p, p + bytes) is device memory of the current device
 * inside one allocation; -1 (logged, prefixed by `what`) otherwise, also
 * when the allocation cannot be looked up.  Allocates nothing. */
int p2_check_device_range(const void *p, size_t bytes, const char *what);

/* sweep.cu: whether planned sweeps run as one kernel each on this
 * register, and the launch of the sweep starting at passes[i] (returns the
 * passes it covers, 1 when passes[i] should run alone, -1 on error). */
bool p2_sweeps_on(const struct p2_dev *d);
long p2_sweep_launch(struct p2_dev *d, const struct phase2_pass *passes,
	size_t npass, size_t i, const struct phase2_rot_rec *d_recs);

#endif /* P2_ENGINE_H */
