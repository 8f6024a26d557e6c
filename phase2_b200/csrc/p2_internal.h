/*
 * p2_internal.h -- interfaces private to libphase2.so: the planner and the
 * device engine (engine.cu).  Plain C types only; engine.cu implements the
 * p2d_* functions with extern "C" linkage.
 */
#ifndef P2_INTERNAL_H
#define P2_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#include "phase2_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Rotation records held in shared memory per pass. */
#define P2_MAX_ROTS_PER_PASS 256
/* Passes are padded to at least this many basis vectors (2^3 amplitudes
 * per thread) to keep enough loads in flight. */
#define P2_DEFAULT_PAD_SPAN 3
/* Queued rotations that trigger an automatic flush. */
#define P2_QUEUE_FLUSH 8192

/* form: enum phase2_form of every pass (and the records it implies);
 * sweep_k, sweep_low: sweep grouping (p2_sweep_for; 0, 0 for none). */
long p2_plan(uint32_t nqb, const struct phase2_rot_in *rots, size_t n,
	int max_span, int max_rots, int pad_span, int form, int sweep_k,
	int sweep_low, struct phase2_pass *passes,
	struct phase2_rot_rec *recs);

/* Sweep grouping the executor uses for a register of nqb qubits whose
 * passes have form `form`: *k = tile - low qubits and *low under the
 * process's sweep shape for FP32-arithmetic registers of tile + 3 to 31
 * qubits, else 0 and 0. */
void p2_sweep_for(uint32_t nqb, int form, int *k, int *low);

/* Pass form for a state precision: exact for FP64, the process's FP32
 * form (phase2_set_fp32_form) for FP32. */
int p2_form_for(int prec);

/* ---- device engine ------------------------------------------------------ */

struct p2_dev;

/* Select and initialise CUDA device `dev`; 0 or -1.  Sets *count to the
 * number of visible devices when non-NULL. */
int p2d_device_init(int dev, int *count);

/* Name of the current CUDA device (as cudaDeviceProp.name); 0 or -1. */
int p2d_device_name(char *buf, size_t n);

/* tuning.c: apply the launch table shipped beside the library (or named
 * by PHASE2_TUNING; "off" skips it) when its GPU name matches. */
void p2_tuning_at_init(void);

/* Register state of 2^nqb amplitudes at precision prec (enum phase2_prec),
 * with its own non-blocking stream.  NULL on failure (logged). */
struct p2_dev *p2d_create(uint32_t nqb, int prec);
void p2d_destroy(struct p2_dev *d);

int p2d_zero(struct p2_dev *d);
int p2d_set(struct p2_dev *d, const uint64_t *idx, const double *z, size_t n);
int p2d_get(struct p2_dev *d, const uint64_t *idx, double *z, size_t n);
int p2d_get_state(struct p2_dev *d, double *out);
int p2d_set_state(struct p2_dev *d, const double *in);

/* Upload `nrec` records and launch `npass` passes on the stream. */
int p2d_run(struct p2_dev *d, const struct phase2_pass *passes, size_t npass,
	const struct phase2_rot_rec *recs, size_t nrec);

int p2d_norm2(struct p2_dev *d, double *out);
int p2d_inner_dense(struct p2_dev *d, const double *trial, double out[2]);

/* Copy elements [first, first + count) of the half {i : bit `bit` of i ==
 * val} of the state to (put = 0) or from (put = 1) the device buffer buf,
 * which holds them contiguously at the register's precision; waits for the
 * copy.  0 or -1 (logged). */
int p2d_slab_copy(struct p2_dev *d, uint32_t bit, uint32_t val,
	uint64_t first, uint64_t count, void *buf, int put);

/* Exchange half (bit, va) of a with half (bit, vb) of b in place (two
 * registers of one size and precision on one device); waits for it. */
int p2d_slab_swap(struct p2_dev *a, struct p2_dev *b, uint32_t bit,
	uint32_t va, uint32_t vb);

/* Wait for the stream; -1 if any CUDA error is pending. */
int p2d_sync(struct p2_dev *d);

/* Device memory on the current device (cudaMalloc / cudaFree). */
void *p2d_buffer_alloc(size_t bytes);
void p2d_buffer_free(void *p);

void p2d_stats(const struct p2_dev *d, struct phase2_stats *st);
void p2d_stats_reset(struct p2_dev *d);
void p2d_set_timing(struct p2_dev *d, int on);
void *p2d_stream(const struct p2_dev *d);

/*
 * Coefficient-matrix trial states (state_prep.c).  occ_a (Ma) and occ_b
 * (Mb) are the alpha and beta occupation masks (beta already shifted by
 * n_sites); det_a/det_b hold ncomp blocks of Ma/Mb determinants.
 * expand: for every (i, j), the unpruned w_k det_a_k[i] det_b_k[j] are
 * added in block order to the amplitude (accumulate) or to a first
 * assignment (not accumulate); inner: out = sum of w da db * amplitude.
 */
int p2d_cm_expand(struct p2_dev *d, uint32_t n_sites, int tapered,
	int accumulate, const uint64_t *occ_a, size_t Ma, const uint64_t *occ_b,
	size_t Mb, const double *w, const double *det_a, const double *det_b,
	size_t ncomp);
int p2d_cm_inner(struct p2_dev *d, uint32_t n_sites, int tapered,
	const uint64_t *occ_a, size_t Ma, const uint64_t *occ_b, size_t Mb,
	double w, const double *det_a, const double *det_b, double out[2]);

/* ---- recorded programs (batched persistent execution) ------------------- */

/*
 * A register can record, instead of execute, what would run on it: a list
 * of ops over its state.  Many registers' programs then run together in one
 * persistent launch (p2d_batch_run).
 */
enum p2_op_kind {
	P2_OP_ZERO = 0,   /* state <- 0 */
	P2_OP_WRITE = 1,  /* writes a .. a+b-1 of widx/wval, in order */
	P2_OP_PASS = 2,   /* pass a of passes (b: cosets per thread a tile,
			   * set by p2d_batch_run) */
	P2_OP_GATHER = 3, /* amplitudes gidx[a .. a+b-1] -> output a .. a+b-1 */
};

struct p2_op {
	uint32_t kind;
	uint32_t a, b;
	uint32_t ntiles; /* work tiles of the op (set by p2d_batch_run) */
};

/* A distinct flush plan of a program: later identical flushes reuse it. */
struct p2_plan_ref {
	uint64_t hash;
	uint32_t pass_off, npass, rec_off, nrec;
};

struct p2_prog {
	struct p2_op *ops;
	size_t nops, ops_cap;
	struct phase2_pass *passes; /* rot_off relative to recs */
	size_t npass, pass_cap;
	struct phase2_rot_rec *recs;
	size_t nrec, rec_cap;
	uint64_t *widx;
	double *wval; /* (re, im) per write */
	size_t nw, w_cap;
	uint64_t *gidx;
	size_t ng, g_cap;
	struct p2_plan_ref *plans;
	size_t nplans, plans_cap;
	uint64_t rotations; /* rotations in the PASS ops */
	long last_plan;     /* plans[] index of the last p2_prog_plan (valid
			     * when nplans > 0) */
	int error;
};

void p2_prog_free(struct p2_prog *pg);
int p2_prog_zero(struct p2_prog *pg);
int p2_prog_write(struct p2_prog *pg, const uint64_t *idx, const double *val,
	size_t n);
/* Append a flush plan's passes (records rot_off-relative to recs);
 * same_as_last: the caller knows it equals the previous call's plan. */
int p2_prog_plan(struct p2_prog *pg, const struct phase2_pass *passes,
	size_t npass, const struct phase2_rot_rec *recs, size_t nrec,
	int same_as_last);
/* Gather n amplitudes; returns the output index of the first, or -1. */
long p2_prog_gather(struct p2_prog *pg, const uint64_t *idx, size_t n);

/* Whether a register's programs can run in p2d_batch_run (FP32 state in
 * the FP32-arithmetic lifted form, at most 31 qubits). */
int p2d_batch_ok(const struct p2_dev *d);

/* Sweep shape of the FP32 pass executor (phase2_set_sweep). */
int p2d_set_sweep(int tile_qubits, int low_qubits);
void p2d_get_sweep(int *tile_qubits, int *low_qubits);
void p2d_set_sweep_kernel(int on);

/* Run n recorded programs, program i on register devs[i], in one
 * persistent launch; gout receives every program's gathered amplitudes
 * (FP64 re, im) in program order.  *kernel_ms (if non-NULL) gets the
 * launch's device time.  0 or -1. */
/* batch.cu: per-instance finish times of the last persistent launch
 * (phase2_batch_finish_ms): cleared at the start of a batched driver call,
 * and re-indexed from launched programs to instances (who[j] = instance
 * of program j; instances not launched get -1). */
void p2_batch_finish_reset(void);
int p2_batch_finish_map(const size_t *who, size_t m, size_t n);

int p2d_batch_run(struct p2_dev *const *devs,
	const struct p2_prog *const *progs, size_t n, double *gout,
	double *kernel_ms);

/* ---- device sampling (qdrift / cmpsit simul on the GPU) --------------- */

/*
 * A sampled run executed on the device.  Sample s's rotation stream is
 * `halves` halves; a forward half applies the head terms 0..length-1 (a
 * fixed table with its own angles) and then `depth` drawn terms, a
 * reversed half (odd halves when reverse_odd) the drawn terms in reverse
 * then the head in reverse.  Half h of sample s draws from generator state
 * rng0[s * halves + h] (xoshiro256** top 53 bits; the term is the smallest
 * i with y[i] > x, its sign with the DBL_EPSILON dead zone picks rphi/rcs).
 * The stream is planned exactly as host flushes of P2_QUEUE_FLUSH
 * rotations would plan it (plan_core.h), and the program zero / write
 * dets / passes / gather dets of every sample runs in one persistent
 * launch per round of samples.  Samples are independent (each starts from
 * the trial state), so small registers run up to P2_QD_MAX_REGS samples at
 * once on copies of the state; the last sample always runs on the register
 * itself, which ends holding its state as after the host loop.
 *   qdrift: halves 1, length 0, rphi = asin(step) * {-1, 0, 1}.
 *   cmpsit: halves 2 * steps, reverse_odd, head = the deterministic terms
 *           at 0.5 * (c * angle_det), rphi = 0.5 * ({-1, 0, 1} * tau).
 */
#define P2_QD_MAX_REGS 256

struct p2_smp_job {
	uint32_t nqb, ndet;
	uint64_t nterms, mask;
	uint32_t depth, length, halves, reverse_odd;
	double rphi[3];   /* angle of a drawn term, sign -1, 0, +1 */
	double rcs[3][2]; /* its cos, sin */
	int max_span, max_rots, form;
	int sweep_k, sweep_low; /* sweep grouping, as p2_sweep_for */
};

/* gout gets ndet amplitudes (re, im) per sample, in sample order;
 * *npass_out: passes executed.  0 or -1. */
int p2d_sampled_device(struct p2_dev *d, const struct p2_smp_job *job,
	const uint64_t *rng0, size_t samples, const double *cdf_y,
	const uint64_t *tflip, const uint64_t *tphase, const double *tcf,
	const uint64_t *hflip, const uint64_t *hphase, const double *hphi,
	const double *hcs, const uint64_t *det_idx, const double *det_val,
	double *gout, uint64_t *npass_out);

#ifdef __cplusplus
}
#endif

#endif /* P2_INTERNAL_H */
