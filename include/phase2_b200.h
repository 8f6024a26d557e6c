#ifndef PHASE2_B200_H
#define PHASE2_B200_H

/*
 * Extensions of this B200 library beyond the phase2 C surface.  None of
 * these has a counterpart in Quantum-for-Life/phase2; code written against
 * the reference headers never needs them.  They select the state precision,
 * the fusion policy and the term order, expose bulk state access, device
 * reductions and counters, and the planner used by qreg_paulirot.
 */

#include <stddef.h>
#include <stdint.h>

#include "phase2/circ.h"
#include "phase2/qreg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- precision ---------------------------------------------------------- */

/* FP64: complex128 state, rotations bit-identical to the reference CPU
 * path.  FP32: complex64 state (half the HBM bytes per sweep); angles and
 * cos/sin are computed in FP64, norms and overlaps are FP64 reductions, and
 * the rotation arithmetic follows the FP32 form (phase2_set_fp32_form). */
enum phase2_prec {
	PHASE2_PREC_FP64 = 0,
	PHASE2_PREC_FP32 = 1,
};

/* Process default used by qreg_init (hence circ_init and the drivers).
 * Initial value: FP64, or the PHASE2_PRECISION environment variable
 * ("fp32"/"fp64") read at world_init.  Returns 0 or -1. */
int phase2_set_precision(int prec);
int phase2_get_precision(void);

/* Arithmetic of FP32 passes (enum phase2_form below), all rotating each
 * amplitude pair by three in-place shears:
 *   PHASE2_FORM_LIFTED            coefficients from FP64 cos/sin, FP64
 *                                 arithmetic, one rounding to FP32 per pass;
 *   PHASE2_FORM_LIFTED_F32        FP32 FMAs on coefficients rounded to FP32
 *                                 (faster; one rounding per shear);
 *   PHASE2_FORM_LIFTED_MIXED      (default) per coset of a pass: FP32
 *                                 arithmetic as LIFTED_F32, except cosets
 *                                 holding an amplitude of magnitude
 *                                 >= 2^-10 (re or im) when the pass starts,
 *                                 which take FP64 arithmetic and one
 *                                 rounding per pass.
 * An FP32 shear absorbs increments below half an ulp of the amplitude it
 * updates, so LIFTED_F32 loses the small updates of large amplitudes; the
 * mixed form keeps FP64 arithmetic for those.  Registers of fewer than 24
 * qubits (whose spread states have many such amplitudes), the persistent
 * batch kernel and device sampling run mixed-form programs with FP64
 * arithmetic on every coset; sweeps are off in this form.
 * Also PHASE2_FP32_FORM=lifted|lifted_f32|mixed at world_init.  Applies to
 * rotations planned afterwards.  0 or -1. */
int phase2_set_fp32_form(int form);
int phase2_get_fp32_form(void);

/* qreg_init at an explicit precision. */
int qreg_init_prec(struct qreg *reg, uint32_t nqb, int prec);
int qreg_precision(const struct qreg *reg);

/* ---- fusion policy ------------------------------------------------------ */

/* A pass streams the state once and applies a run of consecutive rotations
 * whose flip masks span a space of dimension <= max_span (each thread owns
 * whole cosets of that space in registers).  max_span in [1,5];
 * max_rots caps rotations per pass (1 = one rotation per pass, the unfused
 * "plain" path; 0 = no cap beyond the per-pass limit).  Defaults 5 and 0.
 * The process default applies to registers created afterwards. */
int phase2_set_fusion(int max_span, int max_rots);
int qreg_set_fusion(struct qreg *reg, int max_span, int max_rots);

/* Launch choice of the pass kernel for one precision and span M (0..5).
 * FP64: variant 0 loads each thread's cosets straight into registers,
 * variant 1 prefetches the next coset into shared memory with cp.async
 * while the current one is computed.  FP32 (FP64-arithmetic form only;
 * the FP32-arithmetic form has one kernel): variant 0 loads directly,
 * variant 1 stages each warp's next cosets in shared memory with bulk
 * copies (cp.async.bulk), variant 2 with cp.async, variant 3 as 2 in a
 * build for two blocks per SM (more registers a thread); passes that do not
 * qualify for staging (a pivot below qubit 5, registers of fewer than
 * M + 5 qubits or more than 31) load directly.  per_sm caps resident
 * blocks per SM in the grid (0 = default).  Process-wide; the autotuner
 * (phase2_b200/autotune.py) sets these from its measurements.  0 or
 * -1. */
int phase2_tune_set(int prec, int span, int variant, int per_sm);
int phase2_tune_get(int prec, int span, int *variant, int *per_sm);

/* Apply a launch table file (lines "gpu <name>" and "launch <prec> <span>
 * <variant> <per_sm>", '#' comments; written by phase2_b200/autotune.py)
 * if its GPU name equals `gpu` (NULL: the current CUDA device's name).
 * Returns the entries applied, 0 for a table of another GPU, -1 for a
 * missing or malformed file (nothing applied).  world_init applies the
 * table shipped beside the library, tuning_b200.tab (or the file named by
 * PHASE2_TUNING; PHASE2_TUNING=off skips it), before the PHASE2_*
 * settings from the environment. */
int phase2_load_tuning(const char *path, const char *gpu);

/* ---- term order --------------------------------------------------------- */

/* Order used by trott_init / trott2_init and the deterministic part of
 * cmpsit_init.  LEX (default) is the reference's lexicographic sort and
 * keeps results identical to it; GIVEN keeps the caller's order; FLIP
 * sorts by flip mask (stable), which groups terms that fuse into one pass
 * but changes the product formula. */
enum phase2_order {
	PHASE2_ORDER_LEX = 0,
	PHASE2_ORDER_GIVEN = 1,
	PHASE2_ORDER_FLIP = 2,
};
int phase2_set_term_order(int order);
int phase2_get_term_order(void);

/* Stable sort by (flip mask, phase mask). */
void circ_hamil_sort_flip(struct circ_hamil *hm);

/* ---- batched drivers ------------------------------------------------------ */

/*
 * Batched drivers run in one of two ways.  Persistent (default, when every
 * instance is a register of at most 31 qubits of one precision, FP32 in
 * either FP32 form or FP64): each instance's steps
 * are recorded as a program and all programs run in ONE persistent kernel
 * launch that schedules (instance, op, tile) work over all SMs; every
 * instance keeps the pass kernels' arithmetic (FP64: exact, bit-identical
 * to the reference; FP32: that of its form), so results equal the
 * per-instance stream mode's bit for bit.  Otherwise, or after phase2_set_batch_persistent(0):
 * per-instance streams as described below.
 */
int phase2_set_batch_persistent(int on);

/*
 * Run length of the persistent launch (also device sampling's): an op is
 * cut into tiles of 1024 amplitudes, and a warp claims runs of tiles, what
 * is left of the op times the programs running, divided by (resident
 * warps x per_warp), 1 to 16 tiles.
 * Larger per_warp: shorter runs (more claims, finer balance).  Default 2;
 * 1..64, else -1.  Results do not depend on it.
 */
int phase2_set_batch_runs(unsigned int per_warp);
unsigned int phase2_get_batch_runs(void);

/*
 * Sweeps (FP32 registers in PHASE2_FORM_LIFTED_F32, tile + 3 to 31
 * qubits): the planner also closes passes at sweep boundaries, a sweep
 * being a run of passes whose bases, modulo the low `low_qubits` qubits,
 * span at most tile_qubits - low_qubits dimensions (struct
 * phase2_pass.sweep marks its first pass), and the executor runs each
 * sweep as ONE kernel that reads and writes the state once: it walks tiles
 * of 2^tile_qubits amplitudes closed under those passes, the first pass
 * reading from HBM, the middle ones in shared memory, the last writing
 * back.  The FP32 plan therefore depends on the shape; running a plan's
 * sweeps as one kernel each is bit-identical to one kernel per pass
 * (phase2_set_sweep_kernel(0)).  tile_qubits 0 turns sweeps off.  Valid:
 * tile 8..14, low 3..8, tile - low <= 9.  Returns -1 on invalid values.
 */
int phase2_set_sweep(int tile_qubits, int low_qubits);
void phase2_get_sweep(int *tile_qubits, int *low_qubits);
/* on = 0: keep the sweep grouping of plans but run one kernel per pass
 * (the same bits, one state round trip per pass; for comparisons). */
int phase2_set_sweep_kernel(int on);

/*
 * qdrift_simul and cmpsit_simul with device sampling: when the register
 * runs in the persistent kernel (at most 31 qubits; FP64, or FP32 in
 * either form) and the trial state is a MULTIDET, the samples'
 * term draws (CDF inversion of the host generator's
 * uniforms), their pass plans and their passes all run on the GPU: one
 * planning kernel per round of samples (a block per sample) writes the
 * programs that one persistent launch executes, several samples at once
 * on copies of the state where the register is small.  The host only steps
 * the generator to each sample's start.  The overlaps, the register's
 * final state, the generator's end state and the last sample's drawn terms
 * equal the host loop's bit for bit.
 *
 * Modes: OFF (host loop), ON (device whenever the register qualifies),
 * AUTO (default: device for qualifying registers of at most
 * PHASE2_DEVICE_SAMPLING_AUTO_QB qubits, where samples run concurrently;
 * wider registers keep the host loop, whose passes already fill the GPU).
 * Step writers: under AUTO a driver with a step writer attached keeps the
 * host loop, which calls the writer as each sample completes (a writer
 * that flushes per step stays crash-consistent and can report progress);
 * under ON the writer is called for every sample, in sample order, after
 * the device has run them all.  Either way it sees the same (index,
 * overlap) sequence.  Also PHASE2_DEVICE_SAMPLING=off|on|auto.  Returns -1
 * on a bad mode.
 */
enum phase2_device_sampling {
	PHASE2_DEVICE_SAMPLING_OFF = 0,
	PHASE2_DEVICE_SAMPLING_ON = 1,
	PHASE2_DEVICE_SAMPLING_AUTO = 2,
};
#define PHASE2_DEVICE_SAMPLING_AUTO_QB 21
int phase2_set_device_sampling(int mode);

/* Check of the persistent kernel's bounded wait: runs it on a program
 * that can never progress (its only tile taken, never completed), so
 * every warp gives up after idle_limit idle rounds (about a microsecond
 * each) and reports it, without touching any state.  1: the launch ended
 * with the wait reported, 0: it ended without, -1: CUDA error.  No
 * counterpart in the reference (its waits are MPI's). */
int phase2_batch_wait_check(unsigned int idle_limit);

/* Finish time of every instance of the last persistent batch launch, in
 * ms after the launch's first warp started (device global timer), in the
 * order the instances were given: copies min(n, count) values to out and
 * returns the count (0 before any persistent launch).  Shows the tail of
 * uneven batches: the spread between the first and the last instance to
 * finish. */
size_t phase2_batch_finish_ms(double *out, size_t n);

/*
 * Run n independent, already initialised problems of one kind together.
 * Persistent mode (above): one launch for all instances and all their
 * steps.  Stream mode: each keeps its own register (its own CUDA stream),
 * and the host advances them in lockstep, enqueuing instance i's next step
 * as soon as its current overlap has been read, so the GPU overlaps the
 * instances' work (and replays each instance's repeated step plan from a
 * CUDA graph).  Either way results land in each problem's ct.vals and step
 * writer as the single-problem *_simul calls would produce them (the
 * writer is called after the launch in persistent mode).  0, or -1 if any
 * instance failed (the others still run to completion).
 */
struct trott;
struct trott2;
struct qdrift;
struct cmpsit;
struct cmpsit_data;
struct cmpsit_ranct;
int trott_simul_batch(struct trott *const *tts, size_t n);
int trott2_simul_batch(struct trott2 *const *t2s, size_t n);
int qdrift_simul_batch(struct qdrift *const *qds, size_t n);
int cmpsit_simul_batch(struct cmpsit *const *cps, size_t n);

/*
 * The composite driver's term split alone, without a circuit or register:
 * the first dt->length terms by |c| descending (then in the term order of
 * phase2_set_term_order) into rc->hm_det, the rest into rc->hm_ran with
 * its |c| CDF in rc->cdf and lambda_r (circ/cmpsit.c:65-111), exactly as
 * cmpsit_init splits them.  For drivers above the C surface that apply the
 * same rotations to a register of their own (sharded registers).  Needs
 * dt->length < hm->len; 0 or -1.  cmpsit_ranct_free releases it
 * (idempotent).
 */
int cmpsit_ranct_init(struct cmpsit_ranct *rc, const struct circ_hamil *hm,
	const struct cmpsit_data *dt);
void cmpsit_ranct_free(struct cmpsit_ranct *rc);

/* ---- execution control and bulk access ---------------------------------- */

/* Launch all queued rotations (asynchronously).  0 or -1. */
int qreg_flush(struct qreg *reg);

/* Flush and wait for the register's stream.  0, or -1 if a CUDA error was
 * raised on it. */
int qreg_synchronize(struct qreg *reg);

/* Batched amplitude access (one launch and one copy each way). */
int qreg_getamps(struct qreg *reg, const uint64_t *idx, _Complex double *z,
	size_t n);
int qreg_setamps(struct qreg *reg, const uint64_t *idx,
	const _Complex double *z, size_t n);

/* Whole state as interleaved FP64 re/im (2 * namp doubles). */
int qreg_get_state(struct qreg *reg, double *out);
int qreg_set_state(struct qreg *reg, const double *in);

/* sum |a_i|^2 in FP64 on the device: warp-shuffle tree per block, blocks
 * combined with compensated (Neumaier) summation.  0 or -1. */
int qreg_norm2(struct qreg *reg, double *out);

/* <trial|psi> for a dense FP64 trial state given in host memory
 * (2 * namp doubles), reduced on the device like qreg_norm2. */
int qreg_inner_dense(struct qreg *reg, const double *trial, double out[2]);

/* ---- half slabs (registers sharded by high qubits) ---------------------- */

/*
 * Copy elements [first, first + count) of the half {i : bit `bit` of i ==
 * val} of the register's amplitudes (namp / 2 of them, in increasing index
 * order) to (get) or from (put) the contiguous device buffer d_buf, which
 * holds them at the register's precision (complex128 for FP64 registers,
 * complex64 for FP32).  The copy has finished when the call returns.
 *
 * These replace the reference's slab exchange buffers (phase2/qreg.c:
 * 124-142, the backend hooks qreg_backend_exch_init/_waitall of
 * phase2/qreg.h:14-33): a register sharded over 2^g ranks by its g high
 * qubits swaps a high qubit with a local qubit l by exchanging, with the
 * partner rank, the half whose bit l differs from its own rank bit
 * (phase2_b200/sharded.py); get/put move that half, chunk by chunk,
 * through exchange buffers the caller owns (for NCCL, torch tensors).
 *
 * d_buf must be device memory of the register's device, aligned to the
 * element size, with count elements inside one allocation; anything else
 * returns -1 with an error and copies nothing, as do bit >= nqb, val > 1
 * and a range past namp / 2.  0 on success.
 */
int qreg_slab_get(struct qreg *reg, uint32_t bit, uint32_t val,
	uint64_t first, uint64_t count, void *d_buf);
int qreg_slab_put(struct qreg *reg, uint32_t bit, uint32_t val,
	uint64_t first, uint64_t count, const void *d_buf);

/*
 * The same exchange between two registers on one device, in place: the
 * half {i : bit `bit` of i == val_a} of a trades places, element for
 * element in index order, with the half {i : bit of i == val_b} of b.  One
 * kernel reads and writes both halves once (no buffers); it runs the
 * exchange of paired ranks that one process holds on one GPU.  a and b
 * must be distinct registers of one size and precision on one device.
 * Finished when the call returns; 0 or -1.
 */
int qreg_slab_swap(struct qreg *a, struct qreg *b, uint32_t bit,
	uint32_t val_a, uint32_t val_b);

/* ---- counters ----------------------------------------------------------- */

struct phase2_stats {
	uint64_t rotations; /* rotations executed */
	uint64_t passes;    /* passes (fused rotation groups) executed */
	uint64_t launches;  /* kernels launched by this library */
	uint64_t bytes;     /* algorithmic HBM bytes: 2 * namp * elem per
			     * state round trip (sweeps) */
	uint64_t timed_passes;
	double pass_ms;     /* device time of timed pass launches (CUDA events) */
	uint64_t h2d_bytes; /* host-to-device bytes copied for this register */
	uint64_t d2h_bytes; /* device-to-host bytes copied for this register */
	uint64_t graph_replays; /* flushes launched from a captured CUDA graph
				 * (a plan seen before, e.g. every Trotter
				 * step after the second; registers of up to
				 * 24 qubits) */
	uint64_t sweeps;    /* state round trips: one per pass kernel, one per
			     * sweep kernel (several passes, phase2_set_sweep) */
	uint64_t timed_sweeps; /* round trips inside pass_ms */
};

int qreg_get_stats(const struct qreg *reg, struct phase2_stats *st);
void qreg_reset_stats(struct qreg *reg);

/* Record CUDA events around each flush's pass launches on the register's
 * stream and accumulate their elapsed time into pass_ms. */
int qreg_set_timing(struct qreg *reg, int on);

/* The cudaStream_t (as void *) on which all work of this register runs,
 * for callers that record CUDA events around library calls. */
void *qreg_stream(const struct qreg *reg);

/* ---- allocation-free reduction ------------------------------------------ */

/*
 * sum |a_i|^2 of a state the caller already holds in device memory,
 * without allocating anything.  This entry point has no counterpart in the
 * reference.
 *
 * It exists for callers that cannot call cudaMalloc: code whose device
 * memory is owned by its own pool or arena and may not allocate outside
 * it, and latency-critical loops that cannot afford the implicit device
 * synchronisation cudaMalloc/cudaFree bring.  qreg_norm2 computes the same
 * sum but allocates its partials buffer on first use.
 *
 *   d_state  device pointer to namp amplitudes: complex128 (prec =
 *            PHASE2_PREC_FP64) or complex64 (PHASE2_PREC_FP32), memory of
 *            the current device with all namp amplitudes inside one
 *            allocation; a host pointer, another device's memory or a
 *            shorter buffer returns -1 before anything is launched
 *   namp     1 .. 2^34 (the fixed scratch holds 8192 partial sums of up
 *            to 2^21 amplitudes each); larger sizes return -1 with an error
 *   d_out    device pointer to 2 doubles (16-byte aligned, checked like
 *            d_state); receives {sum, 0}
 *   stream   cudaStream_t (NULL = legacy default stream); the call is
 *            asynchronous on it
 *
 * The per-block partial sums live in a static device array (about
 * 128 KiB) that every GPU loading the library holds until the process
 * exits.  The first call on a device looks up that array's address and
 * caches it; make that first call before starting any stream capture.  A
 * cudaDeviceReset invalidates the cached address: do not call this entry
 * point on a device after resetting it in the same process.
 * All calls share the array: two calls whose kernels overlap on the GPU
 * (different streams, no ordering between them) race on it and may
 * return wrong sums.  Calls ordered on one stream are safe; nothing in the
 * array needs to start at zero.  Returns 0 (launched) or -1.
 */
int phase2_norm2_noalloc(const void *d_state, int prec, uint64_t namp,
	double *d_out, void *stream);

/* ---- planner (host) ----------------------------------------------------- */

/* One rotation exp(i phi P) with P = (flip, phase). */
struct phase2_rot_in {
	uint64_t flip, phase;
	double phi;
};

/* Pass descriptor as executed by the device.  Slot u of a thread with
 * representative x (x has zeros at the pivot bits) is amplitude
 * x ^ (xor of basis[k] over the set bits k of u). */
#define PHASE2_MAX_SPAN 5
struct phase2_pass {
	uint32_t span;     /* M: slots per thread = 2^M */
	uint32_t nrot;     /* rotations in this pass */
	uint32_t rot_off;  /* first rotation record */
	uint8_t piv[PHASE2_MAX_SPAN]; /* pivot bits, ascending */
	uint8_t form;      /* PHASE2_FORM_* of every record of the pass */
	uint8_t sweep;     /* 1: the pass starts a sweep (phase2_set_sweep);
			    * the passes up to the next start share one tile
			    * shape and may run as one kernel */
	uint8_t pad;
	uint64_t basis[PHASE2_MAX_SPAN];
	double scale;      /* lifted forms: +-1, applied at the store */
};

/* Arithmetic of a pass (struct phase2_pass.form). */
enum phase2_form {
	PHASE2_FORM_EXACT = 0,      /* FP64 state: the reference's update,
				     * records of form 0 */
	PHASE2_FORM_LIFTED = 1,     /* FP32 state, records of form 1, FP64
				     * arithmetic */
	PHASE2_FORM_LIFTED_F32 = 2, /* FP32 state, records of form 1 with FP32
				     * s, FP32 arithmetic */
	PHASE2_FORM_LIFTED_MIXED = 3, /* records as LIFTED_F32; FP32
				       * arithmetic, FP64 on cosets with an
				       * amplitude >= 2^-10 */
};

/* Rotation record in slot coordinates: the partner of slot u is u ^ U; the
 * sign bit of slot u for a thread with representative x is
 * bit u of smask XOR parity(x & z); odd = 1 multiplies the partner by i.
 *
 * form 0 (exact, FP64 state):   a_u <- c a_u + (+-s) p_u,
 *     p_u the partner (times i when odd);
 * form 1 (lifted, FP32 state):  three in-place shears of the pair,
 *     y_u += t q_u y_w;  y_w += s q_w y_u;  y_u += t q_u y_w,
 *     q_u = (+-1)(odd ? i : 1), q_w = -conj(q_u), t = (1 - cos phi) / s
 *     held in `c`; a rotation with cos(phi) < 0 is stored as
 *     exp(i(phi -+ pi)P) and the pass negates every amplitude once per such
 *     rotation (`scale` = +-1).  For PHASE2_FORM_LIFTED_F32 and
 *     PHASE2_FORM_LIFTED_MIXED passes s is an FP32 value and t is taken
 *     against it. */
struct phase2_rot_rec {
	uint64_t z;
	double c, s;
	uint32_t smask;
	uint8_t U;
	uint8_t W;    /* bit k = parity(basis[k] & z): smask bit u = bit 0 of
		       * smask XOR parity(u & W) */
	uint8_t odd;
	uint8_t form;
};

/* Plan n rotations for an nqb-qubit register of precision prec (FP64:
 * exact form; FP32: the process's FP32 form, mixed by default).  Writes at most n passes and n records;
 * returns the number of passes, or -1. */
long phase2_plan(uint32_t nqb, const struct phase2_rot_in *rots, size_t n,
	int max_span, int max_rots, int prec, struct phase2_pass *passes,
	struct phase2_rot_rec *recs);

/* ---- misc --------------------------------------------------------------- */

const char *phase2_version(void);

/* sizeof of public structs, for FFI layout checks: 0 qreg, 1 circ, 2 trott,
 * 3 trott2, 4 qdrift, 5 cmpsit, 6 circ_hamil_term, 7 phase2_pass,
 * 8 phase2_rot_rec, 9 phase2_stats; 0 for unknown ids. */
size_t phase2_sizeof(int which);

#ifdef __cplusplus
}
#endif

#endif /* PHASE2_B200_H */
