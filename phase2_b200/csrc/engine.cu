/*
 * engine.cu -- device side of libphase2.so for sm_100a (B200).
 *
 * The state vector is one flat array of 2^n complex amplitudes in HBM,
 * complex128 (double2) or complex64 (float2), updated in place.
 *
 * Hot kernels: k_pass<M> (FP64 state), k_pass_lift32<M> and k_pass_lift<M>
 * (FP32 state).  One launch = one HBM sweep that applies a planned run of
 * rotations (plan.c).  Each thread owns whole cosets
 * x + span(basis[0..M-1]): it loads the 2^M amplitudes of a coset into
 * registers, applies every rotation of the run in order (partners of a
 * rotation are always inside the coset), and writes them back.  Warp
 * lanes take consecutive representatives x, so for each slot the warp
 * touches one contiguous 256 B (FP32) or 512 B (FP64) segment: coalesced,
 * one read and one write of every amplitude per pass, no shared-memory
 * staging of amplitudes.  It is a streaming pair sweep on CUDA cores; there
 * is no contraction for the tensor cores to do.
 *
 * FP64 state: products and sums are rounded separately with
 * __dmul_rn/__dadd_rn, never fused, so every amplitude is bit-identical to
 * the reference CPU update a_i <- c a_i + i conj(s z) a_j
 * (phase2/qreg_qreg.c:149-160).  FP32 state: each pair is rotated by three
 * in-place shears (the lifted form), in FP32 FMAs (k_pass_lift32, the
 * default) or in FP64 with one rounding to FP32 per pass (k_pass_lift).
 *
 * Other kernels: gather/scatter of a few amplitudes (overlap, state prep),
 * and a two-stage FP64 sum of squares / inner product (warp-shuffle tree
 * per block, then one block combining the per-block partials with
 * Neumaier compensated summation).
 */
#include <cuda_runtime.h>

#include <float.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "engine"
#include "log.h"

#include "p2_internal.h"
#include "plan_core.h"

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

/* ---- arithmetic --------------------------------------------------------- */

/* Products and sums rounded separately (no FMA contraction), as the
 * reference's CPU build computes them. */
__device__ __forceinline__ double p2_mul(double a, double b)
{
	return __dmul_rn(a, b);
}

/* c*x + t with two roundings. */
__device__ __forceinline__ double p2_cxt(double c, double x, double t)
{
	return __dadd_rn(__dmul_rn(c, x), t);
}

__host__ __device__ constexpr int p2_hibit(int v)
{
	return v <= 1 ? 0 : 1 + p2_hibit(v >> 1);
}

/* k with a zero bit inserted at position h (pair index -> lower slot). */
__host__ __device__ constexpr int p2_ins0(int g, int h)
{
	return ((g >> h) << (h + 1)) | (g & ((1 << h) - 1));
}

/* Bit u of sm moved to the sign position (u is a compile-time constant
 * after unrolling: one shift and one mask, independent per slot). */
__device__ __forceinline__ uint32_t p2_bitmask(uint32_t sm, int u)
{
	return (sm << (31 - u)) & 0x80000000u;
}

/* v with the sign mask (0 or 1 << 31) XORed into its high word. */
__device__ __forceinline__ double p2_sgn(double v, uint32_t mask)
{
	return __hiloint2double(__double2hiint(v) ^ (int)mask,
		__double2loint(v));
}

/*
 * One rotation on the 2^M slots of a coset (FP64 state, exact rounding).
 * The sign of slot u is bit u of sm (the thread's parity already folded
 * in); each slot's sign is extracted independently so the per-slot work
 * has no serial dependency.
 */
template <int M, int U, int ODD>
__device__ __forceinline__ void p2_rot(double (&re)[1 << M],
	double (&im)[1 << M], double c, double s, uint32_t sm, uint32_t W)
{
	(void)W;
	if constexpr (U == 0) {
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			const double su = p2_sgn(s, p2_bitmask(sm, u));
			double tr, ti;
			if constexpr (ODD) {
				tr = p2_mul(-su, im[u]);
				ti = p2_mul(su, re[u]);
			} else {
				tr = p2_mul(su, re[u]);
				ti = p2_mul(su, im[u]);
			}
			re[u] = p2_cxt(c, re[u], tr);
			im[u] = p2_cxt(c, im[u], ti);
		}
	} else {
		constexpr int H = p2_hibit(U);
#pragma unroll
		for (int k = 0; k < (1 << (M - 1)); ++k) {
			const int u = p2_ins0(k, H);
			const int w = u ^ U;
			const double su = p2_sgn(s, p2_bitmask(sm, u));
			const double sw = p2_sgn(s, p2_bitmask(sm, w));
			double tur, tui, twr, twi;
			if constexpr (ODD) {
				tur = p2_mul(-su, im[w]);
				tui = p2_mul(su, re[w]);
				twr = p2_mul(-sw, im[u]);
				twi = p2_mul(sw, re[u]);
			} else {
				tur = p2_mul(su, re[w]);
				tui = p2_mul(su, im[w]);
				twr = p2_mul(sw, re[u]);
				twi = p2_mul(sw, im[u]);
			}
			const double nur = p2_cxt(c, re[u], tur);
			const double nui = p2_cxt(c, im[u], tui);
			const double nwr = p2_cxt(c, re[w], twr);
			const double nwi = p2_cxt(c, im[w], twi);
			re[u] = nur;
			im[u] = nui;
			re[w] = nwr;
			im[w] = nwi;
		}
	}
}

#define P2_CASE(K)                                                             \
	case K:                                                                \
		if constexpr ((K) < (2 << M))                                  \
			p2_rot<M, ((K) >> 1), ((K)&1)>(re, im, c, s, sm, W);   \
		break;

/* key = U << 1 | odd; a jump table over the (U, odd) variants. */
template <int M>
__device__ __forceinline__ void p2_apply(uint32_t key, double (&re)[1 << M],
	double (&im)[1 << M], double c, double s, uint32_t sm, uint32_t W)
{
	switch (key) {
		P2_CASE(0) P2_CASE(1) P2_CASE(2) P2_CASE(3) P2_CASE(4)
		P2_CASE(5) P2_CASE(6) P2_CASE(7) P2_CASE(8) P2_CASE(9)
		P2_CASE(10) P2_CASE(11) P2_CASE(12) P2_CASE(13) P2_CASE(14)
		P2_CASE(15) P2_CASE(16) P2_CASE(17) P2_CASE(18) P2_CASE(19)
		P2_CASE(20) P2_CASE(21) P2_CASE(22) P2_CASE(23) P2_CASE(24)
		P2_CASE(25) P2_CASE(26) P2_CASE(27) P2_CASE(28) P2_CASE(29)
		P2_CASE(30) P2_CASE(31) P2_CASE(32) P2_CASE(33) P2_CASE(34)
		P2_CASE(35) P2_CASE(36) P2_CASE(37) P2_CASE(38) P2_CASE(39)
		P2_CASE(40) P2_CASE(41) P2_CASE(42) P2_CASE(43) P2_CASE(44)
		P2_CASE(45) P2_CASE(46) P2_CASE(47) P2_CASE(48) P2_CASE(49)
		P2_CASE(50) P2_CASE(51) P2_CASE(52) P2_CASE(53) P2_CASE(54)
		P2_CASE(55) P2_CASE(56) P2_CASE(57) P2_CASE(58) P2_CASE(59)
		P2_CASE(60) P2_CASE(61) P2_CASE(62) P2_CASE(63)
	default:
		break;
	}
}
#undef P2_CASE

/* ---- storage ------------------------------------------------------------ */

__device__ __forceinline__ void p2_ld(const double2 *st, uint64_t g,
	double &re, double &im)
{
	const double2 v = st[g];
	re = v.x;
	im = v.y;
}

__device__ __forceinline__ void p2_ld(const float2 *st, uint64_t g,
	double &re, double &im)
{
	const float2 v = st[g];
	re = (double)v.x;
	im = (double)v.y;
}

__device__ __forceinline__ void p2_st(double2 *st, uint64_t g, double re,
	double im)
{
	st[g] = make_double2(re, im);
}

__device__ __forceinline__ void p2_st(float2 *st, uint64_t g, double re,
	double im)
{
	st[g] = make_float2(__double2float_rn(re), __double2float_rn(im));
}

template <int M>
__device__ __forceinline__ uint64_t p2_slot_off(int u, const uint64_t *basis)
{
	uint64_t off = 0;
#pragma unroll
	for (int k = 0; k < M; ++k)
		if (u >> k & 1)
			off ^= basis[k];
	return off;
}

/* ---- the pass kernel ---------------------------------------------------- */

/* Threads per block of the FP64 prefetch kernel: 128, or 64 with 32 slots
 * per thread (three blocks of two stages then fit in shared memory). */
__host__ __device__ constexpr int p2_tpb(int m)
{
	return m >= 5 ? 64 : P2_TPB;
}

/* Resident blocks per SM the register allocation should allow: 2^M FP64
 * complex values need 4 * 2^M registers per thread. */
__host__ __device__ constexpr int p2_min_blocks(int m)
{
	return m >= 5 ? 1 : (m == 4 ? 4 : (m == 3 ? 6 : 8));
}

/* Representative number t -> index x: zeros inserted at the pivots. */
template <int M>
__device__ __forceinline__ uint64_t p2_rep(uint64_t t,
	const struct phase2_pass &p)
{
	uint64_t x = t;
#pragma unroll
	for (int k = 0; k < M; ++k) {
		const uint32_t q = p.piv[k];
		x = ((x >> q) << (q + 1)) | (x & ((UINT64_C(1) << q) - 1));
	}
	return x;
}

/* Asynchronous global -> shared copy of one amplitude. */
__device__ __forceinline__ void p2_cp_async(double2 *smem, const double2 *g)
{
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s),
		"l"(g)
		: "memory");
}

__device__ __forceinline__ void p2_cp_commit()
{
	asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N> __device__ __forceinline__ void p2_cp_wait()
{
	asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

/* The run of rotations of one pass on one coset held in registers. */
template <int M>
__device__ __forceinline__ void p2_apply_run(double (&re)[1 << M],
	double (&im)[1 << M], uint64_t x, const struct phase2_rot_rec *srec,
	uint32_t nrot)
{
	for (uint32_t r = 0; r < nrot; ++r) {
		const uint64_t z = srec[r].z;
		const uint32_t px = (uint32_t)(__popcll(x & z) & 1);
		const uint32_t sm = srec[r].smask ^ (0u - px);
		const uint32_t key = ((uint32_t)srec[r].U << 1) | srec[r].odd;
		p2_apply<M>(key, re, im, srec[r].c, srec[r].s, sm, srec[r].W);
	}
}

/* Stage layout [slot][thread]: a warp's accesses to one slot are 32
 * consecutive elements, conflict-free. */
template <int M>
__device__ __forceinline__ void p2_prefetch(double2 *stage, const double2 *st,
	uint64_t x, const uint64_t (&pb)[M > 0 ? M : 1])
{
#pragma unroll
	for (int u = 0; u < (1 << M); ++u)
		p2_cp_async(&stage[u * blockDim.x + threadIdx.x],
			st + (x ^ p2_slot_off<M>(u, pb)));
}

/*
 * One pass.  Persistent grid: each thread walks representatives
 * t, t + stride, ...; while it applies the rotations to coset t in
 * registers, the 2^M amplitudes of coset t + stride are already on their
 * way into its own shared-memory stage (cp.async), so every warp keeps
 * loads in flight during its compute.  A thread only ever reads the stage
 * slots it copied itself: cp.async.wait_group orders them, no block
 * barrier is needed inside the loop.  The next prefetch into a stage is
 * issued after the values read from it have been consumed (in-order issue),
 * so the stage is never overwritten early.
 */
template <int M>
__global__ void __launch_bounds__(p2_tpb(M), p2_min_blocks(M))
	k_pass_pf(double2 *__restrict__ st, uint64_t nrep, struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs)
{
	extern __shared__ __align__(16) unsigned char p2_dyn[];
	double2 *const stage = (double2 *)p2_dyn;
	__shared__ struct phase2_rot_rec srec[P2_MAX_ROTS_PER_PASS];
	__shared__ uint64_t sbasis[PHASE2_MAX_SPAN];
	for (uint32_t r = threadIdx.x; r < p.nrot; r += blockDim.x)
		srec[r] = recs[p.rot_off + r];
	if (threadIdx.x == 0) {
#pragma unroll
		for (int k = 0; k < M; ++k)
			sbasis[k] = p.basis[k];
	}
	__syncthreads();
	uint64_t pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = p.basis[k];

	const uint32_t nst = (1u << M) * blockDim.x; /* elements per stage */
	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (t < nrep)
		p2_prefetch<M>(stage, st, p2_rep<M>(t, p), pb);
	p2_cp_commit();
	uint32_t cur = 0;
	for (; t < nrep; t += stride) {
		const uint64_t tn = t + stride;
		if (tn < nrep)
			p2_prefetch<M>(stage + (cur ^ 1) * nst, st,
				p2_rep<M>(tn, p), pb);
		p2_cp_commit();
		p2_cp_wait<1>();

		const uint64_t x = p2_rep<M>(t, p);
		double re[1 << M], im[1 << M];
		const double2 *const mine = stage + cur * nst + threadIdx.x;
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			const double2 v = mine[u * blockDim.x];
			re[u] = v.x;
			im[u] = v.y;
		}

		p2_apply_run<M>(re, im, x, srec, p.nrot);
		/* Slot addresses are recomputed from the shared copy of the
		 * basis rather than kept live across the rotations. */
#pragma unroll
		for (int u = 0; u < (1 << M); ++u)
			p2_st(st, x ^ p2_slot_off<M>(u, sbasis), re[u], im[u]);
		cur ^= 1;
	}
	p2_cp_wait<0>();
}

/*
 * One pass, direct variant: each thread loads its coset straight from HBM
 * into registers (all 2^M loads issued back to back), applies the run and
 * stores; latency is hidden by the other resident warps only.  The grid
 * covers every representative once (no persistent loop state).
 */
template <int M>
__global__ void __launch_bounds__(P2_TPB, p2_min_blocks(M))
	k_pass(double2 *__restrict__ st, uint64_t nrep, struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs)
{
	__shared__ struct phase2_rot_rec srec[P2_MAX_ROTS_PER_PASS];
	__shared__ uint64_t sbasis[PHASE2_MAX_SPAN];
	for (uint32_t r = threadIdx.x; r < p.nrot; r += blockDim.x)
		srec[r] = recs[p.rot_off + r];
	if (threadIdx.x == 0) {
#pragma unroll
		for (int k = 0; k < M; ++k)
			sbasis[k] = p.basis[k];
	}
	__syncthreads();
	uint64_t pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = p.basis[k];

	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		t < nrep; t += stride) {
		const uint64_t x = p2_rep<M>(t, p);
		double re[1 << M], im[1 << M];
#pragma unroll
		for (int u = 0; u < (1 << M); ++u)
			p2_ld(st, x ^ p2_slot_off<M>(u, pb), re[u], im[u]);
		p2_apply_run<M>(re, im, x, srec, p.nrot);
#pragma unroll
		for (int u = 0; u < (1 << M); ++u)
			p2_st(st, x ^ p2_slot_off<M>(u, sbasis), re[u], im[u]);
	}
}

/* ---- lifted pass kernel (FP32 storage) ---------------------------------- */

/*
 * One lifted rotation on the 2^M slots of a coset.  A pair (u, w = u ^ U)
 * with sign sigma (bit u of sm) is rotated by three in-place shears,
 *   y_u += t q_u y_w;  y_w += s q_w y_u;  y_u += t q_u y_w,
 * q_u = sigma (odd ? i : 1), q_w = -conj(q_u), t = tan(phi/2): every update
 * writes the register it reads, so a case needs no temporaries and leaves
 * no moves behind.  The partner is held as sigma * y_w during the shears
 * (its sign bits flipped in place), which makes all six FMAs sign-free.
 * U = 0 (the string is diagonal on the coset, and then odd = 1) is the
 * phase c + i sigma s, applied to (re, sigma im) by the same three shears.
 */
template <int M, int U, int ODD>
__device__ __forceinline__ void p2_rot_lift(double (&re)[1 << M],
	double (&im)[1 << M], double t, double s, uint32_t sm)
{
	if constexpr (U == 0) {
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			const uint32_t g = p2_bitmask(sm, u);
			if constexpr (ODD) {
				double v = p2_sgn(im[u], g);
				re[u] = fma(-t, v, re[u]);
				v = fma(s, re[u], v);
				re[u] = fma(-t, v, re[u]);
				im[u] = p2_sgn(v, g);
			} else {
				/* (c +- s) y with c = 1 - t s; a Hermitian string
				 * that is diagonal on the coset never has it */
				const double k = p2_sgn(s, g) + fma(-t, s, 1.0);
				re[u] *= k;
				im[u] *= k;
			}
		}
	} else {
		constexpr int H = p2_hibit(U);
#pragma unroll
		for (int k = 0; k < (1 << (M - 1)); ++k) {
			const int u = p2_ins0(k, H);
			const int w = u ^ U;
			const uint32_t g = p2_bitmask(sm, u);
			double wr = p2_sgn(re[w], g), wi = p2_sgn(im[w], g);
			if constexpr (ODD) {
				re[u] = fma(-t, wi, re[u]);
				im[u] = fma(t, wr, im[u]);
				wr = fma(-s, im[u], wr);
				wi = fma(s, re[u], wi);
				re[u] = fma(-t, wi, re[u]);
				im[u] = fma(t, wr, im[u]);
			} else {
				re[u] = fma(t, wr, re[u]);
				im[u] = fma(t, wi, im[u]);
				wr = fma(-s, re[u], wr);
				wi = fma(-s, im[u], wi);
				re[u] = fma(t, wr, re[u]);
				im[u] = fma(t, wi, im[u]);
			}
			re[w] = p2_sgn(wr, g);
			im[w] = p2_sgn(wi, g);
		}
	}
}

#define P2_CASE_L(K)                                                           \
	case K:                                                                \
		if constexpr ((K) < (2 << M))                                  \
			p2_rot_lift<M, ((K) >> 1), ((K)&1)>(re, im, t, s, sm); \
		break;

/* key = U << 1 | odd */
template <int M>
__device__ __forceinline__ void p2_apply_lift(uint32_t key,
	double (&re)[1 << M], double (&im)[1 << M], double t, double s,
	uint32_t sm)
{
	switch (key) {
		P2_CASE_L(0) P2_CASE_L(1) P2_CASE_L(2) P2_CASE_L(3)
		P2_CASE_L(4) P2_CASE_L(5) P2_CASE_L(6) P2_CASE_L(7)
		P2_CASE_L(8) P2_CASE_L(9) P2_CASE_L(10) P2_CASE_L(11)
		P2_CASE_L(12) P2_CASE_L(13) P2_CASE_L(14) P2_CASE_L(15)
		P2_CASE_L(16) P2_CASE_L(17) P2_CASE_L(18) P2_CASE_L(19)
		P2_CASE_L(20) P2_CASE_L(21) P2_CASE_L(22) P2_CASE_L(23)
		P2_CASE_L(24) P2_CASE_L(25) P2_CASE_L(26) P2_CASE_L(27)
		P2_CASE_L(28) P2_CASE_L(29) P2_CASE_L(30) P2_CASE_L(31)
		P2_CASE_L(32) P2_CASE_L(33) P2_CASE_L(34) P2_CASE_L(35)
		P2_CASE_L(36) P2_CASE_L(37) P2_CASE_L(38) P2_CASE_L(39)
		P2_CASE_L(40) P2_CASE_L(41) P2_CASE_L(42) P2_CASE_L(43)
		P2_CASE_L(44) P2_CASE_L(45) P2_CASE_L(46) P2_CASE_L(47)
		P2_CASE_L(48) P2_CASE_L(49) P2_CASE_L(50) P2_CASE_L(51)
		P2_CASE_L(52) P2_CASE_L(53) P2_CASE_L(54) P2_CASE_L(55)
		P2_CASE_L(56) P2_CASE_L(57) P2_CASE_L(58) P2_CASE_L(59)
		P2_CASE_L(60) P2_CASE_L(61) P2_CASE_L(62) P2_CASE_L(63)
	default:
		break;
	}
}
#undef P2_CASE_L

/* A lifted record as the kernel reads it from shared memory. */
struct p2_lift_rec {
	double t, s;
	uint64_t z;
	uint32_t sm;  /* smask */
	uint32_t key; /* U << 1 | odd */
};

__device__ __forceinline__ uint32_t p2_parity(uint32_t v)
{
	return (uint32_t)__popc(v) & 1u;
}

__device__ __forceinline__ uint32_t p2_parity(uint64_t v)
{
	return (uint32_t)__popcll(v) & 1u;
}

/* x, with its value hidden from the optimiser: store addresses recomputed
 * from it are not merged with the load addresses, which would otherwise
 * stay live (2^M 64-bit pointers) across the whole run of rotations. */
__device__ __forceinline__ uint32_t p2_opaque(uint32_t x)
{
	asm volatile("" : "+r"(x));
	return x;
}

__device__ __forceinline__ uint64_t p2_opaque(uint64_t x)
{
	asm volatile("" : "+l"(x));
	return x;
}

/* Representative number t -> index x in index type IT (32-bit when the
 * register has at most 31 qubits, so that no shift reaches 32). */
template <int M, typename IT>
__device__ __forceinline__ IT p2_rep_t(IT t, const struct phase2_pass &p)
{
	IT x = t;
#pragma unroll
	for (int k = 0; k < M; ++k) {
		const uint32_t q = p.piv[k];
		x = ((x >> q) << (q + 1)) | (x & (((IT)1 << q) - 1));
	}
	return x;
}

/*
 * One FP32 pass in the lifted form: each thread loads its coset straight
 * from HBM (2^M independent 8-byte loads, coalesced across the warp),
 * widens to FP64, applies the run of rotations in registers and narrows
 * once at the store.  Index arithmetic is 32-bit when IT is uint32_t.
 * At M = 5, three resident blocks cap a thread at 168 registers (a few
 * spilled); measured faster than two blocks with no spills.
 */
template <int M, typename IT>
__global__ void __launch_bounds__(P2_TPB, M >= 5 ? 3 : p2_min_blocks(M))
	k_pass_lift(float2 *__restrict__ st, uint64_t nrep,
		struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs)
{
	__shared__ struct p2_lift_rec srec[P2_MAX_ROTS_PER_PASS];
	for (uint32_t r = threadIdx.x; r < p.nrot; r += blockDim.x) {
		const struct phase2_rot_rec in = recs[p.rot_off + r];
		struct p2_lift_rec o;
		o.t = in.c;
		o.s = in.s;
		o.z = in.z;
		o.sm = in.smask;
		o.key = ((uint32_t)in.U << 1) | in.odd;
		srec[r] = o;
	}
	__syncthreads();
	IT pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = (IT)p.basis[k];
	const bool neg = p.scale < 0;
	const uint32_t nrot = p.nrot;

	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		t < nrep; t += stride) {
		const IT x = p2_rep_t<M, IT>((IT)t, p);
		double re[1 << M], im[1 << M];
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			IT off = 0;
#pragma unroll
			for (int k = 0; k < M; ++k)
				if (u >> k & 1)
					off ^= pb[k];
			const float2 v = st[x ^ off];
			re[u] = (double)v.x;
			im[u] = (double)v.y;
		}
		for (uint32_t r = 0; r < nrot; ++r) {
			const struct p2_lift_rec q = srec[r];
			const uint32_t sm = q.sm ^ (0u - p2_parity(x & (IT)q.z));
			p2_apply_lift<M>(q.key, re, im, q.t, q.s, sm);
		}
		if (neg) {
#pragma unroll
			for (int u = 0; u < (1 << M); ++u) {
				re[u] = -re[u];
				im[u] = -im[u];
			}
		}
		const IT xs = p2_opaque(x);
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			IT off = 0;
#pragma unroll
			for (int k = 0; k < M; ++k)
				if (u >> k & 1)
					off ^= pb[k];
			st[xs ^ off] = make_float2(__double2float_rn(re[u]),
				__double2float_rn(im[u]));
		}
	}
}

/* ---- lifted pass kernel, FP32 arithmetic -------------------------------- */

__device__ __forceinline__ float p2_fsgn(float v, uint32_t mask)
{
	return __int_as_float(__float_as_int(v) ^ (int)mask);
}

/*
 * The lifted rotation of p2_rot_lift with the amplitudes in FP32 registers
 * and FP32 FMAs.  s reaches the kernel as an FP32 value and t = (1 - cos
 * phi) / s in FP64 (plan.c); the angle of the three shears is fixed by the
 * product t s (their trace is 2 (1 - t s)), so rounding t to FP32 leaves a
 * relative angle error of at most 2^-25.  The signs go onto the
 * coefficients (one XOR each on a 32-bit register).
 */
template <int M, int U, int ODD>
__device__ __forceinline__ void p2_rot_lift32(float (&re)[1 << M],
	float (&im)[1 << M], float t, float s, uint32_t sm)
{
	if constexpr (U == 0) {
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			const uint32_t g = p2_bitmask(sm, u);
			const float st = p2_fsgn(t, g), ss = p2_fsgn(s, g);
			if constexpr (ODD) {
				re[u] = fmaf(-st, im[u], re[u]);
				im[u] = fmaf(ss, re[u], im[u]);
				re[u] = fmaf(-st, im[u], re[u]);
			} else {
				/* (c +- s) y with c = 1 - t s; a Hermitian string
				 * that is diagonal on the coset never has it */
				const float k = ss + fmaf(-t, s, 1.f);
				re[u] *= k;
				im[u] *= k;
			}
		}
	} else {
		constexpr int H = p2_hibit(U);
#pragma unroll
		for (int k = 0; k < (1 << (M - 1)); ++k) {
			const int u = p2_ins0(k, H);
			const int w = u ^ U;
			const uint32_t g = p2_bitmask(sm, u);
			const float st = p2_fsgn(t, g), ss = p2_fsgn(s, g);
			if constexpr (ODD) {
				re[u] = fmaf(-st, im[w], re[u]);
				im[u] = fmaf(st, re[w], im[u]);
				re[w] = fmaf(-ss, im[u], re[w]);
				im[w] = fmaf(ss, re[u], im[w]);
				re[u] = fmaf(-st, im[w], re[u]);
				im[u] = fmaf(st, re[w], im[u]);
			} else {
				/* the same three shears as six fmaf, two lanes
				 * per packed FMA (round-to-nearest per lane: the
				 * same bits) */
				const float2 a = make_float2(st, st);
				const float2 b = make_float2(-ss, -ss);
				float2 yu = make_float2(re[u], im[u]);
				float2 yw = make_float2(re[w], im[w]);
				yu = __ffma2_rn(a, yw, yu);
				yw = __ffma2_rn(b, yu, yw);
				yu = __ffma2_rn(a, yw, yu);
				re[u] = yu.x;
				im[u] = yu.y;
				re[w] = yw.x;
				im[w] = yw.y;
			}
		}
	}
}

/* A lifted record as the FP32 kernel reads it. */
struct p2_lift32_rec {
	float t, s;
	uint64_t z;
	uint32_t sm;  /* smask */
	uint32_t key; /* U << 1 | odd */
};

#define P2_CASE_L32(K)                                                         \
	case K:                                                                \
		if constexpr ((K) < (2 << M))                                  \
			p2_rot_lift32<M, ((K) >> 1), ((K)&1)>(re, im, q.t,     \
				q.s, sm);                                      \
		break;

template <int M>
__device__ __forceinline__ void p2_apply_lift32(const struct p2_lift32_rec &q,
	float (&re)[1 << M], float (&im)[1 << M], uint32_t sm)
{
	switch (q.key) {
		P2_CASE_L32(0) P2_CASE_L32(1) P2_CASE_L32(2) P2_CASE_L32(3)
		P2_CASE_L32(4) P2_CASE_L32(5) P2_CASE_L32(6) P2_CASE_L32(7)
		P2_CASE_L32(8) P2_CASE_L32(9) P2_CASE_L32(10) P2_CASE_L32(11)
		P2_CASE_L32(12) P2_CASE_L32(13) P2_CASE_L32(14) P2_CASE_L32(15)
		P2_CASE_L32(16) P2_CASE_L32(17) P2_CASE_L32(18) P2_CASE_L32(19)
		P2_CASE_L32(20) P2_CASE_L32(21) P2_CASE_L32(22) P2_CASE_L32(23)
		P2_CASE_L32(24) P2_CASE_L32(25) P2_CASE_L32(26) P2_CASE_L32(27)
		P2_CASE_L32(28) P2_CASE_L32(29) P2_CASE_L32(30) P2_CASE_L32(31)
		P2_CASE_L32(32) P2_CASE_L32(33) P2_CASE_L32(34) P2_CASE_L32(35)
		P2_CASE_L32(36) P2_CASE_L32(37) P2_CASE_L32(38) P2_CASE_L32(39)
		P2_CASE_L32(40) P2_CASE_L32(41) P2_CASE_L32(42) P2_CASE_L32(43)
		P2_CASE_L32(44) P2_CASE_L32(45) P2_CASE_L32(46) P2_CASE_L32(47)
		P2_CASE_L32(48) P2_CASE_L32(49) P2_CASE_L32(50) P2_CASE_L32(51)
		P2_CASE_L32(52) P2_CASE_L32(53) P2_CASE_L32(54) P2_CASE_L32(55)
		P2_CASE_L32(56) P2_CASE_L32(57) P2_CASE_L32(58) P2_CASE_L32(59)
		P2_CASE_L32(60) P2_CASE_L32(61) P2_CASE_L32(62) P2_CASE_L32(63)
	default:
		break;
	}
}
#undef P2_CASE_L32

/* Resident blocks per SM the FP32-arithmetic kernel is built for
 * (2^M FP32 complex values take 2^(M+1) registers per thread). */
__host__ __device__ constexpr int p2_lift32_blocks(int m)
{
	return m >= 5 ? 5 : (m == 4 ? 6 : 8);
}

/* A lifted record repacked for the FP32 kernels' shared memory. */
__device__ __forceinline__ struct p2_lift32_rec p2_lift32_of(
	const struct phase2_rot_rec &in)
{
	struct p2_lift32_rec o;
	o.t = (float)in.c;
	o.s = (float)in.s; /* an FP32 value: exact */
	o.z = in.z;
	o.sm = in.smask;
	o.key = ((uint32_t)in.U << 1) | in.odd;
	return o;
}

/*
 * One coset of a lifted FP32 pass: load the 2^M amplitudes x ^ off(u)
 * into FP32 registers, apply the run of rotations, store them (negated
 * when negm has the sign bit).  CG: loads and stores at L2 only (the
 * persistent batch kernel, whose blocks read what other blocks of the same
 * launch wrote).
 */
template <int M, typename IT, bool CG>
__device__ __forceinline__ void p2_lift32_coset(float2 *__restrict__ st, IT x,
	const IT (&pb)[M > 0 ? M : 1], const struct p2_lift32_rec *srec,
	uint32_t nrot, uint32_t negm)
{
	float re[1 << M], im[1 << M];
#pragma unroll
	for (int u = 0; u < (1 << M); ++u) {
		IT off = 0;
#pragma unroll
		for (int k = 0; k < M; ++k)
			if (u >> k & 1)
				off ^= pb[k];
		const float2 v = CG ? __ldcg(st + (x ^ off)) : st[x ^ off];
		re[u] = v.x;
		im[u] = v.y;
	}
	for (uint32_t r = 0; r < nrot; ++r) {
		const struct p2_lift32_rec q = srec[r];
		const uint32_t sm = q.sm ^ (0u - p2_parity(x & (IT)q.z));
		p2_apply_lift32<M>(q, re, im, sm);
	}
	const IT xs = p2_opaque(x);
#pragma unroll
	for (int u = 0; u < (1 << M); ++u) {
		IT off = 0;
#pragma unroll
		for (int k = 0; k < M; ++k)
			if (u >> k & 1)
				off ^= pb[k];
		const float2 v = make_float2(p2_fsgn(re[u], negm),
			p2_fsgn(im[u], negm));
		if (CG)
			__stcg(st + (xs ^ off), v);
		else
			st[xs ^ off] = v;
	}
}

/*
 * One FP32 pass in the lifted form with FP32 arithmetic: loads go straight
 * into FP32 registers, the run is applied with FP32 FMAs, stores write the
 * registers back.  Half the registers of k_pass_lift (20 resident warps
 * per SM at M = 5) and no conversions.
 */
template <int M, typename IT>
__global__ void __launch_bounds__(P2_TPB, p2_lift32_blocks(M))
	k_pass_lift32(float2 *__restrict__ st, uint64_t nrep,
		struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs)
{
	__shared__ struct p2_lift32_rec srec[P2_MAX_ROTS_PER_PASS];
	for (uint32_t r = threadIdx.x; r < p.nrot; r += blockDim.x)
		srec[r] = p2_lift32_of(recs[p.rot_off + r]);
	__syncthreads();
	IT pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = (IT)p.basis[k];
	const uint32_t negm = p.scale < 0 ? 0x80000000u : 0u;
	const uint32_t nrot = p.nrot;

	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		t < nrep; t += stride)
		p2_lift32_coset<M, IT, false>(st, p2_rep_t<M, IT>((IT)t, p),
			pb, srec, nrot, negm);
}

/* ---- sweeps: several FP32 passes per HBM round trip ---------------------- */

/*
 * A sweep is a run of consecutive passes of one plan whose bases, taken
 * modulo the low L qubits, span a subspace S of rank k with k + L <= the
 * tile width (the planner marks its first pass).  The register splits into
 * tiles R + S + low: 2^k chunks of 2^L contiguous amplitudes, closed under
 * every pass of the sweep.  One block takes a tile at a time: the first
 * pass reads its cosets from HBM, the middle passes work in a
 * shared-memory copy of the tile, the last pass writes back, so the sweep
 * costs one read and one write of the state instead of one per pass.
 *
 * Tile coordinates: amplitude R ^ S(j) ^ l has coordinate (j << L) | l
 * and sits at tile[p2_swz(coordinate)], S(j) the xor of the (reduced,
 * pivots ascending) basis vectors of S selected by j.  For b in S + low,
 * vidx(b) = (b & lowmask) | (bit spiv_i of b) << (L + i) is linear, so a
 * coset x ^ span(pb) of a pass sits at vidx(x ^ R) ^ span(vb) with
 * vb = vidx(pb).  Each pass enumerates its cosets of the tile by virtual
 * representatives (zeros at the virtual pivots vpiv), then moves to the
 * coset's canonical representative, the one with zeros at the physical
 * pivots (row-reduced basis e, virtual images ve), which is the
 * representative the one-pass kernel gives the coset.  Loads, rotations,
 * signs and stores of a coset are then exactly those of k_pass_lift32, so
 * the results are bit-identical to one kernel per pass.
 */
#define P2_SW_MAXPASS 12
#define P2_SW_MAXK 9
#define P2_SW_MAXREC 1024
#define P2_SW_TPB 256
#define P2_SW_MAXTILE 14

struct p2_spass {
	uint32_t span, nrot, rec_off, negm;
	uint32_t pb[PHASE2_MAX_SPAN]; /* physical basis (slot order) */
	uint32_t vb[PHASE2_MAX_SPAN]; /* its tile coordinates */
	uint32_t e[PHASE2_MAX_SPAN];  /* row-reduced basis, pivots piv */
	uint32_t ve[PHASE2_MAX_SPAN]; /* its tile coordinates */
	uint8_t piv[PHASE2_MAX_SPAN], vpiv[PHASE2_MAX_SPAN], pad[2];
};

struct p2_sweep {
	uint32_t np, k, L, rec0, nrec;
	uint32_t sb[P2_SW_MAXK]; /* basis of S: reduced, pivots ascending */
	uint8_t spiv[P2_SW_MAXK], pad[3];
	struct p2_spass p[P2_SW_MAXPASS];
};

/* Shared-memory position of tile coordinate v: bits 0-3 xor the other
 * nibbles, so lanes whose coordinates differ in four distinct nibble
 * positions hit distinct bank pairs (8-byte elements).  Linear and
 * invertible on [0, 2^tile), so offsets can be swizzled on their own. */
__host__ __device__ __forceinline__ uint32_t p2_swz(uint32_t v)
{
	return v ^ (((v >> 4) ^ (v >> 8) ^ (v >> 12)) & 15u);
}

template <int M>
__device__ __forceinline__ void p2_sweep_pass(float2 *__restrict__ st,
	float2 *tile, const struct p2_spass &P, uint32_t R,
	const uint32_t *Stab, uint32_t L, uint32_t tl,
	const struct p2_lift32_rec *srec, bool from_g, bool to_g)
{
	uint32_t pb[M > 0 ? M : 1], vb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k) {
		pb[k] = P.pb[k];
		vb[k] = p2_swz(P.vb[k]);
	}
	const uint32_t lowm = (1u << L) - 1;
	const uint32_t nc = 1u << (tl - M);
	const uint32_t nrot = P.nrot;
	for (uint32_t c = threadIdx.x; c < nc; c += blockDim.x) {
		uint32_t vx = c;
#pragma unroll
		for (int k = 0; k < M; ++k) {
			const uint32_t q = P.vpiv[k];
			vx = ((vx >> q) << (q + 1)) | (vx & ((1u << q) - 1));
		}
		const uint32_t xv = R ^ Stab[vx >> L] ^ (vx & lowm);
		uint32_t x = xv;
#pragma unroll
		for (int k = 0; k < M; ++k)
			if (xv >> P.piv[k] & 1) {
				x ^= P.e[k];
				vx ^= P.ve[k];
			}
		const uint32_t sx = p2_swz(vx);
		float re[1 << M], im[1 << M];
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			uint32_t off = 0, voff = 0;
#pragma unroll
			for (int k = 0; k < M; ++k)
				if (u >> k & 1) {
					off ^= pb[k];
					voff ^= vb[k];
				}
			const float2 v = from_g ? st[x ^ off] : tile[sx ^ voff];
			re[u] = v.x;
			im[u] = v.y;
		}
		for (uint32_t r = 0; r < nrot; ++r) {
			const struct p2_lift32_rec q = srec[P.rec_off + r];
			const uint32_t sm = q.sm ^ (0u - p2_parity(x & (uint32_t)q.z));
			p2_apply_lift32<M>(q, re, im, sm);
		}
		const uint32_t xs = (uint32_t)p2_opaque(x);
		const uint32_t sxs = (uint32_t)p2_opaque(sx);
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			uint32_t off = 0, voff = 0;
#pragma unroll
			for (int k = 0; k < M; ++k)
				if (u >> k & 1) {
					off ^= pb[k];
					voff ^= vb[k];
				}
			const float2 v = make_float2(p2_fsgn(re[u], P.negm),
				p2_fsgn(im[u], P.negm));
			if (to_g)
				st[xs ^ off] = v;
			else
				tile[sxs ^ voff] = v;
		}
	}
}

__global__ void __launch_bounds__(P2_SW_TPB, 2)
	k_sweep32(float2 *__restrict__ st,
		const __grid_constant__ struct p2_sweep sw,
		const struct phase2_rot_rec *__restrict__ recs, uint32_t ntiles)
{
	extern __shared__ __align__(16) unsigned char sm[];
	const uint32_t L = sw.L, tl = sw.k + sw.L;
	float2 *tile = (float2 *)sm;
	struct p2_lift32_rec *srec =
		(struct p2_lift32_rec *)(tile + ((size_t)1 << tl));
	uint32_t *Stab = (uint32_t *)(srec + sw.nrec);
	for (uint32_t r = threadIdx.x; r < sw.nrec; r += blockDim.x)
		srec[r] = p2_lift32_of(recs[sw.rec0 + r]);
	for (uint32_t j = threadIdx.x; j < (1u << sw.k); j += blockDim.x) {
		uint32_t v = 0;
		for (uint32_t i = 0; i < sw.k; ++i)
			if (j >> i & 1)
				v ^= sw.sb[i];
		Stab[j] = v;
	}
	__syncthreads();
	for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
		uint32_t R = t << L;
		for (uint32_t i = 0; i < sw.k; ++i) {
			const uint32_t q = sw.spiv[i];
			R = ((R >> q) << (q + 1)) | (R & ((1u << q) - 1));
		}
		for (uint32_t q = 0; q < sw.np; ++q) {
			const struct p2_spass &P = sw.p[q];
			const bool from_g = q == 0, to_g = q + 1 == sw.np;
			switch (P.span) {
			case 0:
				p2_sweep_pass<0>(st, tile, P, R, Stab, L, tl, srec,
					from_g, to_g);
				break;
			case 1:
				p2_sweep_pass<1>(st, tile, P, R, Stab, L, tl, srec,
					from_g, to_g);
				break;
			case 2:
				p2_sweep_pass<2>(st, tile, P, R, Stab, L, tl, srec,
					from_g, to_g);
				break;
			case 3:
				p2_sweep_pass<3>(st, tile, P, R, Stab, L, tl, srec,
					from_g, to_g);
				break;
			case 4:
				p2_sweep_pass<4>(st, tile, P, R, Stab, L, tl, srec,
					from_g, to_g);
				break;
			default:
				p2_sweep_pass<5>(st, tile, P, R, Stab, L, tl, srec,
					from_g, to_g);
				break;
			}
			__syncthreads();
		}
	}
}

/* ---- persistent batch kernel -------------------------------------------- */

/*
 * Many registers' recorded programs (p2_internal.h) in one launch.  Every
 * op of a program is cut into tiles (a pass: 128 cosets, one per thread;
 * a zero: 4096 amplitudes; a write or gather: one tile); op k+1 of a
 * program starts only when every tile of op k is done, programs are
 * independent.  Each program has a ticket, (op << 32) | next tile: a block
 * claims a tile with one atomicAdd, and the block that completes the last
 * tile of an op publishes the next op by resetting the ticket.  Blocks
 * look for work across programs starting from the last one they served,
 * so small programs interleave and the GPU stays busy without a launch per
 * pass.  Waiting is bounded: a block that finds nothing to claim while no
 * ticket moves for idle_limit consecutive rounds (about a microsecond
 * each; a ticket moves whenever any tile is claimed or any op is
 * published) raises status and returns, so a scheduling fault ends the
 * launch instead of hanging it, while long single-program runs, where most
 * blocks wait on one op at a time, keep going.
 *
 * Ordering: a tile's stores are made visible (each thread fences, then the
 * block barrier) before its completion count; the finisher fences before
 * publishing the next op; a claimer fences after its claim.  State loads
 * and stores go through L2 only (ld/st .cg), since L1 is not coherent
 * across SMs.
 */
/* Cosets per thread in a pass tile: 4 for passes of at least
 * P2_BATCH_BIG_PASS representatives, 1 below (more tiles for small
 * registers, whose passes are otherwise too few tiles to spread). */
#define P2_BATCH_COSETS 4
#define P2_BATCH_BIG_PASS (UINT64_C(1) << 16)
#define P2_BATCH_ZERO_TILE (P2_TPB * 128)

struct p2_binst {
	void *state; /* float2 (FP32) or double2 (FP64) amplitudes */
	uint64_t namp;
	uint32_t op_off, nops;
};

/* Work tiles of an op on a register of namp amplitudes; for a pass of
 * span `span` also the cosets per thread of a tile (*b). */
__host__ __device__ __forceinline__ uint32_t p2_op_tiles(uint32_t kind,
	uint64_t namp, uint32_t span, uint32_t *b)
{
	if (kind == P2_OP_PASS) {
		const uint64_t nrep = namp >> span;
		*b = nrep >= P2_BATCH_BIG_PASS ? P2_BATCH_COSETS : 1;
		const uint64_t per = (uint64_t)*b * P2_TPB;
		return (uint32_t)((nrep + per - 1) / per);
	}
	if (kind == P2_OP_ZERO)
		return (uint32_t)((namp + P2_BATCH_ZERO_TILE - 1) /
			P2_BATCH_ZERO_TILE);
	return 1;
}

struct p2_bctl {
	unsigned long long ticket;
	unsigned int done;
	unsigned int pad;
};

/* The cosets of one pass tile: thread k takes representatives
 * tile * cpt * P2_TPB + j * P2_TPB + k, j < cpt (coalesced per j). */
template <int M>
__device__ __forceinline__ void p2_batch_pass_tile(float2 *st,
	const struct phase2_pass &p, uint32_t tile, uint64_t nrep, uint32_t cpt,
	const struct p2_lift32_rec *srec)
{
	uint32_t pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = (uint32_t)p.basis[k];
	const uint32_t negm = p.scale < 0 ? 0x80000000u : 0u;
	const uint64_t t0 = (uint64_t)tile * cpt * P2_TPB + threadIdx.x;
	for (uint32_t j = 0; j < cpt; ++j) {
		const uint64_t t = t0 + (uint64_t)j * P2_TPB;
		if (t < nrep)
			p2_lift32_coset<M, uint32_t, true>(st,
				p2_rep_t<M, uint32_t>((uint32_t)t, p), pb, srec,
				p.nrot, negm);
	}
}

/* The same for an FP64 register: the exact per-coset arithmetic of
 * k_pass (p2_apply_run), loads and stores at L2 only. */
template <int M>
__device__ __forceinline__ void p2_batch_pass_tile64(double2 *st,
	const struct phase2_pass &p, uint32_t tile, uint64_t nrep, uint32_t cpt,
	const struct phase2_rot_rec *srec)
{
	uint64_t pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = p.basis[k];
	const uint64_t t0 = (uint64_t)tile * cpt * P2_TPB + threadIdx.x;
	for (uint32_t j = 0; j < cpt; ++j) {
		const uint64_t t = t0 + (uint64_t)j * P2_TPB;
		if (t >= nrep)
			continue;
		const uint64_t x = p2_rep<M>(t, p);
		double re[1 << M], im[1 << M];
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			const double2 v = __ldcg(st + (x ^ p2_slot_off<M>(u, pb)));
			re[u] = v.x;
			im[u] = v.y;
		}
		p2_apply_run<M>(re, im, x, srec, p.nrot);
		const uint64_t xs = p2_opaque(x);
#pragma unroll
		for (int u = 0; u < (1 << M); ++u)
			__stcg(st + (xs ^ p2_slot_off<M>(u, pb)),
				make_double2(re[u], im[u]));
	}
}

/* Records as a batch kernel of state type ST holds them in shared
 * memory: repacked lifted records (FP32) or the records themselves
 * (FP64). */
template <typename ST> struct p2_brec;
template <> struct p2_brec<float2> {
	typedef struct p2_lift32_rec type;
	static __device__ __forceinline__ type of(const phase2_rot_rec &r)
	{
		return p2_lift32_of(r);
	}
};
template <> struct p2_brec<double2> {
	typedef struct phase2_rot_rec type;
	static __device__ __forceinline__ type of(const phase2_rot_rec &r)
	{
		return r;
	}
};

template <typename ST>
__global__ void __launch_bounds__(P2_TPB, sizeof(ST) == 8 ? 5 : 2)
	k_batch(const struct p2_binst *__restrict__ inst, uint32_t ninst,
		const struct p2_op *__restrict__ ops,
		const struct phase2_pass *__restrict__ passes,
		const struct phase2_rot_rec *__restrict__ recs,
		const uint64_t *__restrict__ widx,
		const double *__restrict__ wval,
		const uint64_t *__restrict__ gidx, double2 *__restrict__ gout,
		struct p2_bctl *ctl, unsigned int *status,
		unsigned int idle_limit)
{
	constexpr bool F64 = sizeof(ST) == 16;
	typedef typename p2_brec<ST>::type RT;
	__shared__ RT srec[P2_MAX_ROTS_PER_PASS];
	__shared__ uint32_t s_inst, s_seq, s_tile;
	__shared__ int s_what; /* 0 nothing claimable yet, 1 work, 2 exit */
	/* pass whose records srec holds (block-uniform), none at first */
	uint32_t held = 0xffffffffu;
	uint32_t cursor = blockIdx.x % ninst;
	unsigned int idle = 0;
	unsigned long long seen = 0; /* tickets at the last idle round */
	for (;;) {
		if (threadIdx.x == 0) {
			int what = 2;
			unsigned long long sig = 0;
			for (uint32_t k = 0; k < ninst; ++k) {
				const uint32_t i = cursor + k < ninst
					? cursor + k
					: cursor + k - ninst;
				const uint32_t nops = inst[i].nops;
				const unsigned long long tk =
					*(volatile unsigned long long *)&ctl[i]
						 .ticket;
				sig += tk * (2ull * i + 1ull);
				if ((uint32_t)(tk >> 32) >= nops)
					continue; /* program finished */
				what = 0;
				const uint32_t off = inst[i].op_off;
				if ((uint32_t)tk >=
					ops[off + (uint32_t)(tk >> 32)].ntiles)
					continue; /* all tiles taken */
				const unsigned long long got =
					atomicAdd(&ctl[i].ticket, 1ull);
				const uint32_t seq = (uint32_t)(got >> 32);
				const uint32_t tile = (uint32_t)got;
				if (seq < nops && tile < ops[off + seq].ntiles) {
					__threadfence();
					s_inst = i;
					s_seq = seq;
					s_tile = tile;
					cursor = i;
					what = 1;
					break;
				}
			}
			if (what == 0) {
				if (sig != seen) {
					seen = sig;
					idle = 0;
				}
				if (++idle > idle_limit) {
					atomicOr(status, 1u);
					what = 2;
				} else {
					__nanosleep(1000);
				}
			} else if (what == 1) {
				idle = 0;
			}
			s_what = what;
		}
		__syncthreads();
		const int what = s_what;
		if (what == 2)
			return;
		if (what == 1) {
			const uint32_t i = s_inst, seq = s_seq, tile = s_tile;
			ST *const st = (ST *)inst[i].state;
			const uint64_t namp = inst[i].namp;
			const struct p2_op op = ops[inst[i].op_off + seq];
			if (op.kind == P2_OP_PASS) {
				const struct phase2_pass p = passes[op.a];
				/* consecutive tiles of one pass (a Trotter step
				 * replays the same passes) keep their records */
				if (held != op.a) {
					for (uint32_t r = threadIdx.x; r < p.nrot;
						r += blockDim.x)
						srec[r] = p2_brec<ST>::of(
							recs[p.rot_off + r]);
					held = op.a;
					__syncthreads();
				}
				const uint64_t nrep = namp >> p.span;
				if constexpr (F64) {
					switch (p.span) {
					case 0:
						p2_batch_pass_tile64<0>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 1:
						p2_batch_pass_tile64<1>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 2:
						p2_batch_pass_tile64<2>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 3:
						p2_batch_pass_tile64<3>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 4:
						p2_batch_pass_tile64<4>(st, p, tile,
							nrep, op.b, srec);
						break;
					default:
						p2_batch_pass_tile64<5>(st, p, tile,
							nrep, op.b, srec);
						break;
					}
				} else {
					switch (p.span) {
					case 0:
						p2_batch_pass_tile<0>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 1:
						p2_batch_pass_tile<1>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 2:
						p2_batch_pass_tile<2>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 3:
						p2_batch_pass_tile<3>(st, p, tile,
							nrep, op.b, srec);
						break;
					case 4:
						p2_batch_pass_tile<4>(st, p, tile,
							nrep, op.b, srec);
						break;
					default:
						p2_batch_pass_tile<5>(st, p, tile,
							nrep, op.b, srec);
						break;
					}
				}
			} else if (op.kind == P2_OP_ZERO) {
				const uint64_t base =
					(uint64_t)tile * P2_BATCH_ZERO_TILE;
				ST zero;
				zero.x = 0;
				zero.y = 0;
				for (uint32_t k = threadIdx.x;
					k < P2_BATCH_ZERO_TILE; k += blockDim.x)
					if (base + k < namp)
						__stcg(st + base + k, zero);
			} else if (op.kind == P2_OP_WRITE) {
				/* in order: later writes win */
				if (threadIdx.x == 0)
					for (uint32_t e = op.a; e < op.a + op.b; ++e) {
						ST v;
						if constexpr (F64) {
							v.x = wval[2 * e];
							v.y = wval[2 * e + 1];
						} else {
							v.x = (float)wval[2 * e];
							v.y = (float)wval[2 * e + 1];
						}
						__stcg(st + widx[e], v);
					}
			} else {
				for (uint32_t d = threadIdx.x; d < op.b;
					d += blockDim.x) {
					const ST v = __ldcg(st + gidx[op.a + d]);
					gout[op.a + d] = make_double2(v.x, v.y);
				}
			}
			__threadfence();
			__syncthreads();
			if (threadIdx.x == 0) {
				const unsigned int d =
					atomicAdd(&ctl[i].done, 1u) + 1u;
				if (d == op.ntiles) {
					atomicExch(&ctl[i].done, 0u);
					__threadfence();
					atomicExch(&ctl[i].ticket,
						(unsigned long long)(seq + 1) << 32);
				}
			}
		}
		__syncthreads();
	}
}

/* ---- small kernels ------------------------------------------------------ */

template <typename ST>
__global__ void k_gather(const ST *__restrict__ st,
	const uint64_t *__restrict__ idx, double *__restrict__ out, size_t n)
{
	const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
	if (i < n) {
		double re, im;
		p2_ld(st, idx[i], re, im);
		out[2 * i] = re;
		out[2 * i + 1] = im;
	}
}

/* Later entries win on duplicate indices: one thread writes them all in
 * order (n is small: determinants of a state-prep payload). */
template <typename ST>
__global__ void k_scatter(ST *__restrict__ st, const uint64_t *__restrict__ idx,
	const double *__restrict__ val, size_t n)
{
	if (blockIdx.x == 0 && threadIdx.x == 0)
		for (size_t i = 0; i < n; ++i)
			p2_st(st, idx[i], val[2 * i], val[2 * i + 1]);
}

/* Neumaier: s + c carries the running sum and its rounding error. */
__device__ __forceinline__ void p2_neumaier(double &s, double &c, double v)
{
	const double t = s + v;
	if (fabs(s) >= fabs(v))
		c += (s - t) + v;
	else
		c += (v - t) + s;
	s = t;
}

__device__ __forceinline__ double p2_warp_sum(double v)
{
#pragma unroll
	for (int o = 16; o > 0; o >>= 1)
		v += __shfl_xor_sync(0xffffffffu, v, o);
	return v;
}

/* A block's two compensated per-thread sums -> part[2*block + {0,1}]:
 * warp-shuffle tree, then one pass over the warp totals in shared memory. */
__device__ __forceinline__ void p2_block_sum2(double vr, double vi,
	double *__restrict__ part)
{
	vr = p2_warp_sum(vr);
	vi = p2_warp_sum(vi);
	__shared__ double wr[P2_RED_TPB / 32], wi[P2_RED_TPB / 32];
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	if (lane == 0) {
		wr[warp] = vr;
		wi[warp] = vi;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
		for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
			p2_neumaier(s0, c0, wr[w]);
			p2_neumaier(s1, c1, wi[w]);
		}
		part[2 * blockIdx.x] = s0 + c0;
		part[2 * blockIdx.x + 1] = s1 + c1;
	}
}

/* Stage 1: per-block sums of |a|^2 (trial == NULL) or of conj(trial) * a,
 * written to part[2*block + {0,1}].  Each thread accumulates its strided
 * elements with compensation, then a warp-shuffle tree and one pass over
 * the warp totals in shared memory. */
template <typename ST>
__global__ void __launch_bounds__(P2_RED_TPB) k_reduce_partial(
	const ST *__restrict__ st, const double2 *__restrict__ trial, uint64_t n,
	double *__restrict__ part)
{
	double sr = 0.0, cr = 0.0, si = 0.0, ci = 0.0;
	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		i < n; i += stride) {
		double re, im;
		p2_ld(st, i, re, im);
		if (trial) {
			const double2 t = trial[i];
			p2_neumaier(sr, cr, t.x * re + t.y * im);
			p2_neumaier(si, ci, t.x * im - t.y * re);
		} else {
			p2_neumaier(sr, cr, re * re + im * im);
		}
	}
	p2_block_sum2(sr + cr, si + ci, part);
}

/* ---- coefficient-matrix trial states (state_prep.c) --------------------- */

/* Index of an (alpha | beta) occupation: tapered drops bits 0 and n_sites
 * and compacts the rest (reference: state_prep_coeff.c:47-54). */
__device__ __forceinline__ uint64_t p2_cm_index(uint64_t full,
	uint32_t n_sites, int tapered)
{
	if (!tapered)
		return full;
	const uint64_t lo =
		(full >> 1) & ((UINT64_C(1) << (n_sites - 1)) - 1);
	return lo | ((full >> (n_sites + 1)) << (n_sites - 1));
}

/* Slater-Condon expansion: for pair (i, j) every block k whose
 * c = (w_k * det_a_k[i]) * det_b_k[j] is not below 1e-12 in magnitude is
 * added, in block order, to the amplitude (accumulate) or to a first
 * assignment; products and sums rounded separately, as the reference's
 * host loop (state_prep_coeff.c:171-193).  Distinct pairs have distinct
 * indices (fixed particle numbers), so no two threads write one
 * amplitude. */
template <typename ST>
__global__ void k_cm_expand(ST *__restrict__ st,
	const uint64_t *__restrict__ occ_a, const uint64_t *__restrict__ occ_b,
	uint64_t Ma, uint64_t Mb, const double *__restrict__ w,
	const double *__restrict__ det_a, const double *__restrict__ det_b,
	uint32_t ncomp, uint32_t n_sites, int tapered, int accumulate)
{
	const uint64_t n = Ma * Mb;
	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		p < n; p += stride) {
		const uint64_t i = p / Mb, j = p - i * Mb;
		const uint64_t idx =
			p2_cm_index(occ_a[i] | occ_b[j], n_sites, tapered);
		double re = 0.0, im = 0.0;
		bool hit = false;
		for (uint32_t k = 0; k < ncomp; ++k) {
			const double cf = __dmul_rn(
				__dmul_rn(w[k], det_a[k * Ma + i]),
				det_b[k * Mb + j]);
			if (fabs(cf) < 1.0e-12)
				continue;
			if (!hit) {
				hit = true;
				if (accumulate) {
					p2_ld(st, idx, re, im);
					re = __dadd_rn(re, cf);
				} else {
					re = cf;
				}
			} else {
				re = __dadd_rn(re, cf);
			}
		}
		if (hit)
			p2_st(st, idx, re, im);
	}
}

/* Overlap of the real trial state with the register: per-block partial
 * sums of c * a[idx] over the pairs (compensated), then k_reduce_final. */
template <typename ST>
__global__ void __launch_bounds__(P2_RED_TPB) k_cm_inner(
	const ST *__restrict__ st, const uint64_t *__restrict__ occ_a,
	const uint64_t *__restrict__ occ_b, uint64_t Ma, uint64_t Mb, double w,
	const double *__restrict__ det_a, const double *__restrict__ det_b,
	uint32_t n_sites, int tapered, double *__restrict__ part)
{
	double sr = 0.0, cr = 0.0, si = 0.0, ci = 0.0;
	const uint64_t n = Ma * Mb;
	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		p < n; p += stride) {
		const uint64_t i = p / Mb, j = p - i * Mb;
		const double cf = __dmul_rn(__dmul_rn(w, det_a[i]), det_b[j]);
		if (fabs(cf) < 1.0e-12)
			continue;
		double re, im;
		p2_ld(st, p2_cm_index(occ_a[i] | occ_b[j], n_sites, tapered),
			re, im);
		p2_neumaier(sr, cr, __dmul_rn(cf, re));
		p2_neumaier(si, ci, __dmul_rn(cf, im));
	}
	p2_block_sum2(sr + cr, si + ci, part);
}

/* Stage 2: one block combines nblk partials (compensated). */
__global__ void __launch_bounds__(P2_RED_TPB) k_reduce_final(
	const double *__restrict__ part, uint32_t nblk, double *__restrict__ out)
{
	double sr = 0.0, cr = 0.0, si = 0.0, ci = 0.0;
	for (uint32_t b = threadIdx.x; b < nblk; b += blockDim.x) {
		p2_neumaier(sr, cr, part[2 * b]);
		p2_neumaier(si, ci, part[2 * b + 1]);
	}
	__shared__ double a0[P2_RED_TPB], a1[P2_RED_TPB];
	a0[threadIdx.x] = sr + cr;
	a1[threadIdx.x] = si + ci;
	__syncthreads();
	if (threadIdx.x == 0) {
		double s0 = 0.0, c0 = 0.0, s1 = 0.0, c1 = 0.0;
		for (int t = 0; t < (int)blockDim.x; ++t) {
			p2_neumaier(s0, c0, a0[t]);
			p2_neumaier(s1, c1, a1[t]);
		}
		out[0] = s0 + c0;
		out[1] = s1 + c1;
	}
}

/* ---- host side ---------------------------------------------------------- */

extern "C" int p2d_device_init(int dev, int *count)
{
	int n = 0;
	const cudaError_t e = cudaGetDeviceCount(&n);
	if (count)
		*count = e == cudaSuccess ? n : 0;
	if (e != cudaSuccess || n == 0) {
		log_error("no CUDA device: %s",
			e == cudaSuccess ? "device count is 0"
					 : cudaGetErrorString(e));
		return -1;
	}
	if (dev < 0 || dev >= n) {
		log_error("CUDA device %d out of range (count %d)", dev, n);
		return -1;
	}
	CUDA_OK(cudaSetDevice(dev), "cudaSetDevice");
	CUDA_OK(cudaFree(0), "CUDA context init");
	return 0;
}

static int io_reserve(struct p2_dev *d, size_t n)
{
	if (n <= d->io_cap)
		return 0;
	size_t cap = d->io_cap ? d->io_cap : 64;
	while (cap < n)
		cap *= 2;
	CUDA_OK(cudaStreamSynchronize(d->stream), "sync before io growth");
	cudaFree(d->d_idx);
	cudaFree(d->d_val);
	cudaFreeHost(d->h_idx);
	cudaFreeHost(d->h_val);
	d->d_idx = NULL;
	d->d_val = NULL;
	d->h_idx = NULL;
	d->h_val = NULL;
	d->io_cap = 0;
	CUDA_OK(cudaMalloc((void **)&d->d_idx, cap * sizeof(uint64_t)),
		"alloc idx");
	CUDA_OK(cudaMalloc((void **)&d->d_val, cap * 2 * sizeof(double)),
		"alloc val");
	CUDA_OK(cudaMallocHost((void **)&d->h_idx, cap * sizeof(uint64_t)),
		"alloc pinned idx");
	CUDA_OK(cudaMallocHost((void **)&d->h_val, cap * 2 * sizeof(double)),
		"alloc pinned val");
	d->io_cap = cap;
	return 0;
}

extern "C" struct p2_dev *p2d_create(uint32_t nqb, int prec)
{
	if (nqb == 0 || nqb > 40) {
		log_error("p2d_create: nqb=%u out of range", nqb);
		return NULL;
	}
	if (prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32) {
		log_error("p2d_create: unknown precision %d", prec);
		return NULL;
	}
	struct p2_dev *d = (struct p2_dev *)calloc(1, sizeof *d);
	if (!d)
		return NULL;
	d->nqb = nqb;
	d->prec = prec;
	d->elem = prec == PHASE2_PREC_FP64 ? sizeof(double2) : sizeof(float2);
	d->namp = UINT64_C(1) << nqb;
	const size_t bytes = d->namp * d->elem;

	int dev = 0;
	cudaGetDevice(&dev);
	cudaDeviceGetAttribute(&d->sm_count, cudaDevAttrMultiProcessorCount,
		dev);
	if (d->sm_count <= 0)
		d->sm_count = 148;
	d->graphs_on = nqb <= P2_GRAPH_MAX_QB;

	size_t free_b = 0, total_b = 0;
	if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
		bytes > free_b) {
		log_error("p2d_create: state of %zu bytes exceeds free device"
			  " memory (%zu bytes)",
			bytes, free_b);
		free(d);
		return NULL;
	}
	if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) !=
		cudaSuccess)
		goto fail;
	if (cudaMalloc(&d->state, bytes) != cudaSuccess) {
		log_error("p2d_create: cudaMalloc(%zu) failed", bytes);
		goto fail;
	}
	for (int k = 0; k < 2; k++)
		if (cudaEventCreateWithFlags(&d->h_ev[k],
			    cudaEventDisableTiming) != cudaSuccess)
			goto fail;
	if (cudaEventCreate(&d->t0) != cudaSuccess ||
		cudaEventCreate(&d->t1) != cudaSuccess)
		goto fail;
	if (cudaMemsetAsync(d->state, 0, bytes, d->stream) != cudaSuccess)
		goto fail;
	return d;
fail:
	log_error("p2d_create: %s", cudaGetErrorString(cudaGetLastError()));
	p2d_destroy(d);
	return NULL;
}

extern "C" void p2d_destroy(struct p2_dev *d)
{
	if (!d)
		return;
	if (d->stream)
		cudaStreamSynchronize(d->stream);
	cudaFree(d->state);
	cudaFree(d->d_recs);
	for (int k = 0; k < 2; k++) {
		cudaFreeHost(d->h_recs[k]);
		if (d->h_ev[k])
			cudaEventDestroy(d->h_ev[k]);
	}
	cudaFree(d->d_idx);
	cudaFree(d->d_val);
	cudaFreeHost(d->h_idx);
	cudaFreeHost(d->h_val);
	cudaFree(d->d_part);
	cudaFree(d->d_cm);
	for (int k = 0; k < P2_GRAPH_SLOTS; k++) {
		struct p2_graph *g = &d->graphs[k];
		if (g->exec)
			cudaGraphExecDestroy(g->exec);
		cudaFree(g->d_recs);
		free(g->passes);
		free(g->recs);
	}
	if (d->t0)
		cudaEventDestroy(d->t0);
	if (d->t1)
		cudaEventDestroy(d->t1);
	if (d->stream)
		cudaStreamDestroy(d->stream);
	free(d);
}

extern "C" int p2d_zero(struct p2_dev *d)
{
	CUDA_OK(cudaMemsetAsync(d->state, 0, d->namp * d->elem, d->stream),
		"zero state");
	return 0;
}

static int check_idx(const struct p2_dev *d, const uint64_t *idx, size_t n)
{
	for (size_t i = 0; i < n; i++)
		if (idx[i] >= d->namp) {
			log_error("amplitude index %llu out of range (namp %llu)",
				(unsigned long long)idx[i],
				(unsigned long long)d->namp);
			return -1;
		}
	return 0;
}

extern "C" int p2d_set(struct p2_dev *d, const uint64_t *idx, const double *z,
	size_t n)
{
	if (n == 0)
		return 0;
	if (check_idx(d, idx, n) < 0 || io_reserve(d, n) < 0)
		return -1;
	CUDA_OK(cudaStreamSynchronize(d->stream), "sync before set");
	memcpy(d->h_idx, idx, n * sizeof *idx);
	memcpy(d->h_val, z, n * 2 * sizeof(double));
	CUDA_OK(cudaMemcpyAsync(d->d_idx, d->h_idx, n * sizeof *idx,
			cudaMemcpyHostToDevice, d->stream),
		"upload idx");
	CUDA_OK(cudaMemcpyAsync(d->d_val, d->h_val, n * 2 * sizeof(double),
			cudaMemcpyHostToDevice, d->stream),
		"upload val");
	d->h2d_bytes += n * (sizeof(uint64_t) + 2 * sizeof(double));
	if (d->prec == PHASE2_PREC_FP64)
		k_scatter<<<1, 32, 0, d->stream>>>((double2 *)d->state, d->d_idx,
			d->d_val, n);
	else
		k_scatter<<<1, 32, 0, d->stream>>>((float2 *)d->state, d->d_idx,
			d->d_val, n);
	d->launches++;
	CUDA_OK(cudaGetLastError(), "scatter launch");
	CUDA_OK(cudaStreamSynchronize(d->stream), "scatter");
	return 0;
}

extern "C" int p2d_get(struct p2_dev *d, const uint64_t *idx, double *z,
	size_t n)
{
	if (n == 0)
		return 0;
	if (check_idx(d, idx, n) < 0 || io_reserve(d, n) < 0)
		return -1;
	CUDA_OK(cudaStreamSynchronize(d->stream), "sync before get");
	memcpy(d->h_idx, idx, n * sizeof *idx);
	CUDA_OK(cudaMemcpyAsync(d->d_idx, d->h_idx, n * sizeof *idx,
			cudaMemcpyHostToDevice, d->stream),
		"upload idx");
	const unsigned blocks = (unsigned)((n + 127) / 128);
	if (d->prec == PHASE2_PREC_FP64)
		k_gather<<<blocks, 128, 0, d->stream>>>(
			(const double2 *)d->state, d->d_idx, d->d_val, n);
	else
		k_gather<<<blocks, 128, 0, d->stream>>>(
			(const float2 *)d->state, d->d_idx, d->d_val, n);
	d->launches++;
	CUDA_OK(cudaGetLastError(), "gather launch");
	CUDA_OK(cudaMemcpyAsync(d->h_val, d->d_val, n * 2 * sizeof(double),
			cudaMemcpyDeviceToHost, d->stream),
		"download val");
	d->h2d_bytes += n * sizeof(uint64_t);
	d->d2h_bytes += n * 2 * sizeof(double);
	CUDA_OK(cudaStreamSynchronize(d->stream), "gather");
	memcpy(z, d->h_val, n * 2 * sizeof(double));
	return 0;
}

static unsigned grid_for(const struct p2_dev *d, uint64_t work, unsigned tpb,
	unsigned per_sm)
{
	uint64_t b = (work + tpb - 1) / tpb;
	const uint64_t cap = (uint64_t)d->sm_count * per_sm;
	if (b > cap)
		b = cap;
	return b ? (unsigned)b : 1u;
}

extern "C" int p2d_get_state(struct p2_dev *d, double *out)
{
	const size_t bytes = d->namp * sizeof(double2);
	if (d->prec == PHASE2_PREC_FP64) {
		CUDA_OK(cudaMemcpyAsync(out, d->state, bytes,
				cudaMemcpyDeviceToHost, d->stream),
			"download state");
		CUDA_OK(cudaStreamSynchronize(d->stream), "download state");
		return 0;
	}
	/* FP32: download the raw complex64 values into the upper half of
	 * `out` and widen forward in place (element i is read before the
	 * 16 bytes at 16 i are written, and never overlaps a later one). */
	float *raw = (float *)((char *)out + d->namp * sizeof(float2));
	CUDA_OK(cudaMemcpyAsync(raw, d->state, d->namp * sizeof(float2),
			cudaMemcpyDeviceToHost, d->stream),
		"download state");
	CUDA_OK(cudaStreamSynchronize(d->stream), "download state");
	d->d2h_bytes += d->namp * sizeof(float2);
	for (uint64_t i = 0; i < d->namp; i++) {
		const float re = raw[2 * i], im = raw[2 * i + 1];
		out[2 * i] = (double)re;
		out[2 * i + 1] = (double)im;
	}
	(void)bytes;
	return 0;
}

extern "C" int p2d_set_state(struct p2_dev *d, const double *in)
{
	const size_t bytes = d->namp * sizeof(double2);
	CUDA_OK(cudaStreamSynchronize(d->stream), "sync before set_state");
	if (d->prec == PHASE2_PREC_FP64) {
		CUDA_OK(cudaMemcpyAsync(d->state, in, bytes,
				cudaMemcpyHostToDevice, d->stream),
			"upload state");
		CUDA_OK(cudaStreamSynchronize(d->stream), "upload state");
		return 0;
	}
	/* FP32: round to nearest on the host (as __double2float_rn), upload */
	float *raw = (float *)malloc(d->namp * sizeof(float2));
	if (!raw) {
		log_error("set_state: host buffer of %zu bytes",
			(size_t)(d->namp * sizeof(float2)));
		return -1;
	}
	for (uint64_t i = 0; i < 2 * d->namp; i++)
		raw[i] = (float)in[i];
	cudaError_t e = cudaMemcpyAsync(d->state, raw,
		d->namp * sizeof(float2), cudaMemcpyHostToDevice, d->stream);
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(d->stream);
	free(raw);
	CUDA_OK(e, "upload narrowed state");
	d->h2d_bytes += d->namp * sizeof(float2);
	(void)bytes;
	return 0;
}

/*
 * Launch table: per precision and span, which pass kernel runs and how many
 * blocks per SM the grid holds.  FP64: variant 0 direct loads, 1 shared-
 * memory prefetch (per_sm 0: 16 for the direct kernel, the occupancy for
 * the prefetch kernel).  FP32: the lifted kernels, variant 0 only (per_sm
 * 0: 16).  Set by phase2_tune_set (the autotuner) or left at these
 * defaults.
 */
struct p2_tune_entry {
	int variant;
	int per_sm;
};
static struct p2_tune_entry p2_tune[2][PHASE2_MAX_SPAN + 1] = {
	/* FP64: direct loads, 32 blocks per SM (measured 93-96 % of HBM
	 * peak for every span at 28 qubits on B200) */
	{ { 0, 32 }, { 0, 32 }, { 0, 32 }, { 0, 32 }, { 0, 32 }, { 0, 32 } },
	/* FP32: 32 blocks per SM (k_pass_lift32 at span 5: 95 % of HBM peak
	 * at 28 and 30 qubits, ahead of 16 and 8), 16 at span 1
	 * (phase2_b200/tuning_b200.json, 28 qubits) */
	{ { 0, 32 }, { 0, 16 }, { 0, 32 }, { 0, 32 }, { 0, 32 }, { 0, 32 } },
};

extern "C" int phase2_tune_set(int prec, int span, int variant, int per_sm)
{
	if ((prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32) || span < 0 ||
		span > PHASE2_MAX_SPAN || variant < 0 ||
		variant > (prec == PHASE2_PREC_FP64 ? 1 : 0) || per_sm < 0 ||
		per_sm > 64)
		return -1;
	p2_tune[prec][span].variant = variant;
	p2_tune[prec][span].per_sm = per_sm;
	return 0;
}

extern "C" int phase2_tune_get(int prec, int span, int *variant, int *per_sm)
{
	if ((prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32) || span < 0 ||
		span > PHASE2_MAX_SPAN)
		return -1;
	*variant = p2_tune[prec][span].variant;
	*per_sm = p2_tune[prec][span].per_sm;
	return 0;
}

/* Resolved configuration of the prefetch kernel (shared memory opt-in and
 * resident blocks per SM), once per instantiation. */
struct p2_kcfg {
	int ready;
	int tpb;
	size_t smem;
	int per_sm;
};

/* One FP64 pass: direct (variant 0) or prefetch (variant 1) kernel. */
template <int M>
static int launch_pass_t(struct p2_dev *d, const struct phase2_pass &p,
	const struct phase2_rot_rec *recs)
{
	const uint64_t nrep = d->namp >> M;
	const struct p2_tune_entry te = p2_tune[PHASE2_PREC_FP64][M];
	double2 *const sv = (double2 *)d->state;
	if (te.variant != 1) {
		const unsigned per_sm = te.per_sm ? (unsigned)te.per_sm : 16u;
		const unsigned grid = grid_for(d, nrep, P2_TPB, per_sm);
		k_pass<M><<<grid, P2_TPB, 0, d->stream>>>(sv, nrep, p, recs);
		return 0;
	}
	static struct p2_kcfg cfg;
	if (!cfg.ready) {
		cfg.tpb = p2_tpb(M);
		cfg.smem = 2 * ((size_t)1 << M) * cfg.tpb * sizeof(double2);
		CUDA_OK(cudaFuncSetAttribute(k_pass_pf<M>,
				cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)cfg.smem),
			"pass kernel shared memory");
		int per_sm = 0;
		CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
				k_pass_pf<M>, cfg.tpb, cfg.smem),
			"pass kernel occupancy");
		cfg.per_sm = per_sm > 0 ? per_sm : 1;
		cfg.ready = 1;
	}
	const unsigned per_sm = te.per_sm && te.per_sm < cfg.per_sm
		? (unsigned)te.per_sm
		: (unsigned)cfg.per_sm;
	const unsigned grid = grid_for(d, nrep, (unsigned)cfg.tpb, per_sm);
	k_pass_pf<M><<<grid, cfg.tpb, cfg.smem, d->stream>>>(sv, nrep, p, recs);
	return 0;
}

/* One FP32 pass in the lifted form of the pass: FP32 arithmetic
 * (k_pass_lift32) or FP64 arithmetic (k_pass_lift); 32-bit index
 * arithmetic up to 31 qubits. */
template <int M>
static int launch_lift_t(struct p2_dev *d, const struct phase2_pass &p,
	const struct phase2_rot_rec *recs)
{
	const uint64_t nrep = d->namp >> M;
	const struct p2_tune_entry te = p2_tune[PHASE2_PREC_FP32][M];
	const unsigned per_sm = te.per_sm ? (unsigned)te.per_sm : 16u;
	const unsigned grid = grid_for(d, nrep, P2_TPB, per_sm);
	float2 *const sv = (float2 *)d->state;
	const bool narrow = d->nqb <= 31;
	if (p.form == PHASE2_FORM_LIFTED_F32) {
		if (narrow)
			k_pass_lift32<M, uint32_t>
				<<<grid, P2_TPB, 0, d->stream>>>(sv, nrep, p, recs);
		else
			k_pass_lift32<M, uint64_t>
				<<<grid, P2_TPB, 0, d->stream>>>(sv, nrep, p, recs);
	} else if (p.form == PHASE2_FORM_LIFTED) {
		if (narrow)
			k_pass_lift<M, uint32_t>
				<<<grid, P2_TPB, 0, d->stream>>>(sv, nrep, p, recs);
		else
			k_pass_lift<M, uint64_t>
				<<<grid, P2_TPB, 0, d->stream>>>(sv, nrep, p, recs);
	} else {
		log_error("FP32 pass of form %u unsupported", p.form);
		return -1;
	}
	return 0;
}

static int launch_pass(struct p2_dev *d, const struct phase2_pass &p,
	const struct phase2_rot_rec *recs)
{
	const bool f64 = d->prec == PHASE2_PREC_FP64;
	switch (p.span) {
	case 0:
		return f64 ? launch_pass_t<0>(d, p, recs)
			   : launch_lift_t<0>(d, p, recs);
	case 1:
		return f64 ? launch_pass_t<1>(d, p, recs)
			   : launch_lift_t<1>(d, p, recs);
	case 2:
		return f64 ? launch_pass_t<2>(d, p, recs)
			   : launch_lift_t<2>(d, p, recs);
	case 3:
		return f64 ? launch_pass_t<3>(d, p, recs)
			   : launch_lift_t<3>(d, p, recs);
	case 4:
		return f64 ? launch_pass_t<4>(d, p, recs)
			   : launch_lift_t<4>(d, p, recs);
	case 5:
		return f64 ? launch_pass_t<5>(d, p, recs)
			   : launch_lift_t<5>(d, p, recs);
	default:
		log_error("pass span %u unsupported", p.span);
		return -1;
	}
}

static int recs_reserve(struct p2_dev *d, size_t n)
{
	if (n > d->d_recs_cap) {
		size_t cap = d->d_recs_cap ? d->d_recs_cap : 1024;
		while (cap < n)
			cap *= 2;
		CUDA_OK(cudaStreamSynchronize(d->stream), "sync before growth");
		cudaFree(d->d_recs);
		d->d_recs = NULL;
		d->d_recs_cap = 0;
		CUDA_OK(cudaMalloc((void **)&d->d_recs,
				cap * sizeof(struct phase2_rot_rec)),
			"alloc rotation records");
		d->d_recs_cap = cap;
	}
	const int k = d->ring;
	if (d->h_ev_live[k]) {
		CUDA_OK(cudaEventSynchronize(d->h_ev[k]), "staging reuse");
		d->h_ev_live[k] = 0;
	}
	if (n > d->h_recs_cap[k]) {
		size_t cap = d->h_recs_cap[k] ? d->h_recs_cap[k] : 1024;
		while (cap < n)
			cap *= 2;
		cudaFreeHost(d->h_recs[k]);
		d->h_recs[k] = NULL;
		d->h_recs_cap[k] = 0;
		CUDA_OK(cudaMallocHost((void **)&d->h_recs[k],
				cap * sizeof(struct phase2_rot_rec)),
			"alloc pinned records");
		d->h_recs_cap[k] = cap;
	}
	return 0;
}

/* Sweep shape (phase2_set_sweep): tile width and low qubits; 0 = off.
 * p2_sweep_kernel 0: planned sweeps run one kernel per pass. */
static int p2_sweep_tile = 0, p2_sweep_low = 5, p2_sweep_kernel = 1;

extern "C" int p2d_set_sweep(int tile_qubits, int low_qubits)
{
	if (tile_qubits == 0) {
		p2_sweep_tile = 0;
		if (low_qubits >= 3 && low_qubits <= 8)
			p2_sweep_low = low_qubits;
		return 0;
	}
	if (tile_qubits < 8 || tile_qubits > P2_SW_MAXTILE || low_qubits < 3 ||
		low_qubits > 8 || tile_qubits - low_qubits > P2_SW_MAXK)
		return -1;
	p2_sweep_tile = tile_qubits;
	p2_sweep_low = low_qubits;
	return 0;
}

extern "C" void p2d_get_sweep(int *tile_qubits, int *low_qubits)
{
	*tile_qubits = p2_sweep_tile;
	*low_qubits = p2_sweep_low;
}

extern "C" void p2d_set_sweep_kernel(int on)
{
	p2_sweep_kernel = on != 0;
}

/* Row-reduced basis: rows[] with pivots piv[] (each pivot bit set in its
 * row only).  Adds v when independent; returns the rank. */
static int rref_add(uint32_t *rows, int *piv, int n, uint32_t v)
{
	for (int r = 0; r < n; r++)
		if (v >> piv[r] & 1)
			v ^= rows[r];
	if (!v)
		return n;
	const int p = 31 - __builtin_clz(v);
	for (int r = 0; r < n; r++)
		if (rows[r] >> p & 1)
			rows[r] ^= v;
	rows[n] = v;
	piv[n] = p;
	return n + 1;
}

/* Sort rows by pivot, ascending. */
static void rref_sort(uint32_t *rows, int *piv, int n)
{
	for (int a = 1; a < n; a++)
		for (int b = a; b > 0 && piv[b - 1] > piv[b]; b--) {
			const uint32_t t = rows[b];
			rows[b] = rows[b - 1];
			rows[b - 1] = t;
			const int q = piv[b];
			piv[b] = piv[b - 1];
			piv[b - 1] = q;
		}
}

static uint32_t sweep_vidx(const struct p2_sweep &sw, uint32_t b)
{
	uint32_t v = b & ((1u << sw.L) - 1);
	for (uint32_t i = 0; i < sw.k; i++)
		v |= (b >> sw.spiv[i] & 1) << (sw.L + i);
	return v;
}

static uint32_t sweep_phys(const struct p2_sweep &sw, uint32_t v)
{
	uint32_t b = v & ((1u << sw.L) - 1);
	for (uint32_t i = 0; i < sw.k; i++)
		if (v >> (sw.L + i) & 1)
			b ^= sw.sb[i];
	return b;
}

/*
 * The sweep starting at passes[i]: the passes up to the next one that
 * starts a sweep (the planner's grouping, struct phase2_pass.sweep), cut
 * at P2_SW_MAXPASS passes and P2_SW_MAXREC records, and checked to fit
 * the current tile shape.  Fills *sw and returns the number of passes (1:
 * run the pass alone).
 */
static size_t sweep_from(const struct phase2_pass *passes, size_t npass,
	size_t i, struct p2_sweep *sw)
{
	const int tl = p2_sweep_tile, L = p2_sweep_low;
	const uint32_t lowm = (1u << L) - 1;
	uint32_t rows[32];
	int piv[32], n = 0;
	uint32_t nrec = 0;
	size_t j = i;
	for (; j < npass && j - i < P2_SW_MAXPASS; j++) {
		const struct phase2_pass &p = passes[j];
		if ((j > i && p.sweep) || p.form != PHASE2_FORM_LIFTED_F32 ||
			nrec + p.nrot > P2_SW_MAXREC ||
			(j > i && p.rot_off != passes[j - 1].rot_off +
					passes[j - 1].nrot))
			break;
		for (uint32_t k = 0; k < p.span && n <= tl - L; k++)
			n = rref_add(rows, piv, n, (uint32_t)p.basis[k] & ~lowm);
		if (n > tl - L)
			return 1;
		nrec += p.nrot;
	}
	const size_t np = j - i;
	if (np < 2)
		return 1;
	rref_sort(rows, piv, n);
	memset(sw, 0, sizeof *sw);
	sw->np = (uint32_t)np;
	sw->k = (uint32_t)n;
	sw->L = (uint32_t)L;
	sw->rec0 = passes[i].rot_off;
	sw->nrec = nrec;
	for (int r = 0; r < n; r++) {
		sw->sb[r] = rows[r];
		sw->spiv[r] = (uint8_t)piv[r];
	}
	for (size_t q = 0; q < np; q++) {
		const struct phase2_pass &p = passes[i + q];
		struct p2_spass &P = sw->p[q];
		P.span = p.span;
		P.nrot = p.nrot;
		P.rec_off = p.rot_off - sw->rec0;
		P.negm = p.scale < 0 ? 0x80000000u : 0u;
		uint32_t er[PHASE2_MAX_SPAN], vr[PHASE2_MAX_SPAN];
		int ep[PHASE2_MAX_SPAN], vp[PHASE2_MAX_SPAN], ne = 0, nv = 0;
		for (uint32_t k = 0; k < p.span; k++) {
			P.pb[k] = (uint32_t)p.basis[k];
			P.vb[k] = sweep_vidx(*sw, P.pb[k]);
			/* every basis vector must lie in S + low */
			if (sweep_phys(*sw, P.vb[k]) != P.pb[k])
				return 1;
			ne = rref_add(er, ep, ne, P.pb[k]);
			nv = rref_add(vr, vp, nv, P.vb[k]);
		}
		if (ne != (int)p.span || nv != (int)p.span)
			return 1;
		rref_sort(er, ep, ne);
		rref_sort(vr, vp, nv);
		for (uint32_t k = 0; k < p.span; k++) {
			/* the pivots of the one-pass kernel's representatives */
			if ((int)p.piv[k] != ep[k])
				return 1;
			P.e[k] = er[k];
			P.piv[k] = (uint8_t)ep[k];
			P.ve[k] = sweep_vidx(*sw, er[k]);
			P.vpiv[k] = (uint8_t)vp[k];
		}
	}
	return np;
}

static int launch_sweep(struct p2_dev *d, const struct p2_sweep &sw,
	const struct phase2_rot_rec *d_recs)
{
	const uint32_t tl = sw.k + sw.L;
	const size_t smem = ((size_t)8 << tl) +
		(size_t)sw.nrec * sizeof(struct p2_lift32_rec) +
		((size_t)4 << sw.k);
	static int smem_set;
	if (!smem_set) {
		CUDA_OK(cudaFuncSetAttribute(k_sweep32,
				cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)(((size_t)8 << P2_SW_MAXTILE) +
					P2_SW_MAXREC * sizeof(struct p2_lift32_rec) +
					((size_t)4 << P2_SW_MAXK))),
			"sweep kernel shared memory");
		smem_set = 1;
	}
	const uint32_t ntiles = (uint32_t)(d->namp >> tl);
	uint32_t grid = (uint32_t)d->sm_count * 2;
	if (grid > ntiles)
		grid = ntiles;
	k_sweep32<<<grid, P2_SW_TPB, smem, d->stream>>>((float2 *)d->state, sw,
		d_recs, ntiles);
	return 0;
}

/* Launch a plan: planned sweeps as one kernel each (FP32 registers of
 * tile + 3 to 31 qubits), other passes one kernel each.  Returns the
 * kernels launched (state round trips) or -1. */
static long launch_all(struct p2_dev *d, const struct phase2_pass *passes,
	size_t npass, const struct phase2_rot_rec *d_recs)
{
	const bool sweeps = p2_sweep_tile > 0 && p2_sweep_kernel &&
		d->prec == PHASE2_PREC_FP32 && d->nqb <= 31 &&
		d->nqb >= (uint32_t)p2_sweep_tile + 3;
	struct p2_sweep sw;
	long launches = 0;
	for (size_t i = 0; i < npass; launches++) {
		const size_t n = sweeps ? sweep_from(passes, npass, i, &sw) : 1;
		if (n >= 2) {
			if (launch_sweep(d, sw, d_recs) < 0)
				return -1;
		} else if (launch_pass(d, passes[i], d_recs) < 0) {
			return -1;
		}
		i += n;
	}
	return launches;
}

static uint64_t fnv1a(uint64_t h, const void *p, size_t n)
{
	const unsigned char *b = (const unsigned char *)p;
	for (size_t i = 0; i < n; i++)
		h = (h ^ b[i]) * UINT64_C(0x100000001b3);
	return h;
}

/*
 * Flush plans that repeat byte for byte (every step of a Trotter run)
 * are launched from a CUDA graph: the first sighting runs normally, the
 * second captures the pass launches (reading a records buffer owned by
 * the graph), later ones replay it.  Returns the graph to replay, or NULL
 * to launch normally.
 */
static struct p2_graph *graph_for(struct p2_dev *d,
	const struct phase2_pass *passes, size_t npass,
	const struct phase2_rot_rec *recs, size_t nrec)
{
	if (!d->graphs_on || npass < 2)
		return NULL;
	uint64_t h = fnv1a(UINT64_C(0xcbf29ce484222325), passes,
		npass * sizeof *passes);
	h = fnv1a(h, recs, nrec * sizeof *recs);
	d->graph_clock++;
	struct p2_graph *lru = &d->graphs[0];
	for (int k = 0; k < P2_GRAPH_SLOTS; k++) {
		struct p2_graph *g = &d->graphs[k];
		if (g->hash == h && g->npass == npass && g->nrec == nrec &&
			g->passes &&
			!memcmp(g->passes, passes, npass * sizeof *passes) &&
			!memcmp(g->recs, recs, nrec * sizeof *recs)) {
			g->used = d->graph_clock;
			if (g->exec)
				return g;
			/* second sighting: capture */
			if (cudaMalloc((void **)&g->d_recs,
				    nrec * sizeof *recs) != cudaSuccess ||
				cudaMemcpyAsync(g->d_recs, g->recs,
					nrec * sizeof *recs,
					cudaMemcpyHostToDevice,
					d->stream) != cudaSuccess)
				return NULL;
			d->h2d_bytes += nrec * sizeof *recs;
			cudaGraph_t graph = NULL;
			if (cudaStreamBeginCapture(d->stream,
				    cudaStreamCaptureModeThreadLocal) !=
				cudaSuccess)
				return NULL;
			const long rc = launch_all(d, passes, npass, g->d_recs);
			const cudaError_t e = cudaStreamEndCapture(d->stream,
				&graph);
			g->nlaunch = rc > 0 ? (size_t)rc : 0;
			if (rc < 0 || e != cudaSuccess || !graph ||
				cudaGraphInstantiate(&g->exec, graph, 0) !=
					cudaSuccess) {
				if (graph)
					cudaGraphDestroy(graph);
				g->exec = NULL;
				cudaGetLastError();
				return NULL;
			}
			cudaGraphDestroy(graph);
			return g;
		}
		if (g->used < lru->used)
			lru = g;
	}
	/* first sighting: remember the plan in the least recently used slot */
	if (lru->exec)
		cudaGraphExecDestroy(lru->exec);
	if (lru->d_recs) {
		cudaStreamSynchronize(d->stream);
		cudaFree(lru->d_recs);
	}
	free(lru->passes);
	free(lru->recs);
	memset(lru, 0, sizeof *lru);
	lru->passes = (struct phase2_pass *)malloc(npass * sizeof *passes);
	lru->recs = (struct phase2_rot_rec *)malloc(nrec * sizeof *recs);
	if (!lru->passes || !lru->recs) {
		free(lru->passes);
		free(lru->recs);
		memset(lru, 0, sizeof *lru);
		return NULL;
	}
	memcpy(lru->passes, passes, npass * sizeof *passes);
	memcpy(lru->recs, recs, nrec * sizeof *recs);
	lru->hash = h;
	lru->npass = npass;
	lru->nrec = nrec;
	lru->used = d->graph_clock;
	return NULL;
}

extern "C" int p2d_run(struct p2_dev *d, const struct phase2_pass *passes,
	size_t npass, const struct phase2_rot_rec *recs, size_t nrec)
{
	if (npass == 0)
		return 0;
	struct p2_graph *g = graph_for(d, passes, npass, recs, nrec);
	if (!g) {
		if (recs_reserve(d, nrec) < 0)
			return -1;
		const int k = d->ring;
		memcpy(d->h_recs[k], recs, nrec * sizeof *recs);
		CUDA_OK(cudaMemcpyAsync(d->d_recs, d->h_recs[k],
				nrec * sizeof *recs, cudaMemcpyHostToDevice,
				d->stream),
			"upload rotation records");
		CUDA_OK(cudaEventRecord(d->h_ev[k], d->stream),
			"record staging");
		d->h2d_bytes += nrec * sizeof *recs;
		d->h_ev_live[k] = 1;
		d->ring ^= 1;
	}

	if (d->timing)
		CUDA_OK(cudaEventRecord(d->t0, d->stream), "timing start");
	long launches;
	if (g) {
		CUDA_OK(cudaGraphLaunch(g->exec, d->stream), "graph launch");
		d->graph_replays++;
		launches = (long)g->nlaunch;
	} else if ((launches = launch_all(d, passes, npass, d->d_recs)) < 0) {
		return -1;
	}
	CUDA_OK(cudaGetLastError(), "pass launch");
	d->passes += npass;
	d->sweeps += (uint64_t)launches;
	d->launches += (uint64_t)launches;
	d->rotations += nrec;
	if (d->timing) {
		CUDA_OK(cudaEventRecord(d->t1, d->stream), "timing stop");
		CUDA_OK(cudaEventSynchronize(d->t1), "timing wait");
		float ms = 0.0f;
		CUDA_OK(cudaEventElapsedTime(&ms, d->t0, d->t1), "elapsed");
		d->pass_ms += ms;
		d->timed_passes += npass;
		d->timed_sweeps += (uint64_t)launches;
	}
	return 0;
}

/* Partial-sum buffer for `blocks` reduction blocks plus the result. */
static int part_reserve(struct p2_dev *d, unsigned blocks)
{
	if (d->part_cap < 2 * (size_t)blocks + 2) {
		CUDA_OK(cudaStreamSynchronize(d->stream), "sync before partials");
		cudaFree(d->d_part);
		d->d_part = NULL;
		d->part_cap = 0;
		CUDA_OK(cudaMalloc((void **)&d->d_part,
				(2 * (size_t)blocks + 2) * sizeof(double)),
			"alloc partials");
		d->part_cap = 2 * (size_t)blocks + 2;
	}
	return 0;
}

/* Run k_reduce_final over `blocks` partials and download the result. */
static int reduce_finish(struct p2_dev *d, unsigned blocks, double out[2])
{
	k_reduce_final<<<1, P2_RED_TPB, 0, d->stream>>>(d->d_part, blocks,
		d->d_part + 2 * (size_t)blocks);
	d->launches += 1;
	CUDA_OK(cudaGetLastError(), "reduce launch");
	double h[2];
	CUDA_OK(cudaMemcpyAsync(h, d->d_part + 2 * (size_t)blocks, sizeof h,
			cudaMemcpyDeviceToHost, d->stream),
		"download reduction");
	CUDA_OK(cudaStreamSynchronize(d->stream), "reduce");
	d->d2h_bytes += sizeof h;
	out[0] = h[0];
	out[1] = h[1];
	return 0;
}

static int reduce(struct p2_dev *d, const double2 *trial, double out[2])
{
	const unsigned blocks = grid_for(d, d->namp, P2_RED_TPB, 4);
	if (part_reserve(d, blocks) < 0)
		return -1;
	if (d->prec == PHASE2_PREC_FP64)
		k_reduce_partial<<<blocks, P2_RED_TPB, 0, d->stream>>>(
			(const double2 *)d->state, trial, d->namp, d->d_part);
	else
		k_reduce_partial<<<blocks, P2_RED_TPB, 0, d->stream>>>(
			(const float2 *)d->state, trial, d->namp, d->d_part);
	d->launches += 1;
	return reduce_finish(d, blocks, out);
}

/* Upload the expansion tables (occupations, weights, determinants) into
 * the register's table buffer; *p receives the five device pointers. */
static int cm_upload(struct p2_dev *d, const uint64_t *occ_a, size_t Ma,
	const uint64_t *occ_b, size_t Mb, const double *w, size_t ncomp,
	const double *det_a, const double *det_b, void *p[5])
{
	const size_t sz[5] = { Ma * sizeof(uint64_t), Mb * sizeof(uint64_t),
		ncomp * sizeof(double), ncomp * Ma * sizeof(double),
		ncomp * Mb * sizeof(double) };
	const void *src[5] = { occ_a, occ_b, w, det_a, det_b };
	size_t off[5], total = 0;
	for (int k = 0; k < 5; k++) {
		off[k] = total;
		total += (sz[k] + 255) & ~(size_t)255;
	}
	if (total > d->cm_cap) {
		CUDA_OK(cudaStreamSynchronize(d->stream), "sync before tables");
		cudaFree(d->d_cm);
		d->d_cm = NULL;
		d->cm_cap = 0;
		CUDA_OK(cudaMalloc((void **)&d->d_cm, total), "alloc tables");
		d->cm_cap = total;
	}
	for (int k = 0; k < 5; k++) {
		p[k] = d->d_cm + off[k];
		if (sz[k])
			CUDA_OK(cudaMemcpyAsync(p[k], src[k], sz[k],
					cudaMemcpyHostToDevice, d->stream),
				"upload tables");
	}
	d->h2d_bytes += sz[0] + sz[1] + sz[2] + sz[3] + sz[4];
	return 0;
}

extern "C" int p2d_cm_expand(struct p2_dev *d, uint32_t n_sites, int tapered,
	int accumulate, const uint64_t *occ_a, size_t Ma, const uint64_t *occ_b,
	size_t Mb, const double *w, const double *det_a, const double *det_b,
	size_t ncomp)
{
	if (Ma == 0 || Mb == 0 || ncomp == 0)
		return 0;
	void *p[5];
	if (cm_upload(d, occ_a, Ma, occ_b, Mb, w, ncomp, det_a, det_b, p) < 0)
		return -1;
	const uint64_t n = (uint64_t)Ma * Mb;
	const unsigned grid = grid_for(d, n, P2_TPB, 8);
	if (d->prec == PHASE2_PREC_FP64)
		k_cm_expand<<<grid, P2_TPB, 0, d->stream>>>((double2 *)d->state,
			(const uint64_t *)p[0], (const uint64_t *)p[1], Ma, Mb,
			(const double *)p[2], (const double *)p[3],
			(const double *)p[4], (uint32_t)ncomp, n_sites, tapered,
			accumulate);
	else
		k_cm_expand<<<grid, P2_TPB, 0, d->stream>>>((float2 *)d->state,
			(const uint64_t *)p[0], (const uint64_t *)p[1], Ma, Mb,
			(const double *)p[2], (const double *)p[3],
			(const double *)p[4], (uint32_t)ncomp, n_sites, tapered,
			accumulate);
	d->launches += 1;
	CUDA_OK(cudaGetLastError(), "expansion launch");
	return 0;
}

extern "C" int p2d_cm_inner(struct p2_dev *d, uint32_t n_sites, int tapered,
	const uint64_t *occ_a, size_t Ma, const uint64_t *occ_b, size_t Mb,
	double w, const double *det_a, const double *det_b, double out[2])
{
	out[0] = out[1] = 0.0;
	if (Ma == 0 || Mb == 0)
		return 0;
	void *p[5];
	if (cm_upload(d, occ_a, Ma, occ_b, Mb, &w, 1, det_a, det_b, p) < 0)
		return -1;
	const uint64_t n = (uint64_t)Ma * Mb;
	const unsigned blocks = grid_for(d, n, P2_RED_TPB, 4);
	if (part_reserve(d, blocks) < 0)
		return -1;
	if (d->prec == PHASE2_PREC_FP64)
		k_cm_inner<<<blocks, P2_RED_TPB, 0, d->stream>>>(
			(const double2 *)d->state, (const uint64_t *)p[0],
			(const uint64_t *)p[1], Ma, Mb, w, (const double *)p[3],
			(const double *)p[4], n_sites, tapered, d->d_part);
	else
		k_cm_inner<<<blocks, P2_RED_TPB, 0, d->stream>>>(
			(const float2 *)d->state, (const uint64_t *)p[0],
			(const uint64_t *)p[1], Ma, Mb, w, (const double *)p[3],
			(const double *)p[4], n_sites, tapered, d->d_part);
	d->launches += 1;
	return reduce_finish(d, blocks, out);
}

extern "C" int p2d_norm2(struct p2_dev *d, double *out)
{
	double v[2];
	if (reduce(d, NULL, v) < 0)
		return -1;
	*out = v[0];
	return 0;
}

extern "C" int p2d_inner_dense(struct p2_dev *d, const double *trial,
	double out[2])
{
	double2 *t = NULL;
	const size_t bytes = d->namp * sizeof(double2);
	CUDA_OK(cudaMalloc((void **)&t, bytes), "alloc trial");
	cudaError_t e = cudaMemcpyAsync(t, trial, bytes, cudaMemcpyHostToDevice,
		d->stream);
	int rc = e == cudaSuccess ? reduce(d, t, out) : -1;
	cudaStreamSynchronize(d->stream);
	cudaFree(t);
	if (e != cudaSuccess)
		log_error("upload trial: %s", cudaGetErrorString(e));
	return rc;
}

extern "C" int p2d_sync(struct p2_dev *d)
{
	CUDA_OK(cudaStreamSynchronize(d->stream), "stream sync");
	CUDA_OK(cudaGetLastError(), "pending error");
	return 0;
}

extern "C" void p2d_stats(const struct p2_dev *d, struct phase2_stats *st)
{
	st->rotations = d->rotations;
	st->passes = d->passes;
	st->launches = d->launches;
	st->bytes = d->sweeps * 2 * d->namp * d->elem;
	st->timed_passes = d->timed_passes;
	st->pass_ms = d->pass_ms;
	st->h2d_bytes = d->h2d_bytes;
	st->d2h_bytes = d->d2h_bytes;
	st->graph_replays = d->graph_replays;
	st->sweeps = d->sweeps;
	st->timed_sweeps = d->timed_sweeps;
}

extern "C" void p2d_stats_reset(struct p2_dev *d)
{
	d->rotations = d->passes = d->launches = d->timed_passes = 0;
	d->sweeps = d->timed_sweeps = 0;
	d->h2d_bytes = d->d2h_bytes = 0;
	d->graph_replays = 0;
	d->pass_ms = 0.0;
}

extern "C" void p2d_set_timing(struct p2_dev *d, int on)
{
	d->timing = on != 0;
}

extern "C" void *p2d_stream(const struct p2_dev *d)
{
	return (void *)d->stream;
}

/* ---- batched persistent execution --------------------------------------- */

extern "C" int p2d_batch_ok(const struct p2_dev *d)
{
	return d && (d->prec == PHASE2_PREC_FP32 ||
			    d->prec == PHASE2_PREC_FP64) &&
		d->nqb <= 31;
}

static size_t p2_align256(size_t v)
{
	return (v + 255) & ~(size_t)255;
}

/* Idle scheduling rounds (each sleeps ~1 us) before a block gives up. */
#define P2_BATCH_IDLE_LIMIT 2000000u

/* k_batch for FP32 or FP64 registers: its kernel function (occupancy
 * queries) and its launch. */
static const void *batch_kernel(bool f64)
{
	return f64 ? (const void *)k_batch<double2>
		   : (const void *)k_batch<float2>;
}

static void batch_launch(bool f64, unsigned grid, cudaStream_t stream,
	const struct p2_binst *inst, uint32_t ninst, const struct p2_op *ops,
	const struct phase2_pass *passes, const struct phase2_rot_rec *recs,
	const uint64_t *widx, const double *wval, const uint64_t *gidx,
	double2 *gout, struct p2_bctl *ctl, unsigned int *status)
{
	if (f64)
		k_batch<double2><<<grid, P2_TPB, 0, stream>>>(inst, ninst, ops,
			passes, recs, widx, wval, gidx, gout, ctl, status,
			P2_BATCH_IDLE_LIMIT);
	else
		k_batch<float2><<<grid, P2_TPB, 0, stream>>>(inst, ninst, ops,
			passes, recs, widx, wval, gidx, gout, ctl, status,
			P2_BATCH_IDLE_LIMIT);
}

extern "C" int p2d_batch_run(struct p2_dev *const *devs,
	const struct p2_prog *const *progs, size_t n, double *gout,
	double *kernel_ms)
{
	if (n == 0)
		return 0;
	size_t nops = 0, npass = 0, nrec = 0, nw = 0, ng = 0;
	for (size_t i = 0; i < n; i++) {
		if (!p2d_batch_ok(devs[i]) || progs[i]->error ||
			devs[i]->prec != devs[0]->prec) {
			log_error("batch: program %zu cannot run batched", i);
			return -1;
		}
		nops += progs[i]->nops;
		npass += progs[i]->npass;
		nrec += progs[i]->nrec;
		nw += progs[i]->nw;
		ng += progs[i]->ng;
	}
	if (n > UINT32_MAX || nops > UINT32_MAX || npass > UINT32_MAX ||
		nrec > UINT32_MAX || nw > UINT32_MAX || ng > UINT32_MAX) {
		log_error("batch: program too large");
		return -1;
	}
	/* one device buffer: uploaded part, then outputs and control */
	const size_t o_inst = 0;
	const size_t o_ops = p2_align256(o_inst + n * sizeof(struct p2_binst));
	const size_t o_pass = p2_align256(o_ops + nops * sizeof(struct p2_op));
	const size_t o_rec =
		p2_align256(o_pass + npass * sizeof(struct phase2_pass));
	const size_t o_widx =
		p2_align256(o_rec + nrec * sizeof(struct phase2_rot_rec));
	const size_t o_wval = p2_align256(o_widx + nw * sizeof(uint64_t));
	const size_t o_gidx = p2_align256(o_wval + 2 * nw * sizeof(double));
	const size_t up = p2_align256(o_gidx + ng * sizeof(uint64_t));
	const size_t o_gout = up;
	const size_t o_ctl = p2_align256(o_gout + ng * sizeof(double2));
	const size_t o_status = p2_align256(o_ctl + n * sizeof(struct p2_bctl));
	const size_t total = o_status + 256;

	unsigned char *h = (unsigned char *)malloc(up);
	if (!h)
		return -1;
	struct p2_binst *hi = (struct p2_binst *)(h + o_inst);
	struct p2_op *ho = (struct p2_op *)(h + o_ops);
	struct phase2_pass *hp = (struct phase2_pass *)(h + o_pass);
	struct phase2_rot_rec *hr = (struct phase2_rot_rec *)(h + o_rec);
	uint64_t *hwi = (uint64_t *)(h + o_widx);
	double *hwv = (double *)(h + o_wval);
	uint64_t *hgi = (uint64_t *)(h + o_gidx);
	size_t bo = 0, bp = 0, br = 0, bw = 0, bg = 0;
	for (size_t i = 0; i < n; i++) {
		const struct p2_prog *pg = progs[i];
		struct p2_dev *d = devs[i];
		hi[i].state = d->state;
		hi[i].namp = d->namp;
		hi[i].op_off = (uint32_t)bo;
		hi[i].nops = (uint32_t)pg->nops;
		for (size_t k = 0; k < pg->npass; k++) {
			hp[bp + k] = pg->passes[k];
			hp[bp + k].rot_off += (uint32_t)br;
		}
		for (size_t k = 0; k < pg->nops; k++) {
			struct p2_op op = pg->ops[k];
			switch (op.kind) {
			case P2_OP_PASS:
				op.a += (uint32_t)bp;
				op.ntiles = p2_op_tiles(P2_OP_PASS, d->namp,
					hp[op.a].span, &op.b);
				break;
			case P2_OP_ZERO:
				op.ntiles = p2_op_tiles(P2_OP_ZERO, d->namp, 0,
					&op.b);
				break;
			case P2_OP_WRITE:
				op.a += (uint32_t)bw;
				op.ntiles = 1;
				break;
			default:
				op.a += (uint32_t)bg;
				op.ntiles = 1;
				break;
			}
			ho[bo + k] = op;
		}
		if (pg->nrec)
			memcpy(hr + br, pg->recs, pg->nrec * sizeof *hr);
		if (pg->nw) {
			memcpy(hwi + bw, pg->widx, pg->nw * sizeof *hwi);
			memcpy(hwv + 2 * bw, pg->wval,
				2 * pg->nw * sizeof *hwv);
		}
		if (pg->ng)
			memcpy(hgi + bg, pg->gidx, pg->ng * sizeof *hgi);
		bo += pg->nops;
		bp += pg->npass;
		br += pg->nrec;
		bw += pg->nw;
		bg += pg->ng;
	}

	struct p2_dev *d0 = devs[0];
	unsigned char *dbuf = NULL;
	cudaError_t e = cudaSuccess;
	for (size_t i = 0; i < n && e == cudaSuccess; i++)
		e = cudaStreamSynchronize(devs[i]->stream);
	if (e == cudaSuccess)
		e = cudaMalloc((void **)&dbuf, total);
	if (e == cudaSuccess)
		e = cudaMemcpy(dbuf, h, up, cudaMemcpyHostToDevice);
	free(h);
	if (e == cudaSuccess)
		e = cudaMemset(dbuf + o_ctl, 0, total - o_ctl);
	const bool f64 = d0->prec == PHASE2_PREC_FP64;
	int per_sm = 0;
	if (e == cudaSuccess)
		e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
			batch_kernel(f64), P2_TPB, 0);
	if (e != cudaSuccess) {
		cudaFree(dbuf);
		log_error("batch: setup: %s", cudaGetErrorString(e));
		return -1;
	}
	const unsigned grid =
		(unsigned)d0->sm_count * (unsigned)(per_sm > 0 ? per_sm : 1);
	cudaEventRecord(d0->t0, d0->stream);
	batch_launch(f64, grid, d0->stream,
		(const struct p2_binst *)(dbuf + o_inst), (uint32_t)n,
		(const struct p2_op *)(dbuf + o_ops),
		(const struct phase2_pass *)(dbuf + o_pass),
		(const struct phase2_rot_rec *)(dbuf + o_rec),
		(const uint64_t *)(dbuf + o_widx),
		(const double *)(dbuf + o_wval),
		(const uint64_t *)(dbuf + o_gidx), (double2 *)(dbuf + o_gout),
		(struct p2_bctl *)(dbuf + o_ctl),
		(unsigned int *)(dbuf + o_status));
	e = cudaGetLastError();
	cudaEventRecord(d0->t1, d0->stream);
	unsigned int status = 0;
	if (e == cudaSuccess)
		e = cudaStreamSynchronize(d0->stream);
	if (e == cudaSuccess)
		e = cudaMemcpy(&status, dbuf + o_status, sizeof status,
			cudaMemcpyDeviceToHost);
	if (e == cudaSuccess && ng)
		e = cudaMemcpy(gout, dbuf + o_gout, ng * sizeof(double2),
			cudaMemcpyDeviceToHost);
	float ms = 0.0f;
	if (e == cudaSuccess)
		e = cudaEventElapsedTime(&ms, d0->t0, d0->t1);
	cudaFree(dbuf);
	if (e != cudaSuccess) {
		log_error("batch: %s", cudaGetErrorString(e));
		return -1;
	}
	if (status) {
		log_error("batch: a block found no work for %u rounds",
			P2_BATCH_IDLE_LIMIT);
		return -1;
	}
	if (kernel_ms)
		*kernel_ms = ms;
	uint64_t npass_run = 0;
	for (size_t i = 0; i < n; i++) {
		struct p2_dev *d = devs[i];
		const struct p2_prog *pg = progs[i];
		uint64_t np = 0;
		for (size_t k = 0; k < pg->nops; k++)
			np += pg->ops[k].kind == P2_OP_PASS;
		npass_run += np;
		d->passes += np;
		d->sweeps += np;
		d->rotations += pg->rotations;
		d->h2d_bytes += pg->nrec * sizeof(struct phase2_rot_rec) +
			pg->nw * (sizeof(uint64_t) + 2 * sizeof(double));
		d->d2h_bytes += pg->ng * sizeof(double2);
	}
	/* the one launch, timed with events, counts as the first program's */
	d0->launches += 1;
	d0->pass_ms += ms;
	d0->timed_passes += npass_run;
	d0->timed_sweeps += npass_run;
	d0->h2d_bytes += o_pass; /* program tables */
	return 0;
}

/* ---- device-side qDRIFT ------------------------------------------------- */

/* xoshiro256** step (lib/xoshiro256ss.c of the reference). */
__device__ __forceinline__ uint64_t p2_xo_next(uint64_t (&s)[4])
{
	const uint64_t x = s[1] * 5;
	const uint64_t out = ((x << 7) | (x >> 57)) * 9;
	const uint64_t t = s[1] << 17;
	s[2] ^= s[0];
	s[3] ^= s[1];
	s[1] ^= s[2];
	s[0] ^= s[3];
	s[2] ^= t;
	s[3] = (s[3] << 45) | (s[3] >> 19);
	return out;
}

/*
 * Device sampling (p2d_sampled_device).  A sample's rotation stream is
 * `halves` halves of (length + depth) rotations: a forward half is the
 * head terms 0..length-1 then the draws 0..depth-1, a reversed half (odd
 * halves when reverse_odd) the draws depth-1..0 then the head terms
 * length-1..0.  Buffers of a round of g samples, T rotations each:
 * x[(s * halves + h) * depth + i] uniforms, rot/cs/passes/recs at
 * s * T + position, per-chunk pass counts npc[s * C + c].
 */

/* Uniforms of one (sample, half): the half's generator, depth draws. */
__global__ void k_smp_draw(const struct p2_smp_job job, uint32_t s0,
	uint32_t n, const uint64_t *__restrict__ rng0, double *__restrict__ x)
{
	const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
	if (id >= n)
		return;
	uint64_t st[4];
	const size_t g = (size_t)s0 * job.halves + id;
	for (int k = 0; k < 4; ++k)
		st[k] = rng0[4 * g + k];
	double *out = x + (size_t)id * job.depth;
	for (uint32_t i = 0; i < job.depth; ++i)
		out[i] = (double)(p2_xo_next(st) >> 11) * 0x1.0p-53;
}

/* The rotation at every stream position: head terms from the head table,
 * draws by CDF inversion (prob_cdf_inverse: smallest i with y[i] > x,
 * clamped) with the sign dead zone (|c| < DBL_EPSILON -> 0). */
__global__ void k_smp_stream(const struct p2_smp_job job, uint64_t total,
	const double *__restrict__ x, const double *__restrict__ cdf_y,
	const uint64_t *__restrict__ tflip, const uint64_t *__restrict__ tphase,
	const double *__restrict__ tcf, const uint64_t *__restrict__ hflip,
	const uint64_t *__restrict__ hphase, const double *__restrict__ hphi,
	const double *__restrict__ hcs, struct phase2_rot_in *__restrict__ rot,
	double *__restrict__ cs)
{
	const uint64_t per = (uint64_t)job.length + job.depth;
	const uint64_t T = per * job.halves;
	for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		q < total; q += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t s = q / T, p = q - s * T;
		const uint64_t h = p / per, o = p - h * per;
		const bool rev = job.reverse_odd && (h & 1);
		int64_t head = -1, draw = -1;
		if (!rev) {
			if (o < job.length)
				head = (int64_t)o;
			else
				draw = (int64_t)(o - job.length);
		} else {
			if (o < job.depth)
				draw = (int64_t)(job.depth - 1 - o);
			else
				head = (int64_t)(job.length - 1 - (o - job.depth));
		}
		struct phase2_rot_in r;
		double c, sn;
		if (head >= 0) {
			r.flip = hflip[head] & job.mask;
			r.phase = hphase[head] & job.mask;
			r.phi = hphi[head];
			c = hcs[2 * head];
			sn = hcs[2 * head + 1];
		} else {
			const double xv =
				x[(s * job.halves + h) * job.depth + (uint64_t)draw];
			uint64_t lo = 0, hi = job.nterms;
			while (lo < hi) {
				const uint64_t mid = lo + (hi - lo) / 2;
				if (cdf_y[mid] <= xv)
					lo = mid + 1;
				else
					hi = mid;
			}
			const uint64_t k = lo < job.nterms ? lo : job.nterms - 1;
			const double a = tcf[k], f = fabs(a);
			const int sg = f < DBL_EPSILON ? 1 : (a < f ? 0 : 2);
			r.flip = tflip[k] & job.mask;
			r.phase = tphase[k] & job.mask;
			/* selects, not an index (keeps job out of local memory) */
			r.phi = sg == 0 ? job.rphi[0]
					: (sg == 1 ? job.rphi[1] : job.rphi[2]);
			c = sg == 0 ? job.rcs[0][0]
				    : (sg == 1 ? job.rcs[1][0] : job.rcs[2][0]);
			sn = sg == 0 ? job.rcs[0][1]
				     : (sg == 1 ? job.rcs[1][1] : job.rcs[2][1]);
		}
		rot[q] = r;
		cs[2 * q] = c;
		cs[2 * q + 1] = sn;
	}
}

/*
 * One block per P2_QUEUE_FLUSH chunk of a sample's stream: the passes a
 * host flush of that chunk plans (plan_core.h), at the chunk's position;
 * npc gets their count.  The flip masks are staged in shared memory for
 * the sequential boundary scan (thread 0); the records are then filled by
 * all threads, and each pass's scale is the parity of its records' signs.
 */
#define P2_SMP_PLAN_TPB 256
#define P2_SMP_PLAN_SMEM                                                      \
	(P2_QUEUE_FLUSH * (sizeof(uint64_t) + sizeof(uint16_t) + 1) +          \
		P2_QUEUE_FLUSH / 8)

__global__ void __launch_bounds__(P2_SMP_PLAN_TPB)
	k_smp_plan(const struct p2_smp_job job, uint64_t T, uint32_t C,
		const struct phase2_rot_in *__restrict__ rot,
		const double *__restrict__ cs, struct phase2_pass *passes,
		struct phase2_rot_rec *__restrict__ recs, uint32_t *npc)
{
	extern __shared__ __align__(16) unsigned char sm[];
	uint64_t *fl = (uint64_t *)sm;
	uint16_t *pid = (uint16_t *)(fl + P2_QUEUE_FLUSH);
	uint8_t *U = (uint8_t *)(pid + P2_QUEUE_FLUSH);
	uint32_t *neg = (uint32_t *)(U + P2_QUEUE_FLUSH);
	__shared__ long s_np;
	const uint64_t s = blockIdx.x / C, c = blockIdx.x - s * C;
	const uint64_t at = s * T + c * P2_QUEUE_FLUSH;
	const uint32_t n = (uint32_t)(T - c * P2_QUEUE_FLUSH < P2_QUEUE_FLUSH
			? T - c * P2_QUEUE_FLUSH
			: P2_QUEUE_FLUSH);
	for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
		fl[i] = rot[at + i].flip;
	for (uint32_t w = threadIdx.x; w < P2_QUEUE_FLUSH / 32; w += blockDim.x)
		neg[w] = 0;
	__syncthreads();
	if (threadIdx.x == 0)
		s_np = p2_plan_scan(job.nqb, fl, 1, n, job.max_span,
			job.max_rots, P2_DEFAULT_PAD_SPAN, job.form, job.sweep_k,
			job.sweep_low, passes + at, U, 1, pid);
	__syncthreads();
	const long np = s_np;
	if (np < 0) {
		if (threadIdx.x == 0)
			npc[blockIdx.x] = 0;
		return;
	}
	for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
		const uint32_t p = pid[i];
		struct phase2_rot_rec r;
		if (p2_rec_fill(&passes[at + p], fl[i], rot[at + i].phase,
			    cs[2 * (at + i)], cs[2 * (at + i) + 1], U[i], &r))
			atomicXor(&neg[p >> 5], 1u << (p & 31));
		recs[at + i] = r;
	}
	__syncthreads();
	for (uint32_t p = threadIdx.x; p < (uint32_t)np; p += blockDim.x) {
		passes[at + p].scale = (neg[p >> 5] >> (p & 31)) & 1 ? -1.0 : 1.0;
		passes[at + p].rot_off += (uint32_t)at;
	}
	if (threadIdx.x == 0)
		npc[blockIdx.x] = (uint32_t)np;
}

/*
 * Lay out the registers' programs (one thread): sample s0 + s runs on
 * register (last - s0 - s) % nreg, so the run's last sample lands on
 * register 0; a register's samples keep their order.  A sample's ops are
 * zero, write, its chunks' passes in order, gather: poff[s * C + c] is
 * the op index of chunk c's first pass, soff[s] of the sample's zero.
 */
__global__ void k_smp_layout(uint32_t g, uint32_t C,
	const uint32_t *__restrict__ npc, uint64_t last, uint64_t s0,
	uint32_t nreg, uint32_t *soff, uint32_t *poff, struct p2_binst *inst)
{
	if (blockIdx.x != 0 || threadIdx.x != 0)
		return;
	for (uint32_t r = 0; r < nreg; ++r)
		inst[r].nops = 0;
	for (uint32_t s = 0; s < g; ++s) {
		uint32_t n = 3;
		for (uint32_t c = 0; c < C; ++c)
			n += npc[s * C + c];
		inst[(uint32_t)((last - s0 - s) % nreg)].nops += n;
		soff[s] = n; /* count for now */
	}
	uint32_t t = 0;
	for (uint32_t r = 0; r < nreg; ++r) {
		inst[r].op_off = t;
		t += inst[r].nops;
		inst[r].nops = 0; /* filled below */
	}
	for (uint32_t s = 0; s < g; ++s) {
		const uint32_t r = (uint32_t)((last - s0 - s) % nreg);
		const uint32_t n = soff[s];
		soff[s] = inst[r].op_off + inst[r].nops;
		inst[r].nops += n;
		uint32_t o = soff[s] + 2;
		for (uint32_t c = 0; c < C; ++c) {
			poff[s * C + c] = o;
			o += npc[s * C + c];
		}
	}
}

/* Fill the ops laid out by k_smp_layout (grid-stride over chunks). */
__global__ void k_smp_fill(const struct p2_smp_job job, uint32_t g,
	uint32_t C, uint64_t T, uint64_t namp, uint64_t s0,
	const uint32_t *__restrict__ npc, const uint32_t *__restrict__ soff,
	const uint32_t *__restrict__ poff,
	const struct phase2_pass *__restrict__ passes, struct p2_op *ops)
{
	const uint32_t stride = gridDim.x * blockDim.x;
	const uint32_t id0 = blockIdx.x * blockDim.x + threadIdx.x;
	for (uint32_t s = id0; s < g; s += stride) {
		struct p2_op *o = ops + soff[s];
		o[0].kind = P2_OP_ZERO;
		o[0].a = o[0].b = 0;
		o[0].ntiles = p2_op_tiles(P2_OP_ZERO, namp, 0, &o[0].b);
		o[1].kind = P2_OP_WRITE;
		o[1].a = 0;
		o[1].b = job.ndet;
		o[1].ntiles = 1;
		uint32_t np = 0;
		for (uint32_t c = 0; c < C; ++c)
			np += npc[s * C + c];
		struct p2_op *gth = o + 2 + np;
		gth->kind = P2_OP_GATHER;
		gth->a = (uint32_t)((s0 + s) * job.ndet);
		gth->b = job.ndet;
		gth->ntiles = 1;
	}
	for (uint32_t e = id0; e < g * C; e += stride) {
		const uint64_t s = e / C, c = e - s * C;
		const uint64_t at = s * T + c * P2_QUEUE_FLUSH;
		struct p2_op *o = ops + poff[e];
		for (uint32_t p = 0; p < npc[e]; ++p) {
			o[p].kind = P2_OP_PASS;
			o[p].a = (uint32_t)(at + p);
			o[p].ntiles = p2_op_tiles(P2_OP_PASS, namp,
				passes[at + p].span, &o[p].b);
		}
	}
}

/* Rotations held per device round (rotation scratch, plans, program). */
#define P2_SMP_ROUND_ROTS (UINT64_C(1) << 21)
/* Amplitudes of all the registers of one round together (FP32: 512 MiB);
 * from 2^26 amplitudes up the register runs alone. */
#define P2_SMP_ROUND_AMPS (UINT64_C(1) << 26)

extern "C" int p2d_sampled_device(struct p2_dev *d,
	const struct p2_smp_job *job, const uint64_t *rng0, size_t samples,
	const double *cdf_y, const uint64_t *tflip, const uint64_t *tphase,
	const double *tcf, const uint64_t *hflip, const uint64_t *hphase,
	const double *hphi, const double *hcs, const uint64_t *det_idx,
	const double *det_val, double *gout, uint64_t *npass_out)
{
	*npass_out = 0;
	if (samples == 0)
		return 0;
	const uint64_t per = (uint64_t)job->length + job->depth;
	const uint64_t T = per * job->halves;
	if (!p2d_batch_ok(d) || (job->depth && job->nterms == 0) ||
		T >= (UINT64_C(1) << 31) || job->halves == 0 ||
		samples > UINT32_MAX / (job->ndet ? job->ndet : 1)) {
		log_error("device sampling: unsupported register or sizes");
		return -1;
	}
	size_t G = T ? (size_t)(P2_SMP_ROUND_ROTS / T) : 4096;
	if (G < 1)
		G = 1;
	if (G > samples)
		G = samples;
	if (G > 4096)
		G = 4096;
	size_t R = (size_t)(P2_SMP_ROUND_AMPS / d->namp);
	if (R > P2_QD_MAX_REGS)
		R = P2_QD_MAX_REGS;
	if (R > G)
		R = G;
	if (R < 1)
		R = 1;
	const uint32_t C = (uint32_t)((T + P2_QUEUE_FLUSH - 1) / P2_QUEUE_FLUSH);
	const size_t nt = job->nterms, nd = job->ndet, nh = job->length;
	/* device buffer: tables, per-round scratch and program, registers */
	enum { RNG, CDF, TFL, TPH, TCF, HFL, HPH, HPHI, HCS, WIDX, WVAL, GIDX,
		GOUT, X, ROT, CS, PASS, REC, PROG, NPC, SOFF, POFF, REGS, NBUF };
	size_t sz[NBUF], off[NBUF], total = 0;
	/* sizes and offsets for rounds of G samples on R registers */
	auto layout = [&](size_t G, size_t R) {
		const size_t GT = G * T > 0 ? G * T : 1;
		sz[RNG] = 4 * samples * job->halves * sizeof(uint64_t);
		sz[CDF] = nt * sizeof(double);
		sz[TFL] = sz[TPH] = nt * sizeof(uint64_t);
		sz[TCF] = nt * sizeof(double);
		sz[HFL] = sz[HPH] = nh * sizeof(uint64_t);
		sz[HPHI] = nh * sizeof(double);
		sz[HCS] = 2 * nh * sizeof(double);
		sz[WIDX] = nd * sizeof(uint64_t);
		sz[WVAL] = 2 * nd * sizeof(double);
		sz[GIDX] = samples * nd * sizeof(uint64_t);
		sz[GOUT] = samples * nd * sizeof(double2);
		sz[X] = G * job->halves * (size_t)job->depth * sizeof(double);
		sz[ROT] = GT * sizeof(struct phase2_rot_in);
		sz[CS] = 2 * GT * sizeof(double);
		sz[PASS] = GT * sizeof(struct phase2_pass);
		sz[REC] = GT * sizeof(struct phase2_rot_rec);
		sz[PROG] = (G * T + 3 * G) * sizeof(struct p2_op);
		sz[NPC] = sz[POFF] = (G * C ? G * C : 1) * sizeof(uint32_t);
		sz[SOFF] = G * sizeof(uint32_t);
		sz[REGS] = R * (sizeof(struct p2_binst) +
				       sizeof(struct p2_bctl)) +
			sizeof(unsigned int) + (R - 1) * d->namp * d->elem;
		total = 0;
		for (int i = 0; i < NBUF; i++) {
			off[i] = total;
			total += (sz[i] + 255) & ~(size_t)255;
		}
	};
	unsigned char *b = NULL;
	CUDA_OK(cudaStreamSynchronize(d->stream), "device sampling: sync");
	/* on a full device: fewer state copies, then smaller rounds */
	for (;;) {
		layout(G, R);
		if (cudaMalloc((void **)&b, total) == cudaSuccess)
			break;
		cudaGetLastError();
		b = NULL;
		if (R > 1) {
			R = 1;
		} else if (G > 1) {
			G = (G + 1) / 2;
		} else {
			log_error("device sampling: no room for %zu bytes of "
				  "scratch", total);
			return -1;
		}
	}
	uint64_t *gidx = (uint64_t *)malloc(sz[GIDX] ? sz[GIDX] : 1);
	struct p2_binst *hinst = (struct p2_binst *)malloc(
		R * sizeof(struct p2_binst));
	int rc = -1;
	cudaError_t e = gidx && hinst ? cudaSuccess
				      : cudaErrorMemoryAllocation;
	/* registers: the copies first (256-aligned), then inst, ctl, status */
	unsigned char *copies = b + off[REGS];
	struct p2_binst *inst = (struct p2_binst *)(b + off[REGS] +
		(R - 1) * d->namp * d->elem);
	struct p2_bctl *ctl = (struct p2_bctl *)(inst + R);
	unsigned int *status = (unsigned int *)(ctl + R);
	if (e == cudaSuccess) {
		for (size_t s = 0; s < samples; s++)
			for (size_t j = 0; j < nd; j++)
				gidx[s * nd + j] = det_idx[j];
		for (size_t r = 0; r < R; r++) {
			hinst[r].state = r == 0
				? d->state
				: (void *)(copies + (r - 1) * d->namp * d->elem);
			hinst[r].namp = d->namp;
			hinst[r].op_off = hinst[r].nops = 0;
		}
		const void *src[] = { rng0, cdf_y, tflip, tphase, tcf, hflip,
			hphase, hphi, hcs, det_idx, det_val, gidx };
		const int at[] = { RNG, CDF, TFL, TPH, TCF, HFL, HPH, HPHI, HCS,
			WIDX, WVAL, GIDX };
		for (int i = 0; i < 12 && e == cudaSuccess; i++)
			if (sz[at[i]]) {
				e = cudaMemcpyAsync(b + off[at[i]], src[i],
					sz[at[i]], cudaMemcpyHostToDevice,
					d->stream);
				d->h2d_bytes += sz[at[i]];
			}
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(inst, hinst,
				R * sizeof(struct p2_binst),
				cudaMemcpyHostToDevice, d->stream);
	}
	const bool f64 = d->prec == PHASE2_PREC_FP64;
	int per_sm = 0;
	if (e == cudaSuccess)
		e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
			batch_kernel(f64), P2_TPB, 0);
	if (e == cudaSuccess)
		e = cudaFuncSetAttribute(k_smp_plan,
			cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)P2_SMP_PLAN_SMEM);
	/* no op has more tiles than a span-0 pass or a zero (more blocks
	 * would only poll) */
	uint32_t cpt = 0;
	uint64_t most = p2_op_tiles(P2_OP_PASS, d->namp, 0, &cpt);
	const uint32_t zt = p2_op_tiles(P2_OP_ZERO, d->namp, 0, &cpt);
	if (zt > most)
		most = zt;
	most *= R;
	unsigned grid =
		(unsigned)d->sm_count * (unsigned)(per_sm > 0 ? per_sm : 1);
	if (most < grid)
		grid = (unsigned)most;
	uint32_t *npc = (uint32_t *)(b + off[NPC]);
	uint32_t *soff = (uint32_t *)(b + off[SOFF]);
	uint32_t *poff = (uint32_t *)(b + off[POFF]);
	uint64_t nops_run = 0;
	/* PHASE2_SAMPLING_TIMING=1: per-round stage times on stderr */
	const char *tenv = getenv("PHASE2_SAMPLING_TIMING");
	const int timing = tenv && *tenv == '1';
	cudaEvent_t ev[5] = { 0, 0, 0, 0, 0 };
	for (int i = 0; timing && i < 5; i++)
		cudaEventCreate(&ev[i]);
	for (size_t s0 = 0; s0 < samples && e == cudaSuccess; s0 += G) {
		const uint32_t g = (uint32_t)(samples - s0 < G ? samples - s0 : G);
		const uint32_t nreg = (uint32_t)(g < R ? g : R);
		const uint32_t nx = g * job->halves;
		if (timing)
			cudaEventRecord(ev[0], d->stream);
		if (job->depth)
			k_smp_draw<<<(nx + 127) / 128, 128, 0, d->stream>>>(
				*job, (uint32_t)s0, nx,
				(const uint64_t *)(b + off[RNG]),
				(double *)(b + off[X]));
		const uint64_t tot = (uint64_t)g * T;
		if (tot)
			k_smp_stream<<<grid_for(d, tot, P2_TPB, 8), P2_TPB, 0,
				d->stream>>>(*job, tot,
				(const double *)(b + off[X]),
				(const double *)(b + off[CDF]),
				(const uint64_t *)(b + off[TFL]),
				(const uint64_t *)(b + off[TPH]),
				(const double *)(b + off[TCF]),
				(const uint64_t *)(b + off[HFL]),
				(const uint64_t *)(b + off[HPH]),
				(const double *)(b + off[HPHI]),
				(const double *)(b + off[HCS]),
				(struct phase2_rot_in *)(b + off[ROT]),
				(double *)(b + off[CS]));
		if (timing)
			cudaEventRecord(ev[1], d->stream);
		const uint32_t nch = g * C;
		if (nch)
			k_smp_plan<<<nch, P2_SMP_PLAN_TPB, P2_SMP_PLAN_SMEM,
				d->stream>>>(*job, T, C,
				(const struct phase2_rot_in *)(b + off[ROT]),
				(const double *)(b + off[CS]),
				(struct phase2_pass *)(b + off[PASS]),
				(struct phase2_rot_rec *)(b + off[REC]), npc);
		if (timing)
			cudaEventRecord(ev[2], d->stream);
		k_smp_layout<<<1, 32, 0, d->stream>>>(g, C, npc,
			(uint64_t)samples - 1, (uint64_t)s0, nreg, soff, poff,
			inst);
		k_smp_fill<<<(g * C + g + 127) / 128, 128, 0, d->stream>>>(
			*job, g, C, T, d->namp, (uint64_t)s0, npc, soff, poff,
			(const struct phase2_pass *)(b + off[PASS]),
			(struct p2_op *)(b + off[PROG]));
		e = cudaGetLastError();
		if (timing)
			cudaEventRecord(ev[3], d->stream);
		if (e == cudaSuccess)
			e = cudaMemsetAsync(ctl, 0, nreg * sizeof *ctl,
				d->stream);
		if (e == cudaSuccess)
			e = cudaMemsetAsync(status, 0, sizeof(unsigned int),
				d->stream);
		if (e == cudaSuccess)
			batch_launch(f64, grid, d->stream, inst, nreg,
				(const struct p2_op *)(b + off[PROG]),
				(const struct phase2_pass *)(b + off[PASS]),
				(const struct phase2_rot_rec *)(b + off[REC]),
				(const uint64_t *)(b + off[WIDX]),
				(const double *)(b + off[WVAL]),
				(const uint64_t *)(b + off[GIDX]),
				(double2 *)(b + off[GOUT]), ctl, status);
		if (e == cudaSuccess)
			e = cudaGetLastError();
		if (timing)
			cudaEventRecord(ev[4], d->stream);
		/* draw, stream and plan run only when they have work */
		d->launches += 3 + (job->depth != 0) + (tot != 0) + (nch != 0);
		unsigned int st = 0;
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(&st, status, sizeof st,
				cudaMemcpyDeviceToHost, d->stream);
		if (e == cudaSuccess)
			e = cudaMemcpyAsync(hinst, inst,
				nreg * sizeof(struct p2_binst),
				cudaMemcpyDeviceToHost, d->stream);
		if (e == cudaSuccess)
			e = cudaStreamSynchronize(d->stream);
		if (e == cudaSuccess && st) {
			log_error("device sampling: a block found no work for"
				  " %u rounds",
				P2_BATCH_IDLE_LIMIT);
			e = cudaErrorLaunchFailure;
		}
		uint64_t rops = 0;
		for (uint32_t r = 0; e == cudaSuccess && r < nreg; r++)
			rops += hinst[r].nops;
		nops_run += rops - 3ull * g;
		if (timing && e == cudaSuccess) {
			float t[4];
			for (int i = 0; i < 4; i++)
				cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
			fprintf(stderr,
				"device sampling: %u samples x %llu rotations,"
				" %u registers, %llu ops, grid %u: draw+stream"
				" %.3f ms, plan %.3f ms, layout %.3f ms, run"
				" %.3f ms\n",
				g, (unsigned long long)T, nreg,
				(unsigned long long)rops, grid, t[0], t[1], t[2],
				t[3]);
		}
	}
	for (int i = 0; timing && i < 5; i++)
		cudaEventDestroy(ev[i]);
	if (e == cudaSuccess && sz[GOUT])
		e = cudaMemcpy(gout, b + off[GOUT], sz[GOUT],
			cudaMemcpyDeviceToHost);
	if (e == cudaSuccess) {
		d->d2h_bytes += sz[GOUT];
		d->passes += nops_run;
		d->sweeps += nops_run;
		d->rotations += (uint64_t)samples * T;
		*npass_out = nops_run;
		rc = 0;
	} else {
		log_error("device sampling: %s", cudaGetErrorString(e));
	}
	free(gidx);
	free(hinst);
	cudaFree(b);
	return rc;
}

/* ---- allocation-free norm (phase2_norm2_noalloc) ------------------------ */

/*
 * Per-block partial sums for phase2_norm2_noalloc live in this file-scope
 * device array instead of memory obtained from cudaMalloc.  Every GPU that
 * loads the library holds it (about 128 KiB) until the process exits.
 * Host code must not use the symbol as an address: on the host it names a
 * stand-in, so the device address is looked up per device with
 * cudaGetSymbolAddress and passed to the kernels.
 */
#define P2_NOALLOC_MAX_BLOCKS 8192
#define P2_NOALLOC_CHUNK (UINT64_C(1) << 21)
#define P2_NOALLOC_MAX_AMPS ((uint64_t)P2_NOALLOC_MAX_BLOCKS * P2_NOALLOC_CHUNK)
#define P2_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) double
	p2_noalloc_scratch[2 * P2_NOALLOC_MAX_BLOCKS];

static double *p2_noalloc_addr[P2_NOALLOC_MAX_DEVICES];

extern "C" int phase2_norm2_noalloc(const void *d_state, int prec,
	uint64_t namp, double *d_out, void *stream)
{
	if (!d_state || !d_out) {
		log_error("phase2_norm2_noalloc: NULL state or output pointer");
		return -1;
	}
	if (prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32) {
		log_error("phase2_norm2_noalloc: unknown precision %d", prec);
		return -1;
	}
	if (namp == 0 || namp > P2_NOALLOC_MAX_AMPS) {
		log_error("phase2_norm2_noalloc: %llu amplitudes outside"
			  " [1, %llu]: the fixed scratch holds %d partial sums"
			  " of up to %llu amplitudes each",
			(unsigned long long)namp,
			(unsigned long long)P2_NOALLOC_MAX_AMPS,
			P2_NOALLOC_MAX_BLOCKS,
			(unsigned long long)P2_NOALLOC_CHUNK);
		return -1;
	}
	int dev = 0;
	CUDA_OK(cudaGetDevice(&dev), "phase2_norm2_noalloc: current device");
	if (dev < 0 || dev >= P2_NOALLOC_MAX_DEVICES) {
		log_error("phase2_norm2_noalloc: device %d beyond the %d"
			  " supported", dev, P2_NOALLOC_MAX_DEVICES);
		return -1;
	}
	if (!p2_noalloc_addr[dev]) {
		/* first call on this device: resolve the array's address */
		double *ptr = NULL;
		CUDA_OK(cudaGetSymbolAddress((void **)&ptr, p2_noalloc_scratch),
			"phase2_norm2_noalloc: scratch address");
		p2_noalloc_addr[dev] = ptr;
	}
	double *part = p2_noalloc_addr[dev];
	const cudaStream_t s = (cudaStream_t)stream;
	/* Each block writes its own two slots before the final kernel reads
	 * them (stream order), so the array needs no clearing. */
	const unsigned blocks =
		(unsigned)((namp + P2_NOALLOC_CHUNK - 1) / P2_NOALLOC_CHUNK);
	if (prec == PHASE2_PREC_FP64)
		k_reduce_partial<<<blocks, P2_RED_TPB, 0, s>>>(
			(const double2 *)d_state, NULL, namp, part);
	else
		k_reduce_partial<<<blocks, P2_RED_TPB, 0, s>>>(
			(const float2 *)d_state, NULL, namp, part);
	k_reduce_final<<<1, P2_RED_TPB, 0, s>>>(part, blocks, d_out);
	CUDA_OK(cudaGetLastError(), "phase2_norm2_noalloc: launch");
	return 0;
}
