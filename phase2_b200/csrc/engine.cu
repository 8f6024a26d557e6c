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
 *
 * The device helpers these kernels share live in p2_kernels.cuh; the
 * persistent kernel is in batch.cu, device sampling in sampling.cu and
 * sweeps in sweep.cu.
 */
#include <cuda_runtime.h>

#include <float.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "engine"
#include "log.h"

#include "p2_kernels.cuh"

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

/* ---- mixed form: FP32 arithmetic, FP64 on heavy cosets ------------------ */

/* A coset is heavy when one of its amplitudes has |re| or |im| >= this at
 * the start of the pass.  Below it, the absolute error of an FP32 shear
 * (half an ulp) is at most 2^-35. */
#define P2_HEAVY_MIN 0x1p-10f

/* Registers below this many qubits run mixed-form passes on the FP64-
 * arithmetic kernels: a spread state of n qubits has components of
 * standard deviation 2^-(n+1)/2, which reach P2_HEAVY_MIN often below 24
 * qubits (at 22, a quarter of the cosets), and a heavy coset costs its
 * warp a serial FP64 run; at 24 the threshold is 5.7 deviations away. */
#define P2_MIXED_MIN_QB 24

/*
 * The run of rotations on one coset held in shared memory as FP64 (hv: 2^M
 * slots), by the whole warp: lane j rotates pair j (slot u with a zero at
 * the top bit of U, and u ^ U) by the three shears of p2_rot_lift32 in FP64
 * FMAs, or slot j when the string is diagonal on the coset (U = 0).  t is
 * the record's FP64 t and s its FP32 s (exact in FP64); x is the coset's
 * representative (the signs).  Every lane of the warp calls it.
 */
template <int M, typename IT>
__device__ __forceinline__ void p2_heavy_run(double2 *hv, IT x,
	const struct p2_lift32_rec *srec, const double *tt, uint32_t nrot,
	uint32_t lane)
{
	for (uint32_t r = 0; r < nrot; ++r) {
		const struct p2_lift32_rec q = srec[r];
		const uint32_t sm = q.sm ^ (0u - p2_parity(x & (IT)q.z));
		const uint32_t U = q.key >> 1, odd = q.key & 1u;
		const double t = tt[r], s = (double)q.s;
		if (U == 0) {
			if (lane < (1u << M)) {
				const uint32_t b = p2_bitmask(sm, (int)lane);
				const double st = p2_sgn(t, b), ss = p2_sgn(s, b);
				double2 y = hv[lane];
				if (odd) {
					y.x = fma(-st, y.y, y.x);
					y.y = fma(ss, y.x, y.y);
					y.x = fma(-st, y.y, y.x);
				} else {
					const double k = ss + fma(-t, s, 1.0);
					y.x *= k;
					y.y *= k;
				}
				hv[lane] = y;
			}
		} else if (M > 0 && U < (1u << M) &&
			lane < (1u << (M > 0 ? M - 1 : 0))) {
			const uint32_t h = 31u - (uint32_t)__clz(U);
			const uint32_t u = ((lane >> h) << (h + 1)) |
				(lane & ((1u << h) - 1u));
			const uint32_t w = u ^ U;
			const uint32_t b = p2_bitmask(sm, (int)u);
			const double st = p2_sgn(t, b), ss = p2_sgn(s, b);
			double2 yu = hv[u], yw = hv[w];
			if (odd) {
				yu.x = fma(-st, yw.y, yu.x);
				yu.y = fma(st, yw.x, yu.y);
				yw.x = fma(-ss, yu.y, yw.x);
				yw.y = fma(ss, yu.x, yw.y);
				yu.x = fma(-st, yw.y, yu.x);
				yu.y = fma(st, yw.x, yu.y);
			} else {
				yu.x = fma(st, yw.x, yu.x);
				yu.y = fma(st, yw.y, yu.y);
				yw.x = fma(-ss, yu.x, yw.x);
				yw.y = fma(-ss, yu.y, yw.y);
				yu.x = fma(st, yw.x, yu.x);
				yu.y = fma(st, yw.y, yu.y);
			}
			hv[u] = yu;
			hv[w] = yw;
		}
		__syncwarp();
	}
}

/*
 * One FP32 pass in the mixed form.  Each thread loads its coset into FP32
 * registers (as k_pass_lift32); a thread whose coset holds an amplitude of
 * magnitude >= P2_HEAVY_MIN hands it to its warp, which rotates it in FP64
 * in shared memory (p2_heavy_run) and rounds once; the other threads apply
 * the run with FP32 FMAs, the same bits as k_pass_lift32.  The warps walk
 * the cosets 32 at a time, so every lane is present for the heavy runs.
 */
template <int M, typename IT>
__global__ void __launch_bounds__(P2_TPB, p2_lift32_blocks(M))
	k_pass_lift32h(float2 *__restrict__ st, uint64_t nrep,
		struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs)
{
	constexpr int S = 1 << M;
	constexpr unsigned FULL = 0xffffffffu;
	__shared__ struct p2_lift32_rec srec[P2_MAX_ROTS_PER_PASS];
	__shared__ double tt[P2_MAX_ROTS_PER_PASS];
	__shared__ double2 hv_all[P2_TPB / 32][S];
	for (uint32_t r = threadIdx.x; r < p.nrot; r += blockDim.x) {
		srec[r] = p2_lift32_of(recs[p.rot_off + r]);
		tt[r] = recs[p.rot_off + r].c;
	}
	__syncthreads();
	IT pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = (IT)p.basis[k];
	const uint32_t negm = p.scale < 0 ? 0x80000000u : 0u;
	const uint32_t nrot = p.nrot;
	const uint32_t lane = threadIdx.x & 31u;
	double2 *const hv = hv_all[threadIdx.x >> 5];

	const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x +
			(threadIdx.x & ~31u);
		t0 < nrep; t0 += stride) {
		const uint64_t t = t0 + lane;
		const bool active = t < nrep;
		const IT x = p2_rep_t<M, IT>((IT)t, p);
		float re[S], im[S];
		float mx = 0.f;
#pragma unroll
		for (int u = 0; u < S; ++u) {
			IT off = 0;
#pragma unroll
			for (int k = 0; k < M; ++k)
				if (u >> k & 1)
					off ^= pb[k];
			const float2 v = active ? st[x ^ off]
						: make_float2(0.f, 0.f);
			re[u] = v.x;
			im[u] = v.y;
			mx = fmaxf(mx, fmaxf(fabsf(v.x), fabsf(v.y)));
		}
		const bool heavy = active && mx >= P2_HEAVY_MIN;
		unsigned hm = __ballot_sync(FULL, heavy);
		while (hm) {
			const int src = __ffs(hm) - 1;
			hm &= hm - 1;
			const IT hx = __shfl_sync(FULL, x, src);
			if (lane == (uint32_t)src) {
#pragma unroll
				for (int u = 0; u < S; ++u)
					hv[u] = make_double2((double)re[u],
						(double)im[u]);
			}
			__syncwarp();
			p2_heavy_run<M, IT>(hv, hx, srec, tt, nrot, lane);
			if (lane == (uint32_t)src) {
#pragma unroll
				for (int u = 0; u < S; ++u) {
					re[u] = __double2float_rn(hv[u].x);
					im[u] = __double2float_rn(hv[u].y);
				}
			}
			__syncwarp();
		}
		if (active && !heavy) {
			for (uint32_t r = 0; r < nrot; ++r) {
				const struct p2_lift32_rec q = srec[r];
				const uint32_t sm =
					q.sm ^ (0u - p2_parity(x & (IT)q.z));
				p2_apply_lift32<M>(q, re, im, sm);
			}
		}
		if (active) {
			const IT xs = p2_opaque(x);
#pragma unroll
			for (int u = 0; u < S; ++u) {
				IT off = 0;
#pragma unroll
				for (int k = 0; k < M; ++k)
					if (u >> k & 1)
						off ^= pb[k];
				st[xs ^ off] = make_float2(p2_fsgn(re[u], negm),
					p2_fsgn(im[u], negm));
			}
		}
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

extern "C" int p2d_device_name(char *buf, size_t n)
{
	int dev = 0;
	cudaDeviceProp prop;
	if (!buf || n == 0 || cudaGetDevice(&dev) != cudaSuccess ||
		cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
		cudaGetLastError();
		return -1;
	}
	snprintf(buf, n, "%s", prop.name);
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
	/* memory the pool holds but does not use can serve the state too */
	size_t pooled = 0;
	cudaMemPool_t pool;
	uint64_t reserved = 0, used = 0;
	if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
		cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent,
			&reserved) == cudaSuccess &&
		cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent,
			&used) == cudaSuccess &&
		reserved > used)
		pooled = (size_t)(reserved - used);
	cudaGetLastError();
	if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
		bytes > free_b + pooled) {
		log_error("p2d_create: state of %zu bytes exceeds free device"
			  " memory (%zu bytes)",
			bytes, free_b);
		free(d);
		return NULL;
	}
	if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) !=
		cudaSuccess)
		goto fail;
	/* stream-ordered from the default pool (p2_scratch_alloc): creating
	 * and destroying many registers (batches) reuses memory instead of
	 * mapping and unmapping it each time */
	if (p2_scratch_alloc(&d->state, bytes, d->stream) != cudaSuccess) {
		d->state = NULL;
		log_error("p2d_create: allocation of %zu bytes failed", bytes);
		goto fail;
	}
	for (int k = 0; k < 2; k++)
		if (cudaEventCreateWithFlags(&d->h_ev[k],
			    cudaEventDisableTiming) != cudaSuccess)
			goto fail;
	if (cudaEventCreate(&d->t0) != cudaSuccess ||
		cudaEventCreate(&d->t1) != cudaSuccess)
		goto fail;
	if (cudaMalloc((void **)&d->d_status, sizeof *d->d_status) !=
			cudaSuccess ||
		cudaMallocHost((void **)&d->h_status, sizeof *d->h_status) !=
			cudaSuccess ||
		cudaMemsetAsync(d->d_status, 0, sizeof *d->d_status,
			d->stream) != cudaSuccess)
		goto fail;
	*d->h_status = 0;
	if (cudaMemsetAsync(d->state, 0, bytes, d->stream) != cudaSuccess)
		goto fail;
	/* the state is ready for any stream from here on */
	if (cudaStreamSynchronize(d->stream) != cudaSuccess)
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
	if (d->state)
		p2_scratch_free(d->state, d->stream);
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
	cudaFree(d->d_status);
	cudaFreeHost(d->h_status);
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

int p2_status_check(struct p2_dev *d)
{
	if (!d->status_pending)
		return 0;
	CUDA_OK(cudaMemcpyAsync(d->h_status, d->d_status, sizeof *d->h_status,
			cudaMemcpyDeviceToHost, d->stream),
		"read kernel status");
	CUDA_OK(cudaStreamSynchronize(d->stream), "kernel status");
	d->d2h_bytes += sizeof *d->h_status;
	d->status_pending = 0;
	if (*d->h_status) {
		log_error("a pass kernel gave up waiting for its staged loads "
			  "(status %u): the state is not valid",
			*d->h_status);
		*d->h_status = 0;
		CUDA_OK(cudaMemsetAsync(d->d_status, 0, sizeof *d->d_status,
				d->stream),
			"clear kernel status");
		return -1;
	}
	return 0;
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
	return p2_status_check(d);
}

extern "C" int p2d_get_state(struct p2_dev *d, double *out)
{
	const size_t bytes = d->namp * sizeof(double2);
	if (p2_status_check(d) < 0)
		return -1;
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
 * the prefetch kernel).  FP32: the lifted kernels; for passes of the
 * FP64-arithmetic form, variants 1 and 2 run the kernels whose next
 * cosets are staged in shared memory by bulk copies or by cp.async
 * (lift_bulk.cu; per_sm caps their occupancy) where the pass qualifies,
 * variant 0 the direct kernel (per_sm 0: 16).  The
 * FP32-arithmetic form has one kernel.  Set by phase2_tune_set (the
 * autotuner) or left at these defaults.
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
	 * (phase2_b200/tuning_b200.json, 28 qubits); FP64-arithmetic passes
	 * of span 3-5 staged by cp.async (30 qubits: 4.89 TB/s against 4.79
	 * direct and 4.58 bulk-copy staged) */
	{ { 0, 32 }, { 0, 16 }, { 0, 32 }, { 2, 32 }, { 2, 32 }, { 2, 32 } },
};

extern "C" int phase2_tune_set(int prec, int span, int variant, int per_sm)
{
	if ((prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32) || span < 0 ||
		span > PHASE2_MAX_SPAN || variant < 0 ||
		variant > (prec == PHASE2_PREC_FP64 ? 1 : 3) || per_sm < 0 ||
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
	} else if (p.form == PHASE2_FORM_LIFTED_MIXED &&
		d->nqb >= P2_MIXED_MIN_QB) {
		if (narrow)
			k_pass_lift32h<M, uint32_t>
				<<<grid, P2_TPB, 0, d->stream>>>(sv, nrep, p, recs);
		else
			k_pass_lift32h<M, uint64_t>
				<<<grid, P2_TPB, 0, d->stream>>>(sv, nrep, p, recs);
	} else if (p.form == PHASE2_FORM_LIFTED ||
		p.form == PHASE2_FORM_LIFTED_MIXED) {
		/* mixed-form passes of smaller registers: FP64 arithmetic on
		 * every coset (their records are the FP32 form's) */
		/* variants 1 and 2: the next cosets staged in shared memory by
		 * bulk copies or cp.async (lift_bulk.cu), where the pass
		 * qualifies */
		if (te.variant != 0) {
			const int rc = p2_lift_staged_launch(d, &p, recs,
				te.variant, (unsigned)te.per_sm);
			if (rc != 0)
				return rc < 0 ? -1 : 0;
		}
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

/* Launch a plan: planned sweeps as one kernel each (sweep.cu), other
 * passes one kernel each.  Returns the kernels launched (state round
 * trips) or -1. */
static long launch_all(struct p2_dev *d, const struct phase2_pass *passes,
	size_t npass, const struct phase2_rot_rec *d_recs)
{
	const bool sweeps = p2_sweeps_on(d);
	long launches = 0;
	for (size_t i = 0; i < npass; launches++) {
		long n = sweeps ? p2_sweep_launch(d, passes, npass, i, d_recs)
				: 1;
		if (n < 0)
			return -1;
		if (n < 2) {
			if (launch_pass(d, passes[i], d_recs) < 0)
				return -1;
			n = 1;
		}
		i += (size_t)n;
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
			const int pending = d->status_pending;
			d->status_pending = 0;
			const long rc = launch_all(d, passes, npass, g->d_recs);
			g->status = d->status_pending;
			d->status_pending |= pending;
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
		d->status_pending |= g->status;
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
	return p2_status_check(d);
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
	CUDA_OK(p2_scratch_alloc((void **)&t, bytes, d->stream), "alloc trial");
	cudaError_t e = cudaMemcpyAsync(t, trial, bytes, cudaMemcpyHostToDevice,
		d->stream);
	int rc = e == cudaSuccess ? reduce(d, t, out) : -1;
	p2_scratch_free(t, d->stream);
	cudaStreamSynchronize(d->stream);
	if (e != cudaSuccess)
		log_error("upload trial: %s", cudaGetErrorString(e));
	return rc;
}

/* Device memory for a caller of the host layer (exchange buffers of
 * sharded registers), on the current device; NULL on failure. */
extern "C" void *p2d_buffer_alloc(size_t bytes)
{
	void *p = NULL;
	if (cudaMalloc(&p, bytes) != cudaSuccess) {
		cudaGetLastError();
		log_error("device buffer of %zu bytes: allocation failed", bytes);
		return NULL;
	}
	return p;
}

extern "C" void p2d_buffer_free(void *p)
{
	if (p)
		cudaFree(p);
}

extern "C" int p2d_sync(struct p2_dev *d)
{
	CUDA_OK(cudaStreamSynchronize(d->stream), "stream sync");
	CUDA_OK(cudaGetLastError(), "pending error");
	return p2_status_check(d);
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

/* ---- transient buffers --------------------------------------------------- */

cudaError_t p2_scratch_alloc(void **p, size_t bytes, cudaStream_t stream)
{
	/* once per device (devices 0..63): keep up to 1 GiB of freed memory
	 * in the device's default pool */
	static uint64_t pool_ready;
	int dev = 0;
	if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 &&
		!(pool_ready >> dev & 1)) {
		cudaMemPool_t pool;
		if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
			uint64_t keep = UINT64_C(1) << 30;
			cudaMemPoolSetAttribute(pool,
				cudaMemPoolAttrReleaseThreshold, &keep);
		}
		cudaGetLastError(); /* a pool call's failure is not the caller's */
		pool_ready |= UINT64_C(1) << dev;
	}
	return cudaMallocAsync(p, bytes, stream);
}

void p2_scratch_free(void *p, cudaStream_t stream)
{
	if (p)
		cudaFreeAsync(p, stream);
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

/* Address of the array on each device, looked up by the first call there
 * (written once with the same value by any thread that races on it). */
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
	const size_t elem =
		prec == PHASE2_PREC_FP64 ? sizeof(double2) : sizeof(float2);
	if ((uintptr_t)d_state % elem != 0 || (uintptr_t)d_out % 16 != 0) {
		log_error("phase2_norm2_noalloc: state not aligned to %zu bytes"
			  " or output not aligned to 16 bytes",
			elem);
		return -1;
	}
	/* both pointers must be memory of the current device, with the whole
	 * range inside one allocation: a host pointer or a short buffer is
	 * refused here instead of faulting in the kernel */
	if (p2_check_device_range(d_state, (size_t)namp * elem,
		    "phase2_norm2_noalloc: state") < 0 ||
		p2_check_device_range(d_out, 2 * sizeof(double),
			"phase2_norm2_noalloc: output") < 0)
		return -1;
	int dev = 0;
	CUDA_OK(cudaGetDevice(&dev), "phase2_norm2_noalloc: current device");
	if (dev < 0 || dev >= P2_NOALLOC_MAX_DEVICES) {
		log_error("phase2_norm2_noalloc: device %d beyond the %d"
			  " supported", dev, P2_NOALLOC_MAX_DEVICES);
		return -1;
	}
	double *part = __atomic_load_n(&p2_noalloc_addr[dev], __ATOMIC_ACQUIRE);
	if (!part) {
		/* first call on this device: resolve the array's address */
		CUDA_OK(cudaGetSymbolAddress((void **)&part, p2_noalloc_scratch),
			"phase2_norm2_noalloc: scratch address");
		__atomic_store_n(&p2_noalloc_addr[dev], part, __ATOMIC_RELEASE);
	}
	int sms = 0;
	if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
			cudaSuccess ||
		sms <= 0) {
		cudaGetLastError();
		sms = 148;
	}
	const cudaStream_t s = (cudaStream_t)stream;
	/* Enough blocks to stream at full bandwidth (four per SM), at least
	 * one per 2^21 amplitudes so that the array always suffices, at most
	 * one per 256 amplitudes; k_reduce_partial is a grid-stride loop, so
	 * any count gives the same sum terms.  Each block writes its own two
	 * slots before the final kernel reads them (stream order), so the
	 * array needs no clearing. */
	uint64_t blocks = (namp + P2_NOALLOC_CHUNK - 1) / P2_NOALLOC_CHUNK;
	if (blocks < (uint64_t)sms * 4)
		blocks = (uint64_t)sms * 4;
	const uint64_t per256 = (namp + P2_RED_TPB - 1) / P2_RED_TPB;
	if (blocks > per256)
		blocks = per256;
	if (blocks > P2_NOALLOC_MAX_BLOCKS)
		blocks = P2_NOALLOC_MAX_BLOCKS;
	if (prec == PHASE2_PREC_FP64)
		k_reduce_partial<<<(unsigned)blocks, P2_RED_TPB, 0, s>>>(
			(const double2 *)d_state, NULL, namp, part);
	else
		k_reduce_partial<<<(unsigned)blocks, P2_RED_TPB, 0, s>>>(
			(const float2 *)d_state, NULL, namp, part);
	k_reduce_final<<<1, P2_RED_TPB, 0, s>>>(part, (unsigned)blocks, d_out);
	CUDA_OK(cudaGetLastError(), "phase2_norm2_noalloc: launch");
	return 0;
}
