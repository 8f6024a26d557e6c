/*
 * engine.cu -- device side of libphase2.so for sm_100a (B200).
 *
 * The state vector is one flat array of 2^n complex amplitudes in HBM,
 * complex128 (double2) or complex64 (float2), updated in place.
 *
 * Hot kernel: k_pass<M, Storage, EXACT>.  One launch = one HBM sweep that
 * applies a planned run of rotations (plan.c).  Each thread owns whole
 * cosets x + span(basis[0..M-1]): it loads the 2^M amplitudes of a coset
 * into FP64 registers, applies every rotation of the run in order (partners
 * of a rotation are always inside the coset), and writes them back.  Warp
 * lanes take consecutive representatives x, so for each slot the warp
 * touches one contiguous 256 B (FP32) or 512 B (FP64) segment: coalesced,
 * one read and one write of every amplitude per pass, no shared-memory
 * staging of amplitudes.  It is a streaming pair sweep on CUDA cores; there
 * is no contraction for the tensor cores to do.
 *
 * EXACT (FP64 storage): products and sums are rounded separately with
 * __dmul_rn/__dadd_rn, never fused, so every amplitude is bit-identical to
 * the reference CPU update a_i <- c a_i + i conj(s z) a_j
 * (phase2/qreg_qreg.c:149-160).  FP32 storage computes in FP64 with FMA and
 * rounds to FP32 once per pass.
 *
 * Other kernels: gather/scatter of a few amplitudes (overlap, state prep),
 * and a two-stage FP64 sum of squares / inner product (warp-shuffle tree
 * per block, then one block combining the per-block partials with
 * Neumaier compensated summation).
 */
#include <cuda_runtime.h>

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <type_traits>

#define LOG_SUBSYS "engine"
#include "log.h"

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

	int timing;
	cudaEvent_t t0, t1;

	uint64_t rotations, passes, launches, timed_passes;
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

template <bool EXACT>
__device__ __forceinline__ double p2_mul(double a, double b)
{
	if constexpr (EXACT)
		return __dmul_rn(a, b);
	else
		return a * b;
}

/* c*x + t: two roundings (EXACT) or one (FMA). */
template <bool EXACT>
__device__ __forceinline__ double p2_cxt(double c, double x, double t)
{
	if constexpr (EXACT)
		return __dadd_rn(__dmul_rn(c, x), t);
	else
		return fma(c, x, t);
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
template <int M, int U, int ODD, bool EXACT>
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
				tr = p2_mul<EXACT>(-su, im[u]);
				ti = p2_mul<EXACT>(su, re[u]);
			} else {
				tr = p2_mul<EXACT>(su, re[u]);
				ti = p2_mul<EXACT>(su, im[u]);
			}
			re[u] = p2_cxt<EXACT>(c, re[u], tr);
			im[u] = p2_cxt<EXACT>(c, im[u], ti);
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
				tur = p2_mul<EXACT>(-su, im[w]);
				tui = p2_mul<EXACT>(su, re[w]);
				twr = p2_mul<EXACT>(-sw, im[u]);
				twi = p2_mul<EXACT>(sw, re[u]);
			} else {
				tur = p2_mul<EXACT>(su, re[w]);
				tui = p2_mul<EXACT>(su, im[w]);
				twr = p2_mul<EXACT>(sw, re[u]);
				twi = p2_mul<EXACT>(sw, im[u]);
			}
			const double nur = p2_cxt<EXACT>(c, re[u], tur);
			const double nui = p2_cxt<EXACT>(c, im[u], tui);
			const double nwr = p2_cxt<EXACT>(c, re[w], twr);
			const double nwi = p2_cxt<EXACT>(c, im[w], twi);
			re[u] = nur;
			im[u] = nui;
			re[w] = nwr;
			im[w] = nwi;
		}
	}
}

/*
 * Scaled rotation (FP32 storage).  All amplitudes carry a common pending
 * factor, applied once per pass at the store, so one FMA per component:
 *   COT = 0:  y_u <- y_u + (+-r) p_u          (r = s/c, factor c)
 *   COT = 1:  y_u <- r y_u + (+-1) p_u        (r = c/s, factor s)
 * p_u = y_{u^U}, times i when ODD; the sign is bit u of sm.
 */
template <int M, int U, int ODD, int COT>
__device__ __forceinline__ void p2_rot_scaled(double (&re)[1 << M],
	double (&im)[1 << M], double r, uint32_t sm, uint32_t W)
{
	(void)W;
	if constexpr (U == 0) {
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			const uint32_t sg = p2_bitmask(sm, u);
			const double pr = ODD ? -im[u] : re[u];
			const double pi = ODD ? re[u] : im[u];
			if constexpr (!COT) {
				const double ru = p2_sgn(r, sg);
				re[u] = fma(ru, pr, re[u]);
				im[u] = fma(ru, pi, im[u]);
			} else {
				re[u] = fma(r, re[u], p2_sgn(pr, sg));
				im[u] = fma(r, im[u], p2_sgn(pi, sg));
			}
		}
	} else {
		constexpr int H = p2_hibit(U);
#pragma unroll
		for (int k = 0; k < (1 << (M - 1)); ++k) {
			const int u = p2_ins0(k, H);
			const int w = u ^ U;
			const uint32_t sg = p2_bitmask(sm, u);
			const uint32_t sw = p2_bitmask(sm, w);
			const double pur = ODD ? -im[w] : re[w];
			const double pui = ODD ? re[w] : im[w];
			const double pwr = ODD ? -im[u] : re[u];
			const double pwi = ODD ? re[u] : im[u];
			double nur, nui, nwr, nwi;
			if constexpr (!COT) {
				const double ru = p2_sgn(r, sg), rw = p2_sgn(r, sw);
				nur = fma(ru, pur, re[u]);
				nui = fma(ru, pui, im[u]);
				nwr = fma(rw, pwr, re[w]);
				nwi = fma(rw, pwi, im[w]);
			} else {
				nur = fma(r, re[u], p2_sgn(pur, sg));
				nui = fma(r, im[u], p2_sgn(pui, sg));
				nwr = fma(r, re[w], p2_sgn(pwr, sw));
				nwi = fma(r, im[w], p2_sgn(pwi, sw));
			}
			re[u] = nur;
			im[u] = nui;
			re[w] = nwr;
			im[w] = nwi;
		}
	}
}

#define P2_CASE_S(K)                                                           \
	case K:                                                                \
		if constexpr ((K) < (4 << M))                                  \
			p2_rot_scaled<M, ((K) >> 2), (((K) >> 1) & 1),         \
				((K)&1)>(re, im, r, sm, W);                    \
		break;
#define P2_CASE_S8(B)                                                          \
	P2_CASE_S(B + 0) P2_CASE_S(B + 1) P2_CASE_S(B + 2) P2_CASE_S(B + 3)    \
	P2_CASE_S(B + 4) P2_CASE_S(B + 5) P2_CASE_S(B + 6) P2_CASE_S(B + 7)

/* key = U << 2 | odd << 1 | cot */
template <int M>
__device__ __forceinline__ void p2_apply_scaled(uint32_t key,
	double (&re)[1 << M], double (&im)[1 << M], double r, uint32_t sm,
	uint32_t W)
{
	switch (key) {
		P2_CASE_S8(0) P2_CASE_S8(8) P2_CASE_S8(16) P2_CASE_S8(24)
		P2_CASE_S8(32) P2_CASE_S8(40) P2_CASE_S8(48) P2_CASE_S8(56)
		P2_CASE_S8(64) P2_CASE_S8(72) P2_CASE_S8(80) P2_CASE_S8(88)
		P2_CASE_S8(96) P2_CASE_S8(104) P2_CASE_S8(112) P2_CASE_S8(120)
	default:
		break;
	}
}
#undef P2_CASE_S8
#undef P2_CASE_S

#define P2_CASE(K)                                                             \
	case K:                                                                \
		if constexpr ((K) < (2 << M))                                  \
			p2_rot<M, ((K) >> 1), ((K)&1), EXACT>(re, im, c, s,    \
				sm, W);                                        \
		break;

/* key = U << 1 | odd; a jump table over the (U, odd) variants. */
template <int M, bool EXACT>
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

/* Threads per block: 128, except FP64 with 32 slots per thread (64 keeps
 * three blocks of two prefetch stages within shared memory). */
__host__ __device__ constexpr int p2_tpb(int m, int elem_bytes)
{
	return (m >= 5 && elem_bytes == 16) ? 64 : P2_TPB;
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
__device__ __forceinline__ void p2_cp_async(float2 *smem, const float2 *g)
{
	const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
	asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s),
		"l"(g)
		: "memory");
}

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

/* The run of rotations of one pass on one coset held in registers, then
 * the pass-wide factor of the scaled forms. */
template <int M, bool EXACT>
__device__ __forceinline__ void p2_apply_run(double (&re)[1 << M],
	double (&im)[1 << M], uint64_t x, const struct phase2_rot_rec *srec,
	uint32_t nrot, double scale)
{
	for (uint32_t r = 0; r < nrot; ++r) {
		const uint64_t z = srec[r].z;
		const uint32_t px = (uint32_t)(__popcll(x & z) & 1);
		const uint32_t sm = srec[r].smask ^ (0u - px);
		if constexpr (EXACT) {
			const uint32_t key =
				((uint32_t)srec[r].U << 1) | srec[r].odd;
			p2_apply<M, EXACT>(key, re, im, srec[r].c, srec[r].s,
				sm, srec[r].W);
		} else {
			const uint32_t key = ((uint32_t)srec[r].U << 2) |
				((uint32_t)srec[r].odd << 1) |
				(srec[r].form == 2 ? 1u : 0u);
			p2_apply_scaled<M>(key, re, im, srec[r].c, sm,
				srec[r].W);
		}
	}
	if constexpr (!EXACT) {
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			re[u] *= scale;
			im[u] *= scale;
		}
	}
}

/* Stage layout [slot][thread]: a warp's accesses to one slot are 32
 * consecutive elements, conflict-free. */
template <int M, typename ST>
__device__ __forceinline__ void p2_prefetch(ST *stage, const ST *st,
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
template <int M, typename ST, bool EXACT>
__global__ void __launch_bounds__(p2_tpb(M, sizeof(ST)), p2_min_blocks(M))
	k_pass_pf(ST *__restrict__ st, uint64_t nrep, struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs)
{
	extern __shared__ __align__(16) unsigned char p2_dyn[];
	ST *const stage = (ST *)p2_dyn;
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
		const ST *const mine = stage + cur * nst + threadIdx.x;
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			const ST v = mine[u * blockDim.x];
			re[u] = (double)v.x;
			im[u] = (double)v.y;
		}

		p2_apply_run<M, EXACT>(re, im, x, srec, p.nrot, p.scale);
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
template <int M, typename ST, bool EXACT>
__global__ void __launch_bounds__(P2_TPB,
	(M >= 5 && sizeof(ST) == 8) ? 3 : p2_min_blocks(M))
	k_pass(ST *__restrict__ st, uint64_t nrep, struct phase2_pass p,
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
		p2_apply_run<M, EXACT>(re, im, x, srec, p.nrot, p.scale);
#pragma unroll
		for (int u = 0; u < (1 << M); ++u)
			p2_st(st, x ^ p2_slot_off<M>(u, sbasis), re[u], im[u]);
	}
}

/* ---- split pass kernel (FP32 storage) ----------------------------------- */

/* y <- y + (+-r) p  or  y <- r y + (+-1) p, p = partner (times i if ODD) */
template <int ODD, int COT>
__device__ __forceinline__ void p2_split_upd(double &yr, double &yi,
	double qr, double qi, double r, uint32_t sg)
{
	const double pr = ODD ? -qi : qr;
	const double pi = ODD ? qr : qi;
	if constexpr (!COT) {
		const double rv = p2_sgn(r, sg);
		yr = fma(rv, pr, yr);
		yi = fma(rv, pi, yi);
	} else {
		yr = fma(r, yr, p2_sgn(pr, sg));
		yi = fma(r, yi, p2_sgn(pi, sg));
	}
}

/*
 * Scaled rotation on a coset shared by two adjacent lanes: this lane holds
 * the 2^(M-1) slots whose top slot bit equals its lane parity (`half`);
 * slot u = v | half << (M-1).  A rotation whose partner stays in the lane
 * (top bit of U clear) is the ordinary pair update on the local slots;
 * otherwise every local slot's partner is fetched from the other lane with
 * one shuffle per component and each lane updates only its own slots.
 * sm holds this lane's signs (bit v = sign of local slot v).
 */
template <int M, int U, int ODD, int COT>
__device__ __forceinline__ void p2_rot_split(double (&re)[1 << (M - 1)],
	double (&im)[1 << (M - 1)], double r, uint32_t sm, unsigned mask)
{
	constexpr int MH = M - 1;
	constexpr int TOP = 1 << MH;
	if constexpr ((U & TOP) == 0) {
		p2_rot_scaled<MH, U, ODD, COT>(re, im, r, sm, 0u);
	} else {
		/* Local slots v and v ^ UL exchange with the other lane's
		 * v ^ UL and v: fetch both before either is overwritten. */
		constexpr int UL = U & (TOP - 1);
#pragma unroll
		for (int v = 0; v < (1 << MH); ++v) {
			const int v2 = v ^ UL;
			if (v2 < v)
				continue;
			const double ar = __shfl_xor_sync(mask, re[v2], 1);
			const double ai = __shfl_xor_sync(mask, im[v2], 1);
			double br = 0.0, bi = 0.0;
			if (v2 != v) {
				br = __shfl_xor_sync(mask, re[v], 1);
				bi = __shfl_xor_sync(mask, im[v], 1);
			}
			p2_split_upd<ODD, COT>(re[v], im[v], ar, ai, r,
				p2_bitmask(sm, v));
			if (v2 != v)
				p2_split_upd<ODD, COT>(re[v2], im[v2], br, bi, r,
					p2_bitmask(sm, v2));
		}
	}
}

#define P2_CASE_P(K)                                                           \
	case K:                                                                \
		if constexpr ((K) < (4 << M))                                  \
			p2_rot_split<M, ((K) >> 2), (((K) >> 1) & 1),          \
				((K)&1)>(re, im, r, sm, mask);                 \
		break;
#define P2_CASE_P8(B)                                                          \
	P2_CASE_P(B + 0) P2_CASE_P(B + 1) P2_CASE_P(B + 2) P2_CASE_P(B + 3)    \
	P2_CASE_P(B + 4) P2_CASE_P(B + 5) P2_CASE_P(B + 6) P2_CASE_P(B + 7)

template <int M>
__device__ __forceinline__ void p2_apply_split(uint32_t key,
	double (&re)[1 << (M - 1)], double (&im)[1 << (M - 1)], double r,
	uint32_t sm, unsigned mask)
{
	switch (key) {
		P2_CASE_P8(0) P2_CASE_P8(8) P2_CASE_P8(16) P2_CASE_P8(24)
		P2_CASE_P8(32) P2_CASE_P8(40) P2_CASE_P8(48) P2_CASE_P8(56)
		P2_CASE_P8(64) P2_CASE_P8(72) P2_CASE_P8(80) P2_CASE_P8(88)
		P2_CASE_P8(96) P2_CASE_P8(104) P2_CASE_P8(112) P2_CASE_P8(120)
	default:
		break;
	}
}
#undef P2_CASE_P8
#undef P2_CASE_P

/*
 * One FP32 pass with each coset shared by a lane pair (variant 2): half
 * the registers per thread of k_pass, so twice the resident warps to hide
 * load and arithmetic latency.  Both lanes of a pair always have the same
 * representative, so they enter and leave the loop together and every
 * shuffle pairs two active lanes.
 */
template <int M>
__global__ void __launch_bounds__(P2_TPB, M >= 5 ? 4 : 6)
	k_pass_split(float2 *__restrict__ st, uint64_t nrep,
		struct phase2_pass p,
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
	constexpr int MH = M - 1;
	const uint32_t half = threadIdx.x & 1u;
	uint64_t pb[MH > 0 ? MH : 1];
#pragma unroll
	for (int k = 0; k < MH; ++k)
		pb[k] = p.basis[k];
	const uint64_t top = half ? p.basis[MH] : 0;

	const uint64_t stride = ((uint64_t)gridDim.x * blockDim.x) >> 1;
	for (uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 1;
		t < nrep; t += stride) {
		const unsigned mask = __activemask();
		const uint64_t x = p2_rep<M>(t, p) ^ top;
		double re[1 << MH], im[1 << MH];
#pragma unroll
		for (int v = 0; v < (1 << MH); ++v)
			p2_ld(st, x ^ p2_slot_off<MH>(v, pb), re[v], im[v]);
		for (uint32_t r = 0; r < p.nrot; ++r) {
			const uint64_t z = srec[r].z;
			const uint32_t px = (uint32_t)(__popcll(x & z) & 1);
			/* x includes the top basis vector for the upper lane, so
			 * px already carries parity(top & z): local sign bits are
			 * the lower half of smask with that parity folded in */
			uint32_t sm = srec[r].smask;
			if (half)
				sm = (sm >> (1u << MH)) ^
					(((uint32_t)__popcll(top & z) & 1u) ?
							0xffffffffu : 0u);
			sm ^= 0u - px;
			const uint32_t key = ((uint32_t)srec[r].U << 2) |
				((uint32_t)srec[r].odd << 1) |
				(srec[r].form == 2 ? 1u : 0u);
			p2_apply_split<M>(key, re, im, srec[r].c, sm, mask);
		}
#pragma unroll
		for (int v = 0; v < (1 << MH); ++v) {
			re[v] *= p.scale;
			im[v] *= p.scale;
		}
		const uint64_t xs = p2_rep<M>(t, p) ^
			(half ? sbasis[MH] : UINT64_C(0));
#pragma unroll
		for (int v = 0; v < (1 << MH); ++v)
			p2_st(st, xs ^ p2_slot_off<MH>(v, sbasis), re[v], im[v]);
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
	double vr = p2_warp_sum(sr + cr), vi = p2_warp_sum(si + ci);
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
 * Launch table: per precision and span, which pass kernel runs (0 direct,
 * 1 shared-memory prefetch) and how many blocks per SM the grid holds
 * (0: the direct kernel's default of 16, the prefetch kernel's occupancy).
 * Set by phase2_tune_set (the autotuner) or left at these defaults.
 */
struct p2_tune_entry {
	int variant;
	int per_sm;
};
static struct p2_tune_entry p2_tune[2][PHASE2_MAX_SPAN + 1] = {
	/* FP64: direct loads, 32 blocks per SM (measured 93-96 % of HBM
	 * peak for every span at 28 qubits on B200) */
	{ { 0, 32 }, { 0, 32 }, { 0, 32 }, { 0, 32 }, { 0, 32 }, { 0, 32 } },
	/* FP32: prefetch for spans 2-4, direct for 0, 1 and 5 */
	{ { 0, 32 }, { 0, 32 }, { 1, 0 }, { 1, 0 }, { 1, 0 }, { 0, 32 } },
};

extern "C" int phase2_tune_set(int prec, int span, int variant, int per_sm)
{
	if ((prec != PHASE2_PREC_FP64 && prec != PHASE2_PREC_FP32) || span < 0 ||
		span > PHASE2_MAX_SPAN || variant < 0 || variant > 2 ||
		per_sm < 0 || per_sm > 64)
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

template <int M, typename ST, bool EXACT>
static int launch_pass_t(struct p2_dev *d, const struct phase2_pass &p,
	const struct phase2_rot_rec *recs)
{
	const uint64_t nrep = d->namp >> M;
	const struct p2_tune_entry te = p2_tune[d->prec][M];
	if constexpr (std::is_same<ST, float2>::value && M >= 2) {
		if (te.variant == 2) {
			const unsigned per_sm = te.per_sm ? (unsigned)te.per_sm : 16u;
			const unsigned grid = grid_for(d, 2 * nrep, P2_TPB, per_sm);
			k_pass_split<M><<<grid, P2_TPB, 0, d->stream>>>(
				(float2 *)d->state, nrep, p, recs);
			return 0;
		}
	}
	if (te.variant != 1) {
		const unsigned per_sm = te.per_sm ? (unsigned)te.per_sm : 16u;
		const unsigned grid = grid_for(d, nrep, P2_TPB, per_sm);
		k_pass<M, ST, EXACT><<<grid, P2_TPB, 0, d->stream>>>(
			(ST *)d->state, nrep, p, recs);
		return 0;
	}
	static struct p2_kcfg cfg;
	if (!cfg.ready) {
		cfg.tpb = p2_tpb(M, (int)sizeof(ST));
		cfg.smem = 2 * ((size_t)1 << M) * cfg.tpb * sizeof(ST);
		CUDA_OK(cudaFuncSetAttribute(k_pass_pf<M, ST, EXACT>,
				cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)cfg.smem),
			"pass kernel shared memory");
		int per_sm = 0;
		CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
				k_pass_pf<M, ST, EXACT>, cfg.tpb, cfg.smem),
			"pass kernel occupancy");
		cfg.per_sm = per_sm > 0 ? per_sm : 1;
		cfg.ready = 1;
	}
	const unsigned per_sm = te.per_sm && te.per_sm < cfg.per_sm
		? (unsigned)te.per_sm
		: (unsigned)cfg.per_sm;
	const unsigned grid = grid_for(d, nrep, (unsigned)cfg.tpb, per_sm);
	k_pass_pf<M, ST, EXACT><<<grid, cfg.tpb, cfg.smem, d->stream>>>(
		(ST *)d->state, nrep, p, recs);
	return 0;
}

template <typename ST, bool EXACT>
static int launch_pass(struct p2_dev *d, const struct phase2_pass &p,
	const struct phase2_rot_rec *recs)
{
	switch (p.span) {
	case 0:
		return launch_pass_t<0, ST, EXACT>(d, p, recs);
	case 1:
		return launch_pass_t<1, ST, EXACT>(d, p, recs);
	case 2:
		return launch_pass_t<2, ST, EXACT>(d, p, recs);
	case 3:
		return launch_pass_t<3, ST, EXACT>(d, p, recs);
	case 4:
		return launch_pass_t<4, ST, EXACT>(d, p, recs);
	case 5:
		return launch_pass_t<5, ST, EXACT>(d, p, recs);
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

static int launch_all(struct p2_dev *d, const struct phase2_pass *passes,
	size_t npass, const struct phase2_rot_rec *d_recs)
{
	for (size_t i = 0; i < npass; i++) {
		const int rc = d->prec == PHASE2_PREC_FP64
			? launch_pass<double2, true>(d, passes[i], d_recs)
			: launch_pass<float2, false>(d, passes[i], d_recs);
		if (rc < 0)
			return -1;
	}
	return 0;
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
			const int rc = launch_all(d, passes, npass, g->d_recs);
			const cudaError_t e = cudaStreamEndCapture(d->stream,
				&graph);
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
	if (g) {
		CUDA_OK(cudaGraphLaunch(g->exec, d->stream), "graph launch");
		d->graph_replays++;
	} else if (launch_all(d, passes, npass, d->d_recs) < 0) {
		return -1;
	}
	CUDA_OK(cudaGetLastError(), "pass launch");
	d->passes += npass;
	d->launches += npass;
	d->rotations += nrec;
	if (d->timing) {
		CUDA_OK(cudaEventRecord(d->t1, d->stream), "timing stop");
		CUDA_OK(cudaEventSynchronize(d->t1), "timing wait");
		float ms = 0.0f;
		CUDA_OK(cudaEventElapsedTime(&ms, d->t0, d->t1), "elapsed");
		d->pass_ms += ms;
		d->timed_passes += npass;
	}
	return 0;
}

static int reduce(struct p2_dev *d, const double2 *trial, double out[2])
{
	const unsigned blocks = grid_for(d, d->namp, P2_RED_TPB, 4);
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
	if (d->prec == PHASE2_PREC_FP64)
		k_reduce_partial<<<blocks, P2_RED_TPB, 0, d->stream>>>(
			(const double2 *)d->state, trial, d->namp, d->d_part);
	else
		k_reduce_partial<<<blocks, P2_RED_TPB, 0, d->stream>>>(
			(const float2 *)d->state, trial, d->namp, d->d_part);
	k_reduce_final<<<1, P2_RED_TPB, 0, d->stream>>>(d->d_part, blocks,
		d->d_part + 2 * (size_t)blocks);
	d->launches += 2;
	CUDA_OK(cudaGetLastError(), "reduce launch");
	double h[2];
	CUDA_OK(cudaMemcpyAsync(h, d->d_part + 2 * (size_t)blocks, sizeof h,
			cudaMemcpyDeviceToHost, d->stream),
		"download reduction");
	CUDA_OK(cudaStreamSynchronize(d->stream), "reduce");
	out[0] = h[0];
	out[1] = h[1];
	return 0;
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
	st->bytes = d->passes * 2 * d->namp * d->elem;
	st->timed_passes = d->timed_passes;
	st->pass_ms = d->pass_ms;
	st->h2d_bytes = d->h2d_bytes;
	st->d2h_bytes = d->d2h_bytes;
	st->graph_replays = d->graph_replays;
}

extern "C" void p2d_stats_reset(struct p2_dev *d)
{
	d->rotations = d->passes = d->launches = d->timed_passes = 0;
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
