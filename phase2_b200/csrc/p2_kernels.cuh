/*
 * p2_kernels.cuh -- device code shared by the engine's kernels: the FP64
 * pair update (exact rounding) and its coset run, the FP32 lifted shears
 * and their coset run, coset enumeration, asynchronous copies, and the
 * op/tile types of the persistent kernel.  Everything here is inline or a
 * template, so each CUDA source compiles its own copy.
 */
#ifndef P2_KERNELS_CUH
#define P2_KERNELS_CUH

#include "p2_engine.h"

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

#ifndef P2_ROT_GROUP
#define P2_ROT_GROUP 1
#endif

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
		/* pairs P2_ROT_GROUP at a time, step by step (independent
		 * pairs: the same bits, more independent FP64 operations in
		 * flight where the pass is compute-bound) */
		constexpr int H = p2_hibit(U);
		constexpr int NP = 1 << (M - 1);
		constexpr int G = NP < P2_ROT_GROUP ? NP : P2_ROT_GROUP;
#pragma unroll
		for (int g0 = 0; g0 < NP; g0 += G) {
			double tur[G], tui[G], twr[G], twi[G];
#pragma unroll
			for (int j = 0; j < G; ++j) {
				const int u = p2_ins0(g0 + j, H);
				const int w = u ^ U;
				const double su = p2_sgn(s, p2_bitmask(sm, u));
				const double sw = p2_sgn(s, p2_bitmask(sm, w));
				if constexpr (ODD) {
					tur[j] = p2_mul(-su, im[w]);
					tui[j] = p2_mul(su, re[w]);
					twr[j] = p2_mul(-sw, im[u]);
					twi[j] = p2_mul(sw, re[u]);
				} else {
					tur[j] = p2_mul(su, re[w]);
					tui[j] = p2_mul(su, im[w]);
					twr[j] = p2_mul(sw, re[u]);
					twi[j] = p2_mul(sw, im[u]);
				}
			}
#pragma unroll
			for (int j = 0; j < G; ++j) {
				const int u = p2_ins0(g0 + j, H);
				const int w = u ^ U;
				const double nur = p2_cxt(c, re[u], tur[j]);
				const double nui = p2_cxt(c, im[u], tui[j]);
				const double nwr = p2_cxt(c, re[w], twr[j]);
				const double nwi = p2_cxt(c, im[w], twi[j]);
				re[u] = nur;
				im[u] = nui;
				re[w] = nwr;
				im[w] = nwi;
			}
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

/* Asynchronous global -> shared copy of 16 bytes to a shared address. */
__device__ __forceinline__ void p2_cp16(uint32_t dst, const void *src)
{
	asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst),
		"l"(src)
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

/* ---- lifted pass kernel (FP32 storage) ---------------------------------- */

/*
 * One lifted rotation on the 2^M slots of a coset.  A pair (u, w = u ^ U)
 * with sign sigma (bit u of sm) is rotated by three in-place shears,
 *   y_u += t q_u y_w;  y_w += s q_w y_u;  y_u += t q_u y_w,
 * q_u = sigma (odd ? i : 1), q_w = -conj(q_u), t = tan(phi/2): every update
 * writes the register it reads, so a case needs no temporaries and leaves
 * no moves behind.  The sign goes onto the two coefficients (one XOR on the
 * high word of each, sigma t and sigma s); the FMAs then take them with
 * free operand negations.  Rounding is symmetric under negation, so this
 * gives the same bits as flipping the partner's sign around the shears.
 * U = 0 (the string is diagonal on the coset, and then odd = 1) is the
 * phase c + i sigma s, applied to (re, im) by the same three shears.
 *
 * The three shears of a pair depend on each other, so the pairs are taken
 * P2_LIFT_GROUP at a time, shear by shear: each shear of a group is
 * 2 * P2_LIFT_GROUP independent FMAs, enough to cover the FP64 FMA latency
 * (pairs are independent, so the order gives the same bits).
 */
#ifndef P2_LIFT_GROUP
#define P2_LIFT_GROUP 2
#endif
#ifndef P2_LIFT32_GROUP
#define P2_LIFT32_GROUP 4
#endif

template <int M, int U, int ODD>
__device__ __forceinline__ void p2_rot_lift(double (&re)[1 << M],
	double (&im)[1 << M], double t, double s, uint32_t sm)
{
	if constexpr (U == 0) {
		constexpr int S = 1 << M;
		constexpr int G = S < P2_LIFT_GROUP ? S : P2_LIFT_GROUP;
#pragma unroll
		for (int g = 0; g < S; g += G) {
			double st[G], ss[G];
#pragma unroll
			for (int j = 0; j < G; ++j) {
				const uint32_t b = p2_bitmask(sm, g + j);
				st[j] = p2_sgn(t, b);
				ss[j] = p2_sgn(s, b);
			}
			if constexpr (ODD) {
#pragma unroll
				for (int j = 0; j < G; ++j)
					re[g + j] = fma(-st[j], im[g + j], re[g + j]);
#pragma unroll
				for (int j = 0; j < G; ++j)
					im[g + j] = fma(ss[j], re[g + j], im[g + j]);
#pragma unroll
				for (int j = 0; j < G; ++j)
					re[g + j] = fma(-st[j], im[g + j], re[g + j]);
			} else {
				/* (c +- s) y with c = 1 - t s; a Hermitian string
				 * that is diagonal on the coset never has it */
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const double k = ss[j] + fma(-t, s, 1.0);
					re[g + j] *= k;
					im[g + j] *= k;
				}
			}
		}
	} else {
		constexpr int H = p2_hibit(U);
		constexpr int NP = 1 << (M - 1);
		constexpr int G = NP < P2_LIFT_GROUP ? NP : P2_LIFT_GROUP;
#pragma unroll
		for (int g = 0; g < NP; g += G) {
			double st[G], ss[G];
#pragma unroll
			for (int j = 0; j < G; ++j) {
				const uint32_t b = p2_bitmask(sm, p2_ins0(g + j, H));
				st[j] = p2_sgn(t, b);
				ss[j] = p2_sgn(s, b);
			}
			if constexpr (ODD) {
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g + j, H), w = u ^ U;
					re[u] = fma(-st[j], im[w], re[u]);
					im[u] = fma(st[j], re[w], im[u]);
				}
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g + j, H), w = u ^ U;
					re[w] = fma(-ss[j], im[u], re[w]);
					im[w] = fma(ss[j], re[u], im[w]);
				}
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g + j, H), w = u ^ U;
					re[u] = fma(-st[j], im[w], re[u]);
					im[u] = fma(st[j], re[w], im[u]);
				}
			} else {
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g + j, H), w = u ^ U;
					re[u] = fma(st[j], re[w], re[u]);
					im[u] = fma(st[j], im[w], im[u]);
				}
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g + j, H), w = u ^ U;
					re[w] = fma(-ss[j], re[u], re[w]);
					im[w] = fma(-ss[j], im[u], im[w]);
				}
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g + j, H), w = u ^ U;
					re[u] = fma(st[j], re[w], re[u]);
					im[u] = fma(st[j], im[w], im[u]);
				}
			}
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
		/* pairs P2_LIFT32_GROUP at a time, shear by shear (as in
		 * p2_rot_lift: independent pairs, the same bits) */
		constexpr int H = p2_hibit(U);
		constexpr int NP = 1 << (M - 1);
		constexpr int G = NP < P2_LIFT32_GROUP ? NP : P2_LIFT32_GROUP;
#pragma unroll
		for (int g0 = 0; g0 < NP; g0 += G) {
			float st[G], ss[G];
#pragma unroll
			for (int j = 0; j < G; ++j) {
				const uint32_t b = p2_bitmask(sm, p2_ins0(g0 + j, H));
				st[j] = p2_fsgn(t, b);
				ss[j] = p2_fsgn(s, b);
			}
			if constexpr (ODD) {
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g0 + j, H), w = u ^ U;
					re[u] = fmaf(-st[j], im[w], re[u]);
					im[u] = fmaf(st[j], re[w], im[u]);
				}
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g0 + j, H), w = u ^ U;
					re[w] = fmaf(-ss[j], im[u], re[w]);
					im[w] = fmaf(ss[j], re[u], im[w]);
				}
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g0 + j, H), w = u ^ U;
					re[u] = fmaf(-st[j], im[w], re[u]);
					im[u] = fmaf(st[j], re[w], im[u]);
				}
			} else {
				/* the same three shears as six fmaf, two lanes
				 * per packed FMA (round-to-nearest per lane: the
				 * same bits) */
				float2 yu[G], yw[G];
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g0 + j, H), w = u ^ U;
					yu[j] = make_float2(re[u], im[u]);
					yw[j] = make_float2(re[w], im[w]);
				}
#pragma unroll
				for (int j = 0; j < G; ++j)
					yu[j] = __ffma2_rn(make_float2(st[j], st[j]),
						yw[j], yu[j]);
#pragma unroll
				for (int j = 0; j < G; ++j)
					yw[j] = __ffma2_rn(make_float2(-ss[j], -ss[j]),
						yu[j], yw[j]);
#pragma unroll
				for (int j = 0; j < G; ++j)
					yu[j] = __ffma2_rn(make_float2(st[j], st[j]),
						yw[j], yu[j]);
#pragma unroll
				for (int j = 0; j < G; ++j) {
					const int u = p2_ins0(g0 + j, H), w = u ^ U;
					re[u] = yu[j].x;
					im[u] = yu[j].y;
					re[w] = yw[j].x;
					im[w] = yw[j].y;
				}
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

/* ---- persistent batch kernel -------------------------------------------- */

/*
 * Many registers' recorded programs (p2_internal.h) in one launch.  Every
 * op of a program is cut into tiles (a pass: 1024 amplitudes, 32 lanes
 * times 2^(5 - span) cosets; a zero: 16384 amplitudes; a write or gather:
 * one tile); op k+1 of a program starts only when every tile of op k is
 * done, programs are independent.  Each program has a ticket, (op << 32) |
 * next tile, on a line of its own.  Every warp schedules itself, with no
 * block barrier anywhere: its 32 lanes read 32 programs' tickets at once
 * (one memory round trip), the first program with tiles left, in order
 * from the warp's home program, is claimed with one atomicAdd of a run of
 * tiles, the warp runs them, and the warp that completes the last tile of
 * an op publishes the next op by resetting the ticket.  Runs are guided:
 * what is left of the op times the programs seen running, over (warps x
 * per_warp), 1 to P2_BATCH_RUN tiles, so an op is claimed in long runs
 * while every warp that can reach it still gets some, and its last tiles
 * in single ones.  Home programs spread the warps over
 * the programs in proportion to their work, so a long program is not
 * starved by many short ones and its chain of ops does not run alone at
 * the end.  A warp that finds nothing to claim sleeps between looks, 32 ns
 * at first, doubling to about a microsecond, until it claims again.
 * Waiting is bounded: a warp that finds nothing to claim while no ticket
 * moves for idle_limit consecutive rounds (at most about a microsecond
 * each; a ticket moves whenever any tile is claimed or any op is
 * published) raises status and returns, so a scheduling fault ends the
 * launch instead of hanging it, while long single-program runs, where most
 * warps wait on one op at a time, keep going.
 *
 * Ordering: a tile's stores are made visible (each lane fences, then the
 * warp synchronises) before its completion count; the finisher fences
 * before publishing the next op; a claimer fences after its claim, and
 * the other lanes read the claim only through the broadcast.  State loads
 * and stores go through L2 only (ld/st .cg), since L1 is not coherent
 * across SMs.
 */
/* A pass tile is 32 amplitudes a lane: 32 lanes times 2^(5 - span) cosets
 * (a warp's 1024 amplitudes, whatever the span); a warp claims runs of 1
 * to P2_BATCH_RUN tiles. */
#define P2_BATCH_RUN 16
#define P2_BATCH_ZERO_TILE (P2_TPB * 128)
#define P2_BATCH_WARPS (P2_TPB / 32)

struct p2_binst {
	void *state; /* float2 (FP32) or double2 (FP64) amplitudes */
	uint64_t namp;
	uint32_t op_off, nops;
};

/* Work tiles of an op on a register of namp amplitudes; for a pass of
 * span `span` also the cosets per lane of a tile (*b). */
__host__ __device__ __forceinline__ uint32_t p2_op_tiles(uint32_t kind,
	uint64_t namp, uint32_t span, uint32_t *b)
{
	if (kind == P2_OP_PASS) {
		const uint64_t nrep = namp >> span;
		*b = 1u << (span < 5 ? 5 - span : 0);
		const uint64_t per = (uint64_t)*b * 32;
		return (uint32_t)((nrep + per - 1) / per);
	}
	if (kind == P2_OP_ZERO)
		return (uint32_t)((namp + P2_BATCH_ZERO_TILE - 1) /
			P2_BATCH_ZERO_TILE);
	return 1;
}

/* A program's scheduling state, one 128-byte line each: every warp polls
 * the tickets and counts completions with atomics, so two programs never
 * share a line (nor an L2 slice's queue for it). */
struct p2_bctl {
	unsigned long long ticket;
	unsigned int done;
	unsigned int pad;
	unsigned long long end_ns; /* global timer when the program finished */
	unsigned long long line[13];
};

#endif /* P2_KERNELS_CUH */
