/*
 * lift_bulk.cu -- the FP32 lifted pass with FP64 arithmetic
 * (PHASE2_FORM_LIFTED) with its cosets staged in shared memory by bulk
 * asynchronous copies (cp.async.bulk, the TMA engine), so that the loads
 * of the next coset are in flight while the current one is rotated.
 *
 * Why: the FP64-arithmetic pass holds 32 complex doubles per thread (about
 * 160 registers, 12 resident warps per SM).  Loading straight into those
 * registers leaves each warp idle for a full memory latency per coset, and
 * twelve warps cannot cover it.  Here a warp's next coset is requested
 * before the current one is computed, into a second shared-memory stage,
 * and the copy engine does the loading without registers or load
 * instructions of its own: the memory pipeline depth no longer depends on
 * the register budget.
 *
 * Work unit: a warp-coset, 32 consecutive representatives t0 .. t0+31
 * (t0 a multiple of 32) with the 2^M slots of each.  When every pivot of
 * the pass is at bit 5 or above, the representatives are x0 | lane, and
 * slot u of the 32 lanes covers exactly one aligned block of 32
 * amplitudes, (x0 ^ off(u)) & ~31, lane l reading element l ^ (off(u) &
 * 31) of it.  So a warp-coset is 2^M copies of 256 bytes: lane u issues
 * the copy of slot u, lane 0 arms the stage's mbarrier with the byte
 * count.  Passes with a pivot below bit 5 (a span holding a string that
 * flips only qubits 0-4) or registers too small for whole warp-cosets run
 * on the direct kernel instead (engine.cu).
 *
 * Arithmetic: exactly k_pass_lift's (p2_rot_lift: widen to FP64 on load,
 * three FP64 shears per pair and rotation, one rounding to FP32 at the
 * store), so both kernels give the same bits.
 *
 * Every mbarrier wait is bounded (about two seconds of SM clock); a warp
 * that gives up sets *status, waits (bounded) for its other copy in
 * flight and returns.  The host reads *status at its next
 * synchronisation point (engine.cu, p2_status_check).
 */
#include <cuda_runtime.h>

#include <stdint.h>

#define LOG_SUBSYS "engine"
#include "log.h"

#include "p2_kernels.cuh"

#define P2_LB_WARPS 4
#define P2_LB_TPB (32 * P2_LB_WARPS)
/* SM clock cycles a warp waits for a stage before giving up */
#define P2_LB_WAIT_CYCLES (INT64_C(1) << 32)

/* Resident blocks per SM the register allocation is built for: 2^M FP64
 * complex values take 4 * 2^M registers per thread. */
__host__ __device__ constexpr int p2_lb_blocks(int m)
{
	return m >= 5 ? 3 : (m == 4 ? 5 : 8);
}

/* Dynamic shared memory of a block: two stages of 2^M blocks of 256 bytes
 * per warp, plus slack to align the stages to 256 bytes. */
__host__ __device__ constexpr unsigned p2_lb_smem(int m)
{
	return (unsigned)P2_LB_WARPS * 2u * (256u << m) + 256u;
}

__device__ __forceinline__ uint32_t p2_saddr(const void *p)
{
	return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void p2_mbar_init(uint32_t bar, uint32_t count)
{
	asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar),
		"r"(count)
		: "memory");
}

/* Arrive once and expect `bytes` of transactions on the current phase. */
__device__ __forceinline__ void p2_mbar_expect(uint32_t bar, uint32_t bytes)
{
	asm volatile(
		"mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
			bar),
		"r"(bytes)
		: "memory");
}

__device__ __forceinline__ bool p2_mbar_try(uint32_t bar, uint32_t parity)
{
	uint32_t ok;
	asm volatile("{\n\t.reg .pred p;\n\t"
		     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
		     "selp.u32 %0, 1, 0, p;\n\t}"
		: "=r"(ok)
		: "r"(bar), "r"(parity)
		: "memory");
	return ok != 0;
}

/* Wait for the phase of the given parity to complete; false after
 * P2_LB_WAIT_CYCLES. */
__device__ __forceinline__ bool p2_mbar_wait(uint32_t bar, uint32_t parity)
{
	if (p2_mbar_try(bar, parity))
		return true;
	const long long t0 = clock64();
	while (!p2_mbar_try(bar, parity))
		if (clock64() - t0 > P2_LB_WAIT_CYCLES)
			return false;
	return true;
}

/* Bulk copy of `bytes` from global memory into this CTA's shared memory,
 * completing as transactions on the mbarrier. */
__device__ __forceinline__ void p2_bulk_load(uint32_t dst, const void *src,
	uint32_t bytes, uint32_t bar)
{
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::"
		     "complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
		"l"(src), "r"(bytes), "r"(bar)
		: "memory");
}

/* Store the coset back (negated when NEG), narrowing to FP32. */
template <int M, bool NEG>
__device__ __forceinline__ void p2_lb_store(float2 *__restrict__ st,
	uint32_t x, const uint32_t (&pb)[M], const double (&re)[1 << M],
	const double (&im)[1 << M])
{
	const uint32_t xs = p2_opaque(x);
#pragma unroll
	for (int u = 0; u < (1 << M); ++u) {
		uint32_t off = 0;
#pragma unroll
		for (int k = 0; k < M; ++k)
			if (u >> k & 1)
				off ^= pb[k];
		st[xs ^ off] = NEG ? make_float2(__double2float_rn(-re[u]),
					     __double2float_rn(-im[u]))
				   : make_float2(__double2float_rn(re[u]),
					     __double2float_rn(im[u]));
	}
}

template <int M>
__global__ void __launch_bounds__(P2_LB_TPB, p2_lb_blocks(M))
	k_pass_lift_bulk(float2 *__restrict__ st, uint32_t nwc,
		struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs,
		unsigned int *__restrict__ status)
{
	constexpr int S = 1 << M;
	constexpr uint32_t STAGE = 256u * S; /* bytes per stage */
	extern __shared__ __align__(16) unsigned char p2_lb_dyn[];
	__shared__ struct p2_lift_rec srec[P2_MAX_ROTS_PER_PASS];
	__shared__ __align__(8) uint64_t sbar[P2_LB_WARPS][2];

	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
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
	const uint32_t bar0 = p2_saddr(&sbar[wid][0]);
	const uint32_t bar1 = p2_saddr(&sbar[wid][1]);
	if (lane == 0) {
		p2_mbar_init(bar0, 1);
		p2_mbar_init(bar1, 1);
	}
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	__syncthreads();

	/* this warp's two stages, 256-byte aligned */
	const uint32_t dyn = p2_saddr(p2_lb_dyn);
	const uint32_t pad = ((dyn + 255u) & ~255u) - dyn;
	const uint32_t sbase = dyn + pad + wid * 2u * STAGE;
	const float2 *const stage =
		(const float2 *)(p2_lb_dyn + pad + wid * 2u * STAGE);

	uint32_t pb[M], ob[M];
#pragma unroll
	for (int k = 0; k < M; ++k) {
		pb[k] = (uint32_t)p.basis[k];
		ob[k] = pb[k] & 31u;
	}
	/* the block this lane copies for each warp-coset: slot `lane` */
	uint32_t boff = 0;
#pragma unroll
	for (int k = 0; k < M; ++k)
		if (lane >> k & 1)
			boff ^= pb[k];
	boff &= ~31u;
	const uint32_t nrot = p.nrot;
	const bool neg = p.scale < 0;
	const uint32_t nw = gridDim.x * P2_LB_WARPS;

	uint32_t c = blockIdx.x * P2_LB_WARPS + wid;
	/* request warp-coset cc into stage sidx */
	auto issue = [&](uint32_t cc, uint32_t sidx) {
		const uint32_t bar = sidx ? bar1 : bar0;
		__syncwarp();
		if (lane == 0)
			p2_mbar_expect(bar, STAGE);
		__syncwarp();
		if (lane < (uint32_t)S) {
			const uint32_t x0 = p2_rep_t<M, uint32_t>(cc << 5, p);
			/* earlier generic reads of this stage come first */
			asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
			p2_bulk_load(sbase + sidx * STAGE + lane * 256u,
				st + (x0 ^ boff), 256u, bar);
		}
	};
	if (c < nwc)
		issue(c, 0);
	for (uint32_t k = 0; c < nwc; c += nw, ++k) {
		const uint32_t sidx = k & 1u;
		const bool more = c + nw < nwc;
		if (more)
			issue(c + nw, sidx ^ 1u);
		if (!p2_mbar_wait(sidx ? bar1 : bar0, (k >> 1) & 1u)) {
			if (lane == 0)
				atomicOr(status, 1u);
			/* the copy of the next stage may still be in flight */
			if (more)
				(void)p2_mbar_wait(sidx ? bar0 : bar1,
					((k + 1) >> 1) & 1u);
			return;
		}
		const float2 *const sv = stage + sidx * 32u * S;
		double re[S], im[S];
#pragma unroll
		for (int u = 0; u < S; ++u) {
			uint32_t ou = 0;
#pragma unroll
			for (int b = 0; b < M; ++b)
				if (u >> b & 1)
					ou ^= ob[b];
			const float2 v = sv[u * 32 + (lane ^ ou)];
			re[u] = (double)v.x;
			im[u] = (double)v.y;
		}
		const uint32_t x = p2_rep_t<M, uint32_t>(c << 5, p) | lane;
		for (uint32_t r = 0; r < nrot; ++r) {
			const struct p2_lift_rec q = srec[r];
			const uint32_t sm =
				q.sm ^ (0u - p2_parity(x & (uint32_t)q.z));
			p2_apply_lift<M>(q.key, re, im, q.t, q.s, sm);
		}
		if (neg)
			p2_lb_store<M, true>(st, x, pb, re, im);
		else
			p2_lb_store<M, false>(st, x, pb, re, im);
	}
}

/*
 * The same pass with the next warp-coset staged by cp.async instead of the
 * copy engine: the 2^M blocks of 256 bytes are moved as 16-byte pieces,
 * lane l taking piece l % 16 of slot blocks 2j + l / 16, j < 2^M / 2, so
 * one warp instruction moves two blocks (16 per warp-coset at M = 5,
 * against 32 loads per thread in the direct kernel).  Each lane waits for
 * its own pieces (cp.async.wait_group) and the warp then synchronises, as
 * lanes read pieces other lanes copied.  No waits of the kernel's own: the
 * copies complete by themselves.
 */
template <int M, int MINB>
__global__ void __launch_bounds__(P2_LB_TPB, MINB)
	k_pass_lift_pf(float2 *__restrict__ st, uint32_t nwc,
		struct phase2_pass p,
		const struct phase2_rot_rec *__restrict__ recs)
{
	constexpr int S = 1 << M;
	constexpr uint32_t STAGE = 256u * S; /* bytes per stage */
	extern __shared__ __align__(16) unsigned char p2_lb_dyn[];
	__shared__ struct p2_lift_rec srec[P2_MAX_ROTS_PER_PASS];

	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
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

	const uint32_t dyn = p2_saddr(p2_lb_dyn);
	const uint32_t pad = ((dyn + 255u) & ~255u) - dyn;
	/* this lane's piece of the first two slot blocks, stage 0 */
	const uint32_t sdst = dyn + pad + wid * 2u * STAGE + lane * 16u;
	const float2 *const stage =
		(const float2 *)(p2_lb_dyn + pad + wid * 2u * STAGE);

	uint32_t pb[M], ob[M];
#pragma unroll
	for (int k = 0; k < M; ++k) {
		pb[k] = (uint32_t)p.basis[k];
		ob[k] = pb[k] & 31u;
	}
	/* slot bit 0 of this lane's blocks */
	const uint32_t hb = (lane >> 4) ? pb[0] : 0u;
	const char *const src0 = (const char *)st + (lane & 15u) * 16u;
	const uint32_t nrot = p.nrot;
	const bool neg = p.scale < 0;
	const uint32_t nw = gridDim.x * P2_LB_WARPS;

	/* request warp-coset cc into stage sidx (one commit group) */
	auto issue = [&](uint32_t cc, uint32_t sidx) {
		const uint32_t xb = p2_rep_t<M, uint32_t>(cc << 5, p) ^ hb;
#pragma unroll
		for (int j = 0; j < S / 2; ++j) {
			uint32_t o = 0;
#pragma unroll
			for (int k = 1; k < M; ++k)
				if (j >> (k - 1) & 1)
					o ^= pb[k];
			p2_cp16(sdst + sidx * STAGE + (uint32_t)j * 512u,
				src0 + (size_t)((xb ^ o) & ~31u) * 8u);
		}
		p2_cp_commit();
	};

	uint32_t c = blockIdx.x * P2_LB_WARPS + wid;
	if (c < nwc)
		issue(c, 0);
	else
		p2_cp_commit();
	for (uint32_t k = 0; c < nwc; c += nw, ++k) {
		const uint32_t sidx = k & 1u;
		/* every lane has read the stage the next request overwrites */
		__syncwarp();
		if (c + nw < nwc)
			issue(c + nw, sidx ^ 1u);
		else
			p2_cp_commit();
		p2_cp_wait<1>();
		__syncwarp();
		const float2 *const sv = stage + sidx * 32u * S;
		double re[S], im[S];
#pragma unroll
		for (int u = 0; u < S; ++u) {
			uint32_t ou = 0;
#pragma unroll
			for (int b = 0; b < M; ++b)
				if (u >> b & 1)
					ou ^= ob[b];
			const float2 v = sv[u * 32 + (lane ^ ou)];
			re[u] = (double)v.x;
			im[u] = (double)v.y;
		}
		const uint32_t x = p2_rep_t<M, uint32_t>(c << 5, p) | lane;
		for (uint32_t r = 0; r < nrot; ++r) {
			const struct p2_lift_rec q = srec[r];
			const uint32_t sm =
				q.sm ^ (0u - p2_parity(x & (uint32_t)q.z));
			p2_apply_lift<M>(q.key, re, im, q.t, q.s, sm);
		}
		if (neg)
			p2_lb_store<M, true>(st, x, pb, re, im);
		else
			p2_lb_store<M, false>(st, x, pb, re, im);
	}
	p2_cp_wait<0>();
}

struct p2_lb_cfg {
	int ready;
	int per_sm;
};

/* Grid of a staged kernel: resident blocks per SM (occupancy, capped),
 * at most one block per four warp-cosets. */
static unsigned lb_grid(const struct p2_dev *d, int per_sm_occ,
	unsigned per_sm_cap, uint32_t nwc)
{
	unsigned per_sm = (unsigned)per_sm_occ;
	if (per_sm_cap && per_sm_cap < per_sm)
		per_sm = per_sm_cap;
	uint64_t grid = (uint64_t)d->sm_count * per_sm;
	const uint64_t need = (nwc + P2_LB_WARPS - 1) / P2_LB_WARPS;
	if (grid > need)
		grid = need;
	return (unsigned)grid;
}

template <int M, int MINB>
static int pf_launch_t(struct p2_dev *d, const struct phase2_pass *p,
	const struct phase2_rot_rec *recs, unsigned per_sm_cap)
{
	static struct p2_lb_cfg cfg;
	const unsigned smem = p2_lb_smem(M);
	if (!cfg.ready) {
		CUDA_OK(cudaFuncSetAttribute(k_pass_lift_pf<M, MINB>,
				cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)smem),
			"staged pass shared memory");
		int n = 0;
		CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n,
				k_pass_lift_pf<M, MINB>, P2_LB_TPB, smem),
			"staged pass occupancy");
		cfg.per_sm = n > 0 ? n : 1;
		cfg.ready = 1;
	}
	const uint32_t nwc = (uint32_t)((d->namp >> M) >> 5);
	k_pass_lift_pf<M, MINB><<<lb_grid(d, cfg.per_sm, per_sm_cap, nwc),
		P2_LB_TPB, smem, d->stream>>>((float2 *)d->state, nwc, *p,
		recs);
	return 1;
}

template <int M>
static int lb_launch_t(struct p2_dev *d, const struct phase2_pass *p,
	const struct phase2_rot_rec *recs, unsigned per_sm_cap)
{
	static struct p2_lb_cfg cfg;
	const unsigned smem = p2_lb_smem(M);
	if (!cfg.ready) {
		CUDA_OK(cudaFuncSetAttribute(k_pass_lift_bulk<M>,
				cudaFuncAttributeMaxDynamicSharedMemorySize,
				(int)smem),
			"staged pass shared memory");
		int n = 0;
		CUDA_OK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n,
				k_pass_lift_bulk<M>, P2_LB_TPB, smem),
			"staged pass occupancy");
		cfg.per_sm = n > 0 ? n : 1;
		cfg.ready = 1;
	}
	const uint32_t nwc = (uint32_t)((d->namp >> M) >> 5);
	k_pass_lift_bulk<M><<<lb_grid(d, cfg.per_sm, per_sm_cap, nwc),
		P2_LB_TPB, smem, d->stream>>>((float2 *)d->state, nwc, *p,
		recs, d->d_status);
	d->status_pending = 1;
	return 1;
}

extern "C" int p2_lift_staged_launch(struct p2_dev *d,
	const struct phase2_pass *p, const struct phase2_rot_rec *recs,
	int variant, unsigned per_sm_cap)
{
	/* whole warp-cosets of 32-bit indices, every pivot at bit 5 or above */
	if (d->prec != PHASE2_PREC_FP32 ||
		(p->form != PHASE2_FORM_LIFTED &&
			p->form != PHASE2_FORM_LIFTED_MIXED) ||
		d->nqb > 31 || p->span < 3 || p->span > 5 ||
		d->nqb < p->span + 5 || p->piv[0] < 5)
		return 0;
	if (variant == 1) {
		if (!d->d_status)
			return 0;
		switch (p->span) {
		case 3:
			return lb_launch_t<3>(d, p, recs, per_sm_cap);
		case 4:
			return lb_launch_t<4>(d, p, recs, per_sm_cap);
		default:
			return lb_launch_t<5>(d, p, recs, per_sm_cap);
		}
	}
	/* variant 3: at span 5 the build for two blocks per SM, with the
	 * whole register file of those blocks (up to 255 registers a
	 * thread) */
	switch (p->span) {
	case 3:
		return pf_launch_t<3, p2_lb_blocks(3)>(d, p, recs, per_sm_cap);
	case 4:
		return pf_launch_t<4, p2_lb_blocks(4)>(d, p, recs, per_sm_cap);
	default:
		return variant == 3
			? pf_launch_t<5, 2>(d, p, recs, 0)
			: pf_launch_t<5, p2_lb_blocks(5)>(d, p, recs,
				  per_sm_cap);
	}
}
