/*
 * batch.cu -- the persistent kernel (k_batch): recorded programs of many
 * registers (zero, determinant writes, passes, gathers) scheduled as
 * (register, op, tile) work over all SMs in one launch, FP32 or FP64 state;
 * the batched drivers' executor (p2d_batch_run).  Device sampling
 * (sampling.cu) runs its programs through the same kernel.
 */
#include <cuda_runtime.h>

#include <float.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#define LOG_SUBSYS "engine"
#include "log.h"

#include "p2_kernels.cuh"

/* The cosets of a warp's run of pass tiles: lane k takes representatives
 * r0 + j * 32 + k, j < cpt (coalesced per j). */
template <int M>
__device__ __forceinline__ void p2_batch_pass_tile(float2 *st,
	const struct phase2_pass &p, uint64_t r0, uint64_t nrep, uint32_t cpt,
	const struct p2_lift32_rec *srec, uint32_t lane)
{
	uint32_t pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = (uint32_t)p.basis[k];
	const uint32_t negm = p.scale < 0 ? 0x80000000u : 0u;
	const uint64_t t0 = r0 + lane;
	for (uint32_t j = 0; j < cpt; ++j) {
		const uint64_t t = t0 + (uint64_t)j * 32;
		if (t < nrep)
			p2_lift32_coset<M, uint32_t, true>(st,
				p2_rep_t<M, uint32_t>((uint32_t)t, p), pb, srec,
				p.nrot, negm);
	}
}

/* The same for an FP32 register in the FP64-arithmetic form: each coset
 * widened to FP64, the run applied by p2_rot_lift (the arithmetic of
 * k_pass_lift and k_pass_lift_pf, the same bits), one rounding to FP32 at
 * the store (negated when the pass scale is -1). */
template <int M>
__device__ __forceinline__ void p2_batch_pass_tile_x(float2 *st,
	const struct phase2_pass &p, uint64_t r0, uint64_t nrep, uint32_t cpt,
	const struct p2_lift_rec *srec, uint32_t lane)
{
	uint32_t pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = (uint32_t)p.basis[k];
	const bool neg = p.scale < 0;
	const uint64_t t0 = r0 + lane;
	for (uint32_t j = 0; j < cpt; ++j) {
		const uint64_t t = t0 + (uint64_t)j * 32;
		if (t >= nrep)
			continue;
		const uint32_t x = p2_rep_t<M, uint32_t>((uint32_t)t, p);
		double re[1 << M], im[1 << M];
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			uint32_t off = 0;
#pragma unroll
			for (int k = 0; k < M; ++k)
				if (u >> k & 1)
					off ^= pb[k];
			const float2 v = __ldcg(st + (x ^ off));
			re[u] = (double)v.x;
			im[u] = (double)v.y;
		}
		for (uint32_t r = 0; r < p.nrot; ++r) {
			const struct p2_lift_rec q = srec[r];
			const uint32_t sm =
				q.sm ^ (0u - p2_parity(x & (uint32_t)q.z));
			p2_apply_lift<M>(q.key, re, im, q.t, q.s, sm);
		}
		const uint32_t xs = p2_opaque(x);
#pragma unroll
		for (int u = 0; u < (1 << M); ++u) {
			uint32_t off = 0;
#pragma unroll
			for (int k = 0; k < M; ++k)
				if (u >> k & 1)
					off ^= pb[k];
			const double a = neg ? -re[u] : re[u];
			const double b = neg ? -im[u] : im[u];
			__stcg(st + (xs ^ off), make_float2(__double2float_rn(a),
							 __double2float_rn(b)));
		}
	}
}

/* The same for an FP64 register: the exact per-coset arithmetic of
 * k_pass (p2_apply_run), loads and stores at L2 only. */
template <int M>
__device__ __forceinline__ void p2_batch_pass_tile64(double2 *st,
	const struct phase2_pass &p, uint64_t r0, uint64_t nrep, uint32_t cpt,
	const struct phase2_rot_rec *srec, uint32_t lane)
{
	uint64_t pb[M > 0 ? M : 1];
#pragma unroll
	for (int k = 0; k < M; ++k)
		pb[k] = p.basis[k];
	const uint64_t t0 = r0 + lane;
	for (uint32_t j = 0; j < cpt; ++j) {
		const uint64_t t = t0 + (uint64_t)j * 32;
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
template <typename ST, bool X> struct p2_brec;
template <> struct p2_brec<float2, false> {
	typedef struct p2_lift32_rec type;
	static __device__ __forceinline__ type of(const phase2_rot_rec &r)
	{
		return p2_lift32_of(r);
	}
};
template <> struct p2_brec<float2, true> {
	typedef struct p2_lift_rec type;
	static __device__ __forceinline__ type of(const phase2_rot_rec &r)
	{
		struct p2_lift_rec o;
		o.t = r.c;
		o.s = r.s;
		o.z = r.z;
		o.sm = r.smask;
		o.key = ((uint32_t)r.U << 1) | r.odd;
		return o;
	}
};
template <> struct p2_brec<double2, false> {
	typedef struct phase2_rot_rec type;
	static __device__ __forceinline__ type of(const phase2_rot_rec &r)
	{
		return r;
	}
};

/* Span dispatch of a pass tile (FP32 state in either form, or FP64). */
template <typename ST, bool X, typename RT>
__device__ __forceinline__ void p2_batch_pass(ST *st,
	const struct phase2_pass &p, uint64_t r0, uint64_t nrep, uint32_t cpt,
	const RT *srec, uint32_t lane)
{
	if constexpr (X) {
		switch (p.span) {
		case 0:
			p2_batch_pass_tile_x<0>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 1:
			p2_batch_pass_tile_x<1>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 2:
			p2_batch_pass_tile_x<2>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 3:
			p2_batch_pass_tile_x<3>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 4:
			p2_batch_pass_tile_x<4>(st, p, r0, nrep, cpt, srec, lane);
			break;
		default:
			p2_batch_pass_tile_x<5>(st, p, r0, nrep, cpt, srec, lane);
			break;
		}
	} else if constexpr (sizeof(ST) == 16) {
		switch (p.span) {
		case 0:
			p2_batch_pass_tile64<0>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 1:
			p2_batch_pass_tile64<1>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 2:
			p2_batch_pass_tile64<2>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 3:
			p2_batch_pass_tile64<3>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 4:
			p2_batch_pass_tile64<4>(st, p, r0, nrep, cpt, srec, lane);
			break;
		default:
			p2_batch_pass_tile64<5>(st, p, r0, nrep, cpt, srec, lane);
			break;
		}
	} else {
		switch (p.span) {
		case 0:
			p2_batch_pass_tile<0>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 1:
			p2_batch_pass_tile<1>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 2:
			p2_batch_pass_tile<2>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 3:
			p2_batch_pass_tile<3>(st, p, r0, nrep, cpt, srec, lane);
			break;
		case 4:
			p2_batch_pass_tile<4>(st, p, r0, nrep, cpt, srec, lane);
			break;
		default:
			p2_batch_pass_tile<5>(st, p, r0, nrep, cpt, srec, lane);
			break;
		}
	}
}

__device__ __forceinline__ unsigned long long p2_globaltimer()
{
	unsigned long long t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

/* Resident blocks per SM of a k_batch instance: FP32 arithmetic 5, FP32
 * state with FP64 arithmetic 3 (32 complex doubles a thread), FP64 2. */
__host__ __device__ constexpr int p2_batch_blocks(bool f64, bool x)
{
	return f64 ? 2 : (x ? 3 : 5);
}

/* Hash of a program's ticket for the idle check (any move changes it). */
__device__ __forceinline__ unsigned int p2_tk_hash(unsigned long long tk,
	uint32_t i)
{
	return ((unsigned int)tk ^ (unsigned int)(tk >> 32) * 0x9e3779b9u) *
		(2u * i + 1u);
}

template <typename ST, bool X>
__global__ void __launch_bounds__(P2_TPB,
	p2_batch_blocks(sizeof(ST) == 16, X))
	k_batch(const struct p2_binst *__restrict__ inst, uint32_t ninst,
		const struct p2_op *__restrict__ ops,
		const struct phase2_pass *__restrict__ passes,
		const struct phase2_rot_rec *__restrict__ recs,
		const uint64_t *__restrict__ widx,
		const double *__restrict__ wval,
		const uint64_t *__restrict__ gidx, double2 *__restrict__ gout,
		struct p2_bctl *ctl, unsigned int *status,
		const double *__restrict__ cum, unsigned int per_warp,
		unsigned int idle_limit)
{
	constexpr bool F64 = sizeof(ST) == 16;
	constexpr unsigned FULL = 0xffffffffu;
	typedef typename p2_brec<ST, X>::type RT;
	/* each warp keeps the records of the pass it last ran */
	__shared__ RT srec_all[P2_BATCH_WARPS][P2_MAX_ROTS_PER_PASS];
	const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
	RT *const srec = srec_all[wid];
	const uint32_t nwarps = gridDim.x * P2_BATCH_WARPS;
	const uint32_t gw = blockIdx.x * P2_BATCH_WARPS + wid;
	if (lane == 0) {
		/* start of the launch: the earliest warp's timer (status[2..3]
		 * holds its complement, so that zero-initialised memory works
		 * with atomicMax) */
		atomicMax((unsigned long long *)(status + 2),
			~p2_globaltimer());
	}
	/* home program: warps are spread over the programs in proportion to
	 * their work (cum: running totals), so a large program gets many
	 * warps that look at it first; without cum, round robin */
	uint32_t home = gw % ninst;
	if (cum) {
		const double at = ((double)gw + 0.5) / (double)nwarps *
			cum[ninst - 1];
		uint32_t lo = 0, hi = ninst - 1;
		while (lo < hi) {
			const uint32_t mid = (lo + hi) >> 1;
			if (cum[mid] > at)
				hi = mid;
			else
				lo = mid + 1;
		}
		home = lo;
	}
	uint32_t held = 0xffffffffu; /* pass whose records srec holds */
	unsigned int idle = 0;
	unsigned int nap = 32; /* ns slept by the next idle round */
	unsigned int seen = 0; /* ticket hash at the last idle round */
	for (;;) {
		/* look at 32 programs at a time (one lane each, from home on)
		 * and claim a run of tiles from the first that has some:
		 * what = 0 nothing claimable yet, 1 work, 2 exit */
		int what = 2;
		uint32_t ci = 0, cseq = 0, cfirst = 0, cend = 0;
		unsigned int sig = 0, live = 0;
		for (uint32_t base = 0; base < ninst && what != 1; base += 32) {
			const uint32_t k = base + lane;
			uint32_t i = 0, seq = 0, nt = 0, off = 0, nops = 0;
			unsigned long long tk = 0;
			bool avail = false;
			if (k < ninst) {
				i = home + k < ninst ? home + k : home + k - ninst;
				tk = *(volatile unsigned long long *)&ctl[i].ticket;
				sig += p2_tk_hash(tk, i);
				seq = (uint32_t)(tk >> 32);
				nops = inst[i].nops;
				off = inst[i].op_off;
				if (seq < nops) {
					what = 0;
					nt = ops[off + seq].ntiles;
					avail = (uint32_t)tk < nt;
				}
			}
			live += __popc(__ballot_sync(FULL,
				k < ninst && seq < nops));
			unsigned int m = __ballot_sync(FULL, avail);
			while (m) {
				const int src = __ffs(m) - 1;
				m &= m - 1;
				int ok = 0;
				if (lane == (uint32_t)src) {
					/* guided run: the warp's share of what is
					 * left of the op (the warps split over the
					 * programs seen running), cut into per_warp
					 * runs, 1 to P2_BATCH_RUN tiles */
					const uint64_t rem = nt - (uint32_t)tk;
					uint64_t n = rem * live /
						((uint64_t)nwarps * per_warp);
					n = n < 1 ? 1 : n > P2_BATCH_RUN ? P2_BATCH_RUN : n;
					const unsigned long long got =
						atomicAdd(&ctl[i].ticket,
							(unsigned long long)n);
					const uint32_t gs = (uint32_t)(got >> 32);
					const uint32_t first = (uint32_t)got;
					if (gs < nops) {
						const uint32_t gnt = gs == seq
							? nt : ops[off + gs].ntiles;
						if (first < gnt) {
							__threadfence();
							ok = 1;
							ci = i;
							cseq = gs;
							cfirst = first;
							cend = first + n < gnt
								? first + n : gnt;
						}
					}
				}
				const int who = __ballot_sync(FULL, ok);
				if (who) {
					const int w = __ffs(who) - 1;
					ci = __shfl_sync(FULL, ci, w);
					cseq = __shfl_sync(FULL, cseq, w);
					cfirst = __shfl_sync(FULL, cfirst, w);
					cend = __shfl_sync(FULL, cend, w);
					what = 1;
					break;
				}
			}
			if (what != 1)
				what = __any_sync(FULL, what == 0) ? 0 : 2;
		}
		if (what == 2)
			return;
		if (what == 0) {
			sig = __reduce_add_sync(FULL, sig);
			if (sig != seen) {
				seen = sig;
				idle = 0;
			}
			if (++idle > idle_limit) {
				if (lane == 0)
					atomicOr(status, 1u);
				return;
			}
			__nanosleep(nap);
			if (nap < 1024)
				nap <<= 1;
			continue;
		}
		idle = 0;
		nap = 32;
		const uint32_t i = ci, seq = cseq;
		ST *const st = (ST *)inst[i].state;
		const uint64_t namp = inst[i].namp;
		const struct p2_op op = ops[inst[i].op_off + seq];
		if (op.kind == P2_OP_PASS) {
			const struct phase2_pass p = passes[op.a];
			/* consecutive tiles of one pass (a Trotter step replays
			 * the same passes) keep their records */
			if (held != op.a) {
				__syncwarp();
				for (uint32_t r = lane; r < p.nrot; r += 32)
					srec[r] = p2_brec<ST, X>::of(
						recs[p.rot_off + r]);
				held = op.a;
				__syncwarp();
			}
			p2_batch_pass<ST, X, RT>(st, p,
				(uint64_t)cfirst * op.b * 32, namp >> p.span,
				(cend - cfirst) * op.b, srec, lane);
		} else if (op.kind == P2_OP_ZERO) {
			const uint64_t lo = (uint64_t)cfirst * P2_BATCH_ZERO_TILE;
			uint64_t hi = (uint64_t)cend * P2_BATCH_ZERO_TILE;
			hi = hi < namp ? hi : namp;
			ST zero;
			zero.x = 0;
			zero.y = 0;
			for (uint64_t k = lo + lane; k < hi; k += 32)
				__stcg(st + k, zero);
		} else if (op.kind == P2_OP_WRITE) {
			/* in order: later writes win */
			if (lane == 0)
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
			for (uint32_t d = lane; d < op.b; d += 32) {
				const ST v = __ldcg(st + gidx[op.a + d]);
				gout[op.a + d] = make_double2(v.x, v.y);
			}
		}
		__threadfence();
		__syncwarp();
		if (lane == 0) {
			const unsigned int cnt = cend - cfirst;
			const unsigned int d = atomicAdd(&ctl[i].done, cnt) + cnt;
			if (d == op.ntiles) {
				atomicExch(&ctl[i].done, 0u);
				if (seq + 1 == inst[i].nops)
					ctl[i].end_ns = p2_globaltimer();
				__threadfence();
				atomicExch(&ctl[i].ticket,
					(unsigned long long)(seq + 1) << 32);
			}
		}
	}
}

/* ---- bounded-wait check -------------------------------------------------- */

/*
 * The persistent kernel on a program that can never make progress: one
 * instance whose only op has one tile, with the ticket preset past that
 * tile (taken) and no completion ever counted.  Every warp then finds
 * nothing to claim while no ticket moves, so each gives up after
 * idle_limit rounds, raises status and returns; no state memory is
 * touched.  Returns 1 when the launch ended that way, 0 when it ended
 * without raising status, -1 on a CUDA error.
 */
extern "C" int phase2_batch_wait_check(unsigned int idle_limit)
{
	struct p2_binst hinst;
	struct p2_op hop;
	struct p2_bctl hctl;
	memset(&hinst, 0, sizeof hinst);
	memset(&hop, 0, sizeof hop);
	memset(&hctl, 0, sizeof hctl);
	hinst.namp = 256;
	hinst.op_off = 0;
	hinst.nops = 1;
	hop.kind = P2_OP_ZERO;
	hop.ntiles = 1;
	hctl.ticket = 1; /* op 0, tile 1: the op's only tile is taken */
	unsigned char *buf = NULL;
	const size_t o_state = 0, o_inst = 256, o_op = 512, o_ctl = 768,
		     o_status = 1024, total = 1280;
	cudaError_t e = cudaMalloc((void **)&buf, total);
	if (e == cudaSuccess) {
		hinst.state = buf + o_state;
		e = cudaMemset(buf, 0, total);
	}
	if (e == cudaSuccess)
		e = cudaMemcpy(buf + o_inst, &hinst, sizeof hinst,
			cudaMemcpyHostToDevice);
	if (e == cudaSuccess)
		e = cudaMemcpy(buf + o_op, &hop, sizeof hop,
			cudaMemcpyHostToDevice);
	if (e == cudaSuccess)
		e = cudaMemcpy(buf + o_ctl, &hctl, sizeof hctl,
			cudaMemcpyHostToDevice);
	unsigned int status = 0;
	if (e == cudaSuccess) {
		k_batch<float2, false><<<2, P2_TPB>>>(
			(const struct p2_binst *)(buf + o_inst), 1,
			(const struct p2_op *)(buf + o_op), NULL, NULL, NULL,
			NULL, NULL, NULL, (struct p2_bctl *)(buf + o_ctl),
			(unsigned int *)(buf + o_status), NULL, 2, idle_limit);
		e = cudaGetLastError();
	}
	if (e == cudaSuccess)
		e = cudaDeviceSynchronize();
	if (e == cudaSuccess)
		e = cudaMemcpy(&status, buf + o_status, sizeof status,
			cudaMemcpyDeviceToHost);
	cudaFree(buf);
	if (e != cudaSuccess) {
		log_error("batch wait check: %s", cudaGetErrorString(e));
		return -1;
	}
	return status ? 1 : 0;
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

/* Finish time of every program of the last persistent launch, in ms after
 * the launch's first warp started (phase2_batch_finish_ms). */
static double *last_finish;
static size_t last_n;

static cudaError_t finish_times(const unsigned char *d_ctl,
	const unsigned char *d_status, size_t n)
{
	struct p2_bctl *c = (struct p2_bctl *)malloc(n * sizeof *c);
	double *f = (double *)realloc(last_finish, n * sizeof *f);
	if (!c || !f) {
		free(c);
		if (f)
			last_finish = f;
		return cudaErrorMemoryAllocation;
	}
	last_finish = f;
	unsigned long long start = 0;
	cudaError_t e = cudaMemcpy(c, d_ctl, n * sizeof *c,
		cudaMemcpyDeviceToHost);
	if (e == cudaSuccess)
		e = cudaMemcpy(&start, d_status + 8, sizeof start,
			cudaMemcpyDeviceToHost);
	start = ~start;
	for (size_t i = 0; i < n && e == cudaSuccess; i++)
		f[i] = c[i].end_ns >= start ? (double)(c[i].end_ns - start) / 1e6
					    : 0.0;
	last_n = e == cudaSuccess ? n : 0;
	free(c);
	return e;
}

extern "C" void p2_batch_finish_reset(void)
{
	last_n = 0;
}

extern "C" int p2_batch_finish_map(const size_t *who, size_t m, size_t n)
{
	if (last_n != m)
		return -1;
	double *f = (double *)malloc((n ? n : 1) * sizeof *f);
	if (!f)
		return -1;
	for (size_t i = 0; i < n; i++)
		f[i] = -1.0;
	for (size_t j = 0; j < m; j++)
		if (who[j] < n)
			f[who[j]] = last_finish[j];
	free(last_finish);
	last_finish = f;
	last_n = n;
	return 0;
}

extern "C" size_t phase2_batch_finish_ms(double *out, size_t n)
{
	const size_t k = n < last_n ? n : last_n;
	if (out && k)
		memcpy(out, last_finish, k * sizeof *out);
	return last_n;
}

/* Runs a warp's share of an op is cut into (phase2_set_batch_runs). */
static unsigned int g_batch_runs = 2;

extern "C" int phase2_set_batch_runs(unsigned int per_warp)
{
	if (per_warp < 1 || per_warp > 64)
		return -1;
	g_batch_runs = per_warp;
	return 0;
}

extern "C" unsigned int phase2_get_batch_runs(void)
{
	return g_batch_runs;
}

/* k_batch for FP32 or FP64 registers: its kernel function (occupancy
 * queries) and its launch.  Mixed-form programs run on the FP64-arithmetic
 * instance (every coset in FP64; their records are the FP32 form's). */
int p2_batch_kind(int prec, int form)
{
	if (prec == PHASE2_PREC_FP64)
		return P2_BK_F64;
	return form == PHASE2_FORM_LIFTED || form == PHASE2_FORM_LIFTED_MIXED
		? P2_BK_F32X : P2_BK_F32;
}

const void *p2_batch_kernel(int kind)
{
	return kind == P2_BK_F64 ? (const void *)k_batch<double2, false>
		: kind == P2_BK_F32X ? (const void *)k_batch<float2, true>
				      : (const void *)k_batch<float2, false>;
}

void p2_batch_launch(int kind, unsigned grid, cudaStream_t stream,
	const struct p2_binst *inst, uint32_t ninst, const struct p2_op *ops,
	const struct phase2_pass *passes, const struct phase2_rot_rec *recs,
	const uint64_t *widx, const double *wval, const uint64_t *gidx,
	double2 *gout, struct p2_bctl *ctl, unsigned int *status,
	const double *cum)
{
	if (kind == P2_BK_F64)
		k_batch<double2, false><<<grid, P2_TPB, 0, stream>>>(inst,
			ninst, ops, passes, recs, widx, wval, gidx, gout, ctl,
			status, cum, g_batch_runs, P2_BATCH_IDLE_LIMIT);
	else if (kind == P2_BK_F32X)
		k_batch<float2, true><<<grid, P2_TPB, 0, stream>>>(inst,
			ninst, ops, passes, recs, widx, wval, gidx, gout, ctl,
			status, cum, g_batch_runs, P2_BATCH_IDLE_LIMIT);
	else
		k_batch<float2, false><<<grid, P2_TPB, 0, stream>>>(inst,
			ninst, ops, passes, recs, widx, wval, gidx, gout, ctl,
			status, cum, g_batch_runs, P2_BATCH_IDLE_LIMIT);
}

/* Host seconds (PHASE2_BATCH_TIMING breakdown). */
static double p2_now(void)
{
	struct timespec ts;
	clock_gettime(CLOCK_MONOTONIC, &ts);
	return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
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
	const size_t o_cum = p2_align256(o_gidx + ng * sizeof(uint64_t));
	const size_t up = p2_align256(o_cum + n * sizeof(double));
	const size_t o_gout = up;
	const size_t o_ctl = p2_align256(o_gout + ng * sizeof(double2));
	const size_t o_status = p2_align256(o_ctl + n * sizeof(struct p2_bctl));
	const size_t total = o_status + 256;

	/* the kernel instance for the precision and the form the programs'
	 * passes were planned in (one process-wide FP32 form), and its
	 * resident blocks */
	struct p2_dev *d0 = devs[0];
	int form = d0->prec == PHASE2_PREC_FP64 ? PHASE2_FORM_EXACT
						: PHASE2_FORM_LIFTED_F32;
	for (size_t i = 0; i < n && d0->prec != PHASE2_PREC_FP64; i++)
		if (progs[i]->npass) {
			form = progs[i]->passes[0].form;
			break;
		}
	const int kind = p2_batch_kind(d0->prec, form);
	int per_sm = 0;
	cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
		p2_batch_kernel(kind), P2_TPB, 0);
	if (e != cudaSuccess) {
		log_error("batch: setup: %s", cudaGetErrorString(e));
		return -1;
	}
	unsigned grid =
		(unsigned)d0->sm_count * (unsigned)(per_sm > 0 ? per_sm : 1);

	const double tb0 = p2_now();
	unsigned char *h = (unsigned char *)malloc(up);
	if (!h)
		return -1;
	/* warps that can ever find work at once: the largest op of every
	 * program (more would only poll) */
	uint64_t busiest = 0;
	struct p2_binst *hi = (struct p2_binst *)(h + o_inst);
	struct p2_op *ho = (struct p2_op *)(h + o_ops);
	struct phase2_pass *hp = (struct phase2_pass *)(h + o_pass);
	struct phase2_rot_rec *hr = (struct phase2_rot_rec *)(h + o_rec);
	uint64_t *hwi = (uint64_t *)(h + o_widx);
	double *hwv = (double *)(h + o_wval);
	uint64_t *hgi = (uint64_t *)(h + o_gidx);
	/* running totals of the programs' work (amplitudes times rotations
	 * plus two per pass for its loads and stores): home programs */
	double *hcum = (double *)(h + o_cum);
	double work = 0;
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
		uint32_t most = 1;
		for (size_t k = 0; k < pg->nops; k++) {
			struct p2_op op = pg->ops[k];
			switch (op.kind) {
			case P2_OP_PASS:
				op.a += (uint32_t)bp;
				op.ntiles = p2_op_tiles(P2_OP_PASS, d->namp,
					hp[op.a].span, &op.b);
				work += (double)d->namp * (hp[op.a].nrot + 2.0);
				break;
			case P2_OP_ZERO:
				op.ntiles = p2_op_tiles(P2_OP_ZERO, d->namp, 0,
					&op.b);
				work += (double)d->namp;
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
			if (op.ntiles > most)
				most = op.ntiles;
		}
		busiest += most;
		work += 1.0; /* every program at least one unit */
		hcum[i] = work;
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

	const uint64_t want = (busiest + P2_BATCH_WARPS - 1) / P2_BATCH_WARPS;
	if (want < grid)
		grid = (unsigned)want;
	unsigned char *dbuf = NULL;
	const double tb1 = p2_now();
	for (size_t i = 0; i < n && e == cudaSuccess; i++)
		e = cudaStreamSynchronize(devs[i]->stream);
	const double tb2 = p2_now();
	if (e == cudaSuccess)
		e = p2_scratch_alloc((void **)&dbuf, total, d0->stream);
	/* on the stream that owns the pool allocation (a pageable upload is
	 * staged before the call returns, so h may be freed after it) */
	if (e == cudaSuccess)
		e = cudaMemcpyAsync(dbuf, h, up, cudaMemcpyHostToDevice,
			d0->stream);
	free(h);
	const double tb3 = p2_now();
	if (e == cudaSuccess)
		e = cudaMemsetAsync(dbuf + o_ctl, 0, total - o_ctl, d0->stream);
	if (e != cudaSuccess) {
		p2_scratch_free(dbuf, d0->stream);
		log_error("batch: setup: %s", cudaGetErrorString(e));
		return -1;
	}
	cudaEventRecord(d0->t0, d0->stream);
	p2_batch_launch(kind, grid, d0->stream,
		(const struct p2_binst *)(dbuf + o_inst), (uint32_t)n,
		(const struct p2_op *)(dbuf + o_ops),
		(const struct phase2_pass *)(dbuf + o_pass),
		(const struct phase2_rot_rec *)(dbuf + o_rec),
		(const uint64_t *)(dbuf + o_widx),
		(const double *)(dbuf + o_wval),
		(const uint64_t *)(dbuf + o_gidx), (double2 *)(dbuf + o_gout),
		(struct p2_bctl *)(dbuf + o_ctl),
		(unsigned int *)(dbuf + o_status),
		(const double *)(dbuf + o_cum));
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
	if (e == cudaSuccess)
		e = finish_times(dbuf + o_ctl, dbuf + o_status, n);
	float ms = 0.0f;
	if (e == cudaSuccess)
		e = cudaEventElapsedTime(&ms, d0->t0, d0->t1);
	const double tb4 = p2_now();
	p2_scratch_free(dbuf, d0->stream);
	if (getenv("PHASE2_BATCH_TIMING"))
		log_info("batch run: build %.3f s, stream sync %.3f s, alloc+upload"
			 " %.3f s (%zu bytes), kernel+download %.3f s, free %.3f s",
			tb1 - tb0, tb2 - tb1, tb3 - tb2, up, tb4 - tb3,
			p2_now() - tb4);
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

