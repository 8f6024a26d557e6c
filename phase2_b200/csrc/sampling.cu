/*
 * sampling.cu -- device sampling for qdrift and cmpsit
 * (p2d_sampled_device): per round of samples, the draws (xoshiro256**),
 * the rotation streams (CDF inversion, head terms), the plans (the host
 * planner's own code, plan_core.h) and the programs the persistent kernel
 * (batch.cu) runs, several samples at once on copies of small registers.
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
#include "plan_core.h"

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
		sz[NPC] = sz[POFF] = (G * C != 0 ? G * C : 1) * sizeof(uint32_t);
		sz[SOFF] = G * sizeof(uint32_t);
		sz[REGS] = R * (sizeof(struct p2_binst) +
				       sizeof(struct p2_bctl)) +
			4 * sizeof(unsigned int) + (R - 1) * d->namp * d->elem;
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
		if (p2_scratch_alloc((void **)&b, total, d->stream) ==
			cudaSuccess)
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
	const int kind = p2_batch_kind(d->prec, job->form);
	int per_sm = 0;
	if (e == cudaSuccess)
		e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm,
			p2_batch_kernel(kind), P2_TPB, 0);
	if (e == cudaSuccess)
		e = cudaFuncSetAttribute(k_smp_plan,
			cudaFuncAttributeMaxDynamicSharedMemorySize,
			(int)P2_SMP_PLAN_SMEM);
	/* no op has more tiles than a span-0 pass or a zero (more warps
	 * would only poll) */
	unsigned grid =
		(unsigned)d->sm_count * (unsigned)(per_sm > 0 ? per_sm : 1);
	uint32_t cpt = 0;
	uint64_t most = p2_op_tiles(P2_OP_PASS, d->namp, 0, &cpt);
	const uint32_t zt = p2_op_tiles(P2_OP_ZERO, d->namp, 0, &cpt);
	if (zt > most)
		most = zt;
	most = (most * R + P2_BATCH_WARPS - 1) / P2_BATCH_WARPS;
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
			e = cudaMemsetAsync(status, 0, 4 * sizeof(unsigned int),
				d->stream);
		if (e == cudaSuccess)
			p2_batch_launch(kind, grid, d->stream, inst, nreg,
				(const struct p2_op *)(b + off[PROG]),
				(const struct phase2_pass *)(b + off[PASS]),
				(const struct phase2_rot_rec *)(b + off[REC]),
				(const uint64_t *)(b + off[WIDX]),
				(const double *)(b + off[WVAL]),
				(const uint64_t *)(b + off[GIDX]),
				(double2 *)(b + off[GOUT]), ctl, status, NULL);
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
	p2_scratch_free(b, d->stream);
	return rc;
}

