/*
 * sweep.cu -- sweeps (phase2_set_sweep): a plan's run of passes whose
 * bases fit one shared-memory tile, run as one kernel with one read and
 * one write of the state (k_sweep32), and the host code that checks a
 * planned sweep against the tile shape and lays out its descriptor.
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

bool p2_sweeps_on(const struct p2_dev *d)
{
	return p2_sweep_tile > 0 && p2_sweep_kernel &&
		d->prec == PHASE2_PREC_FP32 && d->nqb <= 31 &&
		d->nqb >= (uint32_t)p2_sweep_tile + 3;
}

long p2_sweep_launch(struct p2_dev *d, const struct phase2_pass *passes,
	size_t npass, size_t i, const struct phase2_rot_rec *d_recs)
{
	struct p2_sweep sw;
	const size_t n = sweep_from(passes, npass, i, &sw);
	if (n < 2)
		return 1;
	return launch_sweep(d, sw, d_recs) < 0 ? -1 : (long)n;
}
