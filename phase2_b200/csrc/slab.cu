/*
 * slab.cu -- half-slab gather and scatter for registers sharded by high
 * qubits (qreg_slab_get / qreg_slab_put).
 *
 * A register of nqb qubits split over 2^g ranks keeps 2^(nqb-g) amplitudes
 * per rank: the rank number supplies the g high index bits.  The reference
 * applies a rotation whose flip touches a high qubit by swapping the whole
 * slab with the partner rank and rotating both copies (phase2/qreg.c:
 * 124-142, phase2/qreg_cuda.c:139-162).  The sharded register of this
 * library (phase2_b200/sharded.py) instead swaps a high qubit with a local
 * qubit l: each rank sends the half of its slab whose bit l differs from
 * its own rank bit and receives the partner's matching half into the same
 * places.  These kernels move such a half (the amplitudes whose index has
 * bit `bit` equal to `val`, in increasing index order) between the
 * register's state and a contiguous device buffer, in chunks, so that the
 * exchange buffers stay small.
 */
#include <cuda.h>
#include <cuda_runtime.h>

#include <stdint.h>
#include <stdio.h>

#define LOG_SUBSYS "engine"
#include "log.h"

#include "p2_engine.h"

/* Element j of the half {i : bit `bit` of i == val}: j with a bit of value
 * val inserted at position `bit`. */
__device__ __forceinline__ uint64_t p2_half_index(uint64_t j, uint32_t bit,
	uint64_t val)
{
	const uint64_t low = j & ((UINT64_C(1) << bit) - 1);
	return ((j ^ low) << 1) | (val << bit) | low;
}

/*
 * T is one state element (float2, double2) or, for FP32 halves with bit >=
 * 1, a pair of them (float4): elements 2m and 2m + 1 of such a half are
 * neighbours in the state, so indices below count in units of T.
 */
/* Items per thread and loop trip, all loaded before any is stored: with
 * one 16-byte item in flight per thread the copy stalls on memory latency
 * (ncu: long-scoreboard stalls, DRAM well below its peak). */
#define P2_SLAB_UNROLL 4

template <typename T, bool PUT>
__global__ void __launch_bounds__(256) k_slab_copy(T *__restrict__ st,
	T *__restrict__ buf, uint32_t bit, uint64_t val, uint64_t first,
	uint64_t count)
{
	const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t k0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		k0 < count; k0 += nt * P2_SLAB_UNROLL) {
		T v[P2_SLAB_UNROLL];
#pragma unroll
		for (int u = 0; u < P2_SLAB_UNROLL; ++u) {
			const uint64_t k = k0 + u * nt;
			if (k < count)
				v[u] = PUT ? buf[k]
					   : st[p2_half_index(first + k, bit, val)];
		}
#pragma unroll
		for (int u = 0; u < P2_SLAB_UNROLL; ++u) {
			const uint64_t k = k0 + u * nt;
			if (k < count) {
				if (PUT)
					st[p2_half_index(first + k, bit, val)] = v[u];
				else
					buf[k] = v[u];
			}
		}
	}
}

/* Exchange element j of half (bit, va) of a with element j of half (bit,
 * vb) of b, for j < count (units of T as in k_slab_copy). */
template <typename T>
__global__ void __launch_bounds__(256) k_slab_swap(T *__restrict__ a,
	T *__restrict__ b, uint32_t bit, uint64_t va, uint64_t vb,
	uint64_t count)
{
	const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
	for (uint64_t j0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
		j0 < count; j0 += nt * P2_SLAB_UNROLL) {
		T x[P2_SLAB_UNROLL], y[P2_SLAB_UNROLL];
#pragma unroll
		for (int u = 0; u < P2_SLAB_UNROLL; ++u) {
			const uint64_t j = j0 + u * nt;
			if (j < count) {
				x[u] = a[p2_half_index(j, bit, va)];
				y[u] = b[p2_half_index(j, bit, vb)];
			}
		}
#pragma unroll
		for (int u = 0; u < P2_SLAB_UNROLL; ++u) {
			const uint64_t j = j0 + u * nt;
			if (j < count) {
				a[p2_half_index(j, bit, va)] = y[u];
				b[p2_half_index(j, bit, vb)] = x[u];
			}
		}
	}
}

typedef CUresult (*p2_addr_range_fn)(CUdeviceptr *, size_t *, CUdeviceptr);

/* 0 if [p, p + bytes) is device memory of the current device inside one
 * allocation; -1 (logged) otherwise, also when the allocation cannot be
 * looked up (no copy runs unchecked). */
int p2_check_device_range(const void *p, size_t bytes, const char *what)
{
	int dev = 0;
	cudaPointerAttributes a;
	if (cudaGetDevice(&dev) != cudaSuccess ||
		cudaPointerGetAttributes(&a, p) != cudaSuccess) {
		cudaGetLastError();
		log_error("%s: cannot query the buffer pointer", what);
		return -1;
	}
	if ((a.type != cudaMemoryTypeDevice &&
		    a.type != cudaMemoryTypeManaged) ||
		a.device != dev) {
		log_error("%s: the buffer is not device memory of device %d",
			what, dev);
		return -1;
	}
	static p2_addr_range_fn range_fn;
	static int looked_up;
	if (!looked_up) {
		void *fn = NULL;
		cudaDriverEntryPointQueryResult q;
		if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &fn,
			    cudaEnableDefault, &q) == cudaSuccess &&
			q == cudaDriverEntryPointSuccess)
			range_fn = (p2_addr_range_fn)fn;
		cudaGetLastError();
		looked_up = 1;
	}
	if (!range_fn) {
		log_error("%s: cannot look up the buffer's allocation", what);
		return -1;
	}
	CUdeviceptr base = 0;
	size_t size = 0;
	const CUdeviceptr ptr = (CUdeviceptr)(uintptr_t)p;
	if (range_fn(&base, &size, ptr) != CUDA_SUCCESS || ptr < base ||
		ptr - base > size || bytes > size - (ptr - base)) {
		log_error("%s: %zu bytes at the buffer pointer exceed its"
			  " allocation", what, bytes);
		return -1;
	}
	return 0;
}

extern "C" int p2d_slab_copy(struct p2_dev *d, uint32_t bit, uint32_t val,
	uint64_t first, uint64_t count, void *buf, int put)
{
	const char *what = put ? "qreg_slab_put" : "qreg_slab_get";
	if (bit >= d->nqb || val > 1) {
		log_error("%s: bit %u / value %u outside a %u-qubit register",
			what, bit, val, d->nqb);
		return -1;
	}
	const uint64_t nhalf = d->namp >> 1;
	if (first > nhalf || count > nhalf - first) {
		log_error("%s: elements [%llu, +%llu) outside the half of %llu",
			what, (unsigned long long)first,
			(unsigned long long)count, (unsigned long long)nhalf);
		return -1;
	}
	if (count == 0)
		return 0;
	if (!buf) {
		log_error("%s: NULL buffer", what);
		return -1;
	}
	if ((uintptr_t)buf % d->elem) {
		log_error("%s: buffer not aligned to %zu bytes", what, d->elem);
		return -1;
	}
	if (p2_check_device_range(buf, count * d->elem, what) < 0)
		return -1;
	const unsigned grid = grid_for(d, count, 256, 8);
	if (d->prec == PHASE2_PREC_FP64) {
		double2 *st = (double2 *)d->state, *b = (double2 *)buf;
		if (put)
			k_slab_copy<double2, true><<<grid, 256, 0, d->stream>>>(
				st, b, bit, val, first, count);
		else
			k_slab_copy<double2, false><<<grid, 256, 0, d->stream>>>(
				st, b, bit, val, first, count);
	} else if (bit >= 1 && first % 2 == 0 && count % 2 == 0 &&
		(uintptr_t)buf % 16 == 0) {
		/* pairs of FP32 amplitudes: 16-byte accesses; bit - 1 is the
		 * bit's position in pair units */
		float4 *st = (float4 *)d->state, *b = (float4 *)buf;
		const unsigned g2 = grid_for(d, count / 2, 256, 8);
		if (put)
			k_slab_copy<float4, true><<<g2, 256, 0, d->stream>>>(
				st, b, bit - 1, val, first / 2, count / 2);
		else
			k_slab_copy<float4, false><<<g2, 256, 0, d->stream>>>(
				st, b, bit - 1, val, first / 2, count / 2);
	} else {
		float2 *st = (float2 *)d->state, *b = (float2 *)buf;
		if (put)
			k_slab_copy<float2, true><<<grid, 256, 0, d->stream>>>(
				st, b, bit, val, first, count);
		else
			k_slab_copy<float2, false><<<grid, 256, 0, d->stream>>>(
				st, b, bit, val, first, count);
	}
	CUDA_OK(cudaGetLastError(), "slab copy launch");
	d->launches++;
	CUDA_OK(cudaStreamSynchronize(d->stream), "slab copy");
	return 0;
}

extern "C" int p2d_slab_swap(struct p2_dev *a, struct p2_dev *b,
	uint32_t bit, uint32_t va, uint32_t vb)
{
	if (a == b || a->nqb != b->nqb || a->prec != b->prec) {
		log_error("qreg_slab_swap: needs two registers of one size and"
			  " precision");
		return -1;
	}
	if (bit >= a->nqb || va > 1 || vb > 1) {
		log_error("qreg_slab_swap: bit %u / values %u %u outside a"
			  " %u-qubit register", bit, va, vb, a->nqb);
		return -1;
	}
	cudaPointerAttributes pa, pb;
	CUDA_OK(cudaPointerGetAttributes(&pa, a->state), "slab swap: state a");
	CUDA_OK(cudaPointerGetAttributes(&pb, b->state), "slab swap: state b");
	if (pa.device != pb.device) {
		log_error("qreg_slab_swap: registers on devices %d and %d",
			pa.device, pb.device);
		return -1;
	}
	/* b's queued work first; the swap itself runs on a's stream */
	CUDA_OK(cudaStreamSynchronize(b->stream), "slab swap: stream b");
	const uint64_t nhalf = a->namp >> 1;
	if (a->prec == PHASE2_PREC_FP64) {
		k_slab_swap<double2><<<grid_for(a, nhalf, 256, 8), 256, 0,
			a->stream>>>((double2 *)a->state, (double2 *)b->state,
			bit, va, vb, nhalf);
	} else if (bit >= 1) {
		k_slab_swap<float4><<<grid_for(a, nhalf / 2, 256, 8), 256, 0,
			a->stream>>>((float4 *)a->state, (float4 *)b->state,
			bit - 1, va, vb, nhalf / 2);
	} else {
		k_slab_swap<float2><<<grid_for(a, nhalf, 256, 8), 256, 0,
			a->stream>>>((float2 *)a->state, (float2 *)b->state,
			bit, va, vb, nhalf);
	}
	CUDA_OK(cudaGetLastError(), "slab swap launch");
	a->launches++;
	CUDA_OK(cudaStreamSynchronize(a->stream), "slab swap");
	return 0;
}
