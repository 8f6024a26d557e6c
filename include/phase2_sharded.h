/*
 * phase2_sharded.h -- registers sharded by their high qubits, for C hosts.
 *
 * An nqb-qubit register over world = 2^g ranks keeps L = nqb - g qubits
 * on each rank: rank r holds the 2^L amplitudes whose physical index has r
 * in its g high bits (the reference's layout, phase2/qreg.c:46-66).  The
 * reference applies a rotation whose flip touches a high qubit by
 * exchanging the whole slab with the partner rank, mixing, rotating both
 * copies and adding (phase2/qreg.c:124-142, phase2/qreg_qreg.c:123-166).
 * Here a high qubit is swapped in instead: high position h (rank bit
 * b = h - L) and a local position l trade places, which moves half of
 * every slab across the pair (r, r ^ 2^b) once, and the qubit then stays
 * local.  The local position chosen is, among those outside the rotation's
 * flip, the one whose qubit the rotations that follow flip again farthest
 * ahead (within 4096 rotations).  A Z on a high position is the fixed
 * sign (-1)^popc(r & z_hi) of P on rank r's slab, so each rank applies
 * exp(i sigma phi P_lo) to its slab with the ordinary engine: an FP64
 * sharded register gives the bits of one register of nqb qubits.
 *
 * A process holds one or more of the ranks (its own, or all of them on one
 * GPU).  Pairs that it holds both halves of trade them in place
 * (qreg_slab_swap); pairs split between processes go through the caller's
 * transport, chunk by chunk (qreg_slab_get into a device buffer of the
 * library, exchange, qreg_slab_put).  Every process must make the same
 * calls in the same order, with the same arguments: swap decisions depend
 * only on the rotation sequence, so the transport sees the same sequence
 * of exchanges and sums on every rank.
 *
 * Same functions as the Python layer (phase2_b200/sharded.py), for hosts
 * that drive NCCL, MPI or a transport of their own from C.
 */
#ifndef PHASE2_SHARDED_H
#define PHASE2_SHARDED_H

#include <stddef.h>
#include <stdint.h>

#include "circ/cmpsit.h"
#include "phase2/circ.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * The caller's transport between processes.
 * exchange: send `bytes` from device memory `send` to rank `peer` and
 *   receive `bytes` from it into device memory `recv` (both buffers the
 *   library's, on this process's GPU); `rank` is the sending rank of this
 *   process.  Both ranks of the pair make the matching call.  Finished when
 *   it returns; 0 or -1.  A process makes a swap's exchanges in increasing
 *   order of its ranks (whatever order `ranks` listed them in), which is
 *   increasing order of the pairs on every process: a blocking pairwise
 *   transport cannot deadlock.  After a failed exchange the register's
 *   state is undefined until the next prepst.
 * sum: element-wise sum of n doubles (host memory) over the processes, in
 *   place, the same result on every process (each process passes the sum
 *   over the ranks it holds).  0 or -1.
 * A process that holds every rank needs no transport (pass NULL).
 */
struct phase2_shard_io {
	int (*exchange)(void *ctx, uint32_t rank, uint32_t peer,
		const void *send, void *recv, size_t bytes);
	int (*sum)(void *ctx, double *vals, size_t n);
	void *ctx;
};

struct phase2_sharded;

/*
 * nqb qubits over `world` ranks (a power of two, nqb - log2(world) >= 1
 * local qubits); this process holds ranks[0..nranks) (distinct, below
 * world), as registers of precision prec (PHASE2_PREC_FP32 / _FP64) on
 * the current device.  chunk: amplitudes per exchange through the
 * transport (0: 2^26).  World must be initialised.  NULL on error.
 */
struct phase2_sharded *phase2_sharded_new(uint32_t nqb, uint32_t world,
	const uint32_t *ranks, uint32_t nranks, int prec,
	const struct phase2_shard_io *io, uint64_t chunk);
void phase2_sharded_free(struct phase2_sharded *s);

/* exp(+i phi[k] P_k) for k = 0..n-1 in order, P_k = (flip[k], phase[k])
 * over global qubits (struct paulis pak[0] / pak[1]).  0 or -1 (a flip
 * wider than the local qubits, or a string beyond the register). */
int phase2_sharded_paulirot(struct phase2_sharded *s, const uint64_t *flip,
	const uint64_t *phase, const double *phi, size_t n);

/* |psi> = sum_d cf[d] |idx[d]> (global indices; later entries win). */
int phase2_sharded_prepst(struct phase2_sharded *s, const uint64_t *idx,
	const _Complex double *cf, size_t ndet);

/* Amplitudes at global indices, on every process. */
int phase2_sharded_getamps(struct phase2_sharded *s, const uint64_t *idx,
	_Complex double *out, size_t n);

/* sum_d conj(cf[d]) a[idx[d]], in det order (circ_measure's expression). */
int phase2_sharded_measure(struct phase2_sharded *s, const uint64_t *idx,
	const _Complex double *cf, size_t ndet, _Complex double *z);

/* sum |a_i|^2: each rank's device reduction, added in rank order. */
int phase2_sharded_norm2(struct phase2_sharded *s, double *out);

/* Run every queued rotation of the ranks held and wait for the device;
 * -1 if a CUDA error is pending. */
int phase2_sharded_synchronize(struct phase2_sharded *s);

/* pos[q]: the physical position of global qubit q (nqb entries). */
int phase2_sharded_layout(const struct phase2_sharded *s, uint32_t *pos);

/* Qubit swaps performed, amplitudes this process sent or traded. */
void phase2_sharded_counters(const struct phase2_sharded *s,
	uint64_t *swaps, uint64_t *exchanged);

/*
 * The drivers on a sharded register, one overlap per step or sample into
 * out (the reference's drivers, circ/trott.c:44-65, circ/trott2.c:44-74,
 * circ/qdrift.c:95-134, circ/cmpsit.c:151-235): trott / trott2 (order2)
 * sort a copy of the Hamiltonian with circ_hamil_sort_lex; qdrift draws
 * with prob_cdf and xoshiro256** as qdrift_simul does for the same seed
 * (non-zero); cmpsit splits the terms with cmpsit_ranct_init and draws as
 * cmpsit_simul.  Every process draws the same sequence.  0 or -1.
 */
int phase2_sharded_trott(struct phase2_sharded *s,
	const struct circ_hamil *hm, const struct circ_muldet *md, size_t steps,
	double delta, int order2, _Complex double *out);
int phase2_sharded_qdrift(struct phase2_sharded *s,
	const struct circ_hamil *hm, const struct circ_muldet *md,
	size_t samples, size_t depth, double step_size, uint64_t seed,
	_Complex double *out);
int phase2_sharded_cmpsit(struct phase2_sharded *s,
	const struct circ_hamil *hm, const struct circ_muldet *md,
	const struct cmpsit_data *dt, _Complex double *out);

#ifdef __cplusplus
}
#endif

#endif /* PHASE2_SHARDED_H */
