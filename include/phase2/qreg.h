#ifndef QREG_H
#define QREG_H

/*
 * State-vector register resident in GPU memory.
 *
 * Replaces include/phase2/qreg.h of Quantum-for-Life/phase2 (lines 20-85)
 * with the same functions and field names.  Differences that follow from
 * running on one B200 without MPI:
 *
 *   - One rank: qb_hi = 0, qb_lo = nqb, namp = 2^nqb.
 *   - The canonical state lives in device memory (reg->backend), in place:
 *     no partner buffer, so 2^nqb * 16 B (FP64) or 2^nqb * 8 B (FP32).
 *   - reg->amp is a host shadow used only by qreg_sync_*; it is allocated
 *     at init for nqb <= 24 and on the first qreg_sync_device_to_host call
 *     otherwise.  reg->buf is always NULL.
 *   - reqs_snd / reqs_rcv keep their names for source compatibility but are
 *     opaque and unused.
 *   - qreg_paulirot may defer work: rotations are queued and executed in
 *     fused passes on the register's CUDA stream.  Every call that observes
 *     or replaces the state (getamp, setamp, zero, sync_*) first drains the
 *     queue, so results are as if each rotation ran immediately.
 */

#include <stddef.h>
#include <stdint.h>

#include "phase2/paulis.h"
#include "phase2/world.h"

#ifdef __cplusplus
extern "C" {
#endif

#define QREG_MAX_WIDTH (64)

/* Reference: qreg.h:25-42. */
struct qreg {
	struct world_info wd;

	uint32_t qb_lo, qb_hi;

	_Complex double *amp, *buf;
	uint64_t namp;

	int msg_count;
	void *reqs_snd, *reqs_rcv;
	size_t nreqs;

	void *backend;
};

/* Allocate a zeroed-on-demand register of nqb qubits in device memory at
 * the process default precision (FP64 unless changed, see phase2_b200.h).
 * Requires a ready world; 1 <= nqb <= QREG_MAX_WIDTH and the state must fit
 * in device memory.  0 or -1 (reference: qreg.h:48). */
int qreg_init(struct qreg *reg, uint32_t qb);

/* Release device and host memory (reference: qreg.h:50). */
void qreg_free(struct qreg *reg);

/* *z = amplitude i, read back as FP64 (reference: qreg.h:54). */
void qreg_getamp(struct qreg *reg, uint64_t i, _Complex double *z);

/* amplitude i = z (rounded to FP32 on an FP32 register)
 * (reference: qreg.h:58). */
void qreg_setamp(struct qreg *reg, uint64_t i, _Complex double z);

/* All amplitudes = 0 (reference: qreg.h:61). */
void qreg_zero(struct qreg *reg);

/* Bulk copy between the host shadow reg->amp and the device state
 * (reference: qreg.h:79-80). */
void qreg_sync_host_to_device(struct qreg *reg);
void qreg_sync_device_to_host(struct qreg *reg);

/* Apply prod_k exp(i phis[k] (code_hi (x) codes_lo[k])) in order k = 0..n-1
 * (reference: qreg.h:84-85).  With one rank code_hi acts on no qubit
 * beyond qb_lo; any bits it carries are combined with codes_lo[k]. */
void qreg_paulirot(struct qreg *reg, struct paulis code_hi,
	const struct paulis *codes_lo, const double *phis, size_t ncodes);

#ifdef __cplusplus
}
#endif

#endif /* QREG_H */
