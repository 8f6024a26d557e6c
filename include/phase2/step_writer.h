#ifndef PHASE2_STEP_WRITER_H
#define PHASE2_STEP_WRITER_H

/*
 * Per-step output callback of the drivers.  Replaces
 * include/phase2/step_writer.h of Quantum-for-Life/phase2 (lines 21-24):
 * `write` is called once per step (or sample) with that step's overlap and
 * returns 0 or -1; a NULL writer disables per-step output.
 */

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

struct phase2_step_writer {
	void *ctx;
	int (*write)(void *ctx, size_t step_idx, _Complex double z);
};

#ifdef __cplusplus
}
#endif

#endif /* PHASE2_STEP_WRITER_H */
