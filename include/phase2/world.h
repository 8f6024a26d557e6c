#ifndef WORLD_H
#define WORLD_H

/*
 * Process lifecycle.  Replaces include/phase2/world.h of
 * Quantum-for-Life/phase2 (lines 16-77).  This library runs one process per
 * GPU with no MPI: the world is a single rank (size 1, rank 0) and
 * world_init binds the process to CUDA device LOCAL_RANK (default 0).
 * world_init fails (WORLD_ERR) when no CUDA device is usable, so the product
 * never runs without its GPU kernels.
 */

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Reference: world.h:16-21. */
enum world_stat {
	WORLD_UNDEF = -1,
	WORLD_READY = 0,
	WORLD_DONE = 1,
	WORLD_ERR = 2,
};

/* Backend number as in the reference build switch (0 = CPU, 2 = CUDA);
 * this library is a CUDA backend. */
#ifndef PHASE2_BACKEND
#define PHASE2_BACKEND 2
#endif
#define WORLD_BACKEND "B200"

/* Reference: world.h:33-38. */
struct world_info {
	enum world_stat stat;
	int size;
	int rank;
	uint64_t seed;
};

/* Start logging, select the CUDA device.  seed must be non-zero.
 * Returns WORLD_READY or WORLD_ERR (reference: world.h:54). */
int world_init(int *argc, char ***argv, uint64_t seed);

/* Returns WORLD_DONE or WORLD_ERR (reference: world.h:66). */
int world_free(void);

/* Snapshot of the world state; returns wd->stat (reference: world.h:75). */
int world_info(struct world_info *wd);

#ifdef __cplusplus
}
#endif

#endif /* WORLD_H */
