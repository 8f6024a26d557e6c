/*
 * world.c -- process lifecycle (include/phase2/world.h).  Same contract as
 * phase2/world.c of Quantum-for-Life/phase2 (lines 19-112) for one rank:
 * a zero seed is an error, logging starts, and the backend is brought up,
 * which here means binding CUDA device LOCAL_RANK (default 0).  No device
 * means WORLD_ERR: the library has no CPU fallback.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "world"
#include "log.h"

#include "phase2/world.h"

#include "p2_internal.h"
#include "p2_host.h"

static struct world_info WORLD = {
	.stat = WORLD_UNDEF,
	.size = 0,
	.rank = 0,
	.seed = UINT64_C(0x77dd8e60521fb661),
};

int world_init(int *argc, char ***argv, uint64_t seed)
{
	(void)argc;
	(void)argv;
	if (seed == 0)
		return WORLD.stat = WORLD_ERR;
	if (log_init() < 0)
		return WORLD.stat = WORLD_ERR;

	int dev = 0;
	const char *lr = getenv("LOCAL_RANK");
	if (lr && *lr)
		dev = atoi(lr);
	if (p2d_device_init(dev, NULL) < 0) {
		log_error("world_init: CUDA device %d unavailable", dev);
		return WORLD.stat = WORLD_ERR;
	}
	/* the shipped launch table first, so that settings from the
	 * environment override it */
	p2_tuning_at_init();
	p2_settings_from_env();

	WORLD.size = 1;
	WORLD.rank = 0;
	WORLD.seed = seed;
	WORLD.stat = WORLD_READY;
	log_info("*** Init ***");
	log_info("World size: %d", WORLD.size);
	log_info("Backend: %s (device %d)", WORLD_BACKEND, dev);
	return WORLD.stat;
}

int world_free(void)
{
	if (WORLD.stat == WORLD_READY)
		WORLD.stat = WORLD_DONE;
	log_fini();
	return WORLD.stat;
}

int world_info(struct world_info *wd)
{
	if (wd)
		*wd = WORLD;
	return WORLD.stat;
}
