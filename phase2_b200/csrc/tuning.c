/*
 * tuning.c -- the measured launch table shipped beside the library
 * (tuning_b200.tab, written by phase2_b200/autotune.py from its timings)
 * and its loading at world_init.
 *
 * File format, one entry per line ('#' starts a comment line):
 *   gpu <device name as the CUDA runtime reports it>
 *   launch <prec 0|1> <span 0..5> <variant> <per_sm>
 *   batch_runs <1..64>     (phase2_set_batch_runs: persistent run length)
 * A table applies only to a device of the same name: launch choices that
 * were measured on one GPU are not carried to another.
 */
#define _GNU_SOURCE

#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define LOG_SUBSYS "tuning"
#include "log.h"

#include "phase2_b200.h"

#include "p2_internal.h"

#define TUNING_FILE "tuning_b200.tab"

static void chomp(char *s)
{
	size_t n = strlen(s);
	while (n && (s[n - 1] == '\n' || s[n - 1] == '\r' || s[n - 1] == ' ' ||
		       s[n - 1] == '\t'))
		s[--n] = '\0';
}

int phase2_load_tuning(const char *path, const char *gpu)
{
	char name[256];
	if (!path)
		return -1;
	if (!gpu) {
		if (p2d_device_name(name, sizeof name) < 0)
			return -1;
		gpu = name;
	}
	FILE *f = fopen(path, "r");
	if (!f) {
		log_debug("no launch table at %s", path);
		return -1;
	}
	/* first pass: validate every line and find the GPU name */
	char line[512];
	int match = -1, bad = 0;
	while (fgets(line, sizeof line, f)) {
		chomp(line);
		char *p = line;
		while (*p == ' ' || *p == '\t')
			p++;
		if (*p == '\0' || *p == '#')
			continue;
		if (strncmp(p, "gpu ", 4) == 0) {
			match = strcmp(p + 4, gpu) == 0;
			continue;
		}
		int prec, span, variant, per_sm, runs;
		char tail;
		if (strncmp(p, "batch_runs ", 11) == 0) {
			if (sscanf(p, "batch_runs %d %c", &runs, &tail) != 1 ||
				runs < 1 || runs > 64) {
				log_error("launch table %s: bad line \"%s\"", path,
					p);
				bad = 1;
				break;
			}
			continue;
		}
		if (sscanf(p, "launch %d %d %d %d %c", &prec, &span, &variant,
			    &per_sm, &tail) != 4 ||
			prec < 0 || prec > 1 || span < 0 ||
			span > PHASE2_MAX_SPAN) {
			log_error("launch table %s: bad line \"%s\"", path, p);
			bad = 1;
			break;
		}
	}
	if (bad || match < 0) {
		if (!bad)
			log_error("launch table %s: no gpu line", path);
		fclose(f);
		return -1;
	}
	if (!match) {
		fclose(f);
		log_debug("launch table %s is for another GPU", path);
		return 0;
	}
	/* second pass: apply */
	rewind(f);
	int applied = 0;
	while (fgets(line, sizeof line, f)) {
		int prec, span, variant, per_sm, runs;
		char *p = line;
		while (*p == ' ' || *p == '\t')
			p++;
		if (sscanf(p, "batch_runs %d", &runs) == 1) {
			phase2_set_batch_runs((unsigned int)runs);
			applied++;
			continue;
		}
		if (sscanf(p, "launch %d %d %d %d", &prec, &span, &variant,
			    &per_sm) == 4) {
			if (phase2_tune_set(prec, span, variant, per_sm) < 0) {
				log_error("launch table %s: entry %d %d %d %d "
					  "refused",
					path, prec, span, variant, per_sm);
				fclose(f);
				return -1;
			}
			applied++;
		}
	}
	fclose(f);
	return applied;
}

void p2_tuning_at_init(void)
{
	const char *env = getenv("PHASE2_TUNING");
	if (env && strcmp(env, "off") == 0)
		return;
	char path[4096];
	if (env && *env) {
		snprintf(path, sizeof path, "%s", env);
	} else {
		/* the table ships in the directory of this library */
		Dl_info info;
		if (!dladdr((void *)&phase2_load_tuning, &info) ||
			!info.dli_fname)
			return;
		snprintf(path, sizeof path, "%s", info.dli_fname);
		char *slash = strrchr(path, '/');
		if (slash)
			slash[1] = '\0';
		else
			path[0] = '\0';
		strncat(path, TUNING_FILE, sizeof path - strlen(path) - 1);
	}
	const int n = phase2_load_tuning(path, NULL);
	if (n > 0)
		log_info("launch table: %d entries from %s", n, path);
}
