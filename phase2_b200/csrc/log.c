/*
 * log.c -- leveled logger with the phase2 environment contract
 * (include/log.h of Quantum-for-Life/phase2): PHASE2_LOG sets the
 * threshold, PHASE2_LOG_ALL is accepted for parity (there is one rank).
 */
#define _POSIX_C_SOURCE 200809L

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "log.h"

int log_threshold = LOG_INFO;

static int log_ready;

static const char *const LEVEL_TAG[] = { "TRACE", "DEBUG", "INFO", "WARN",
	"ERROR", "FATAL" };

static int level_from(const char *s, int *out)
{
	if (!s || !*s)
		return -1;
	switch (s[0] | 0x20) {
	case 't':
		*out = LOG_TRACE;
		return 0;
	case 'd':
		*out = LOG_DEBUG;
		return 0;
	case 'i':
		*out = LOG_INFO;
		return 0;
	case 'w':
		*out = LOG_WARN;
		return 0;
	case 'e':
		*out = LOG_ERROR;
		return 0;
	case 'f':
		*out = LOG_FATAL;
		return 0;
	}
	return -1;
}

int log_init(void)
{
	if (log_ready)
		return 0;
	int lvl;
	if (level_from(getenv(PHASE2_LOG_ENVVAR), &lvl) == 0)
		log_threshold = lvl;
	setvbuf(stderr, NULL, _IONBF, 0);
	log_ready = 1;
	return 0;
}

void log_fini(void)
{
	fflush(stdout);
	fflush(stderr);
}

void log_emit(int level, const char *subsys, const char *file, int line,
	const char *fmt, ...)
{
	(void)file;
	(void)line;
	if (level < LOG_TRACE)
		level = LOG_TRACE;
	if (level > LOG_FATAL)
		level = LOG_FATAL;
	struct timespec ts;
	struct tm tm;
	clock_gettime(CLOCK_REALTIME, &ts);
	localtime_r(&ts.tv_sec, &tm);
	char stamp[32];
	strftime(stamp, sizeof stamp, "%Y-%m-%d %H:%M:%S", &tm);
	char msg[4096];
	va_list ap;
	va_start(ap, fmt);
	vsnprintf(msg, sizeof msg, fmt, ap);
	va_end(ap);
	FILE *out = level >= LOG_WARN ? stderr : stdout;
	fprintf(out, "%s.%03ld %-5s [%s] %s\n", stamp, ts.tv_nsec / 1000000L,
		LEVEL_TAG[level], subsys ? subsys : "?", msg);
	fflush(out);
}
