#ifndef LOG_H
#define LOG_H

/*
 * Leveled logger with the same environment contract as the phase2
 * logger (reference: include/log.h:1-94):
 *
 *   PHASE2_LOG      threshold: trace|debug|info|warn|error|fatal (first
 *                   letter is enough; default info)
 *   PHASE2_LOG_ALL  1 = every rank logs (one rank here; kept for parity)
 *
 * Line format: "YYYY-MM-DD HH:MM:SS.mmm LEVEL [subsys] message".  TRACE,
 * DEBUG and INFO go to stdout, WARN and above to stderr.  log_trace and
 * log_debug compile to nothing unless DEBUG is defined.
 */

#define PHASE2_LOG_ENVVAR "PHASE2_LOG"
#define PHASE2_LOG_ALL_ENVVAR "PHASE2_LOG_ALL"

#ifndef LOG_SUBSYS
#define LOG_SUBSYS "?"
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum log_level {
	LOG_TRACE = 0,
	LOG_DEBUG = 1,
	LOG_INFO = 2,
	LOG_WARN = 3,
	LOG_ERROR = 4,
	LOG_FATAL = 5,
};

/* Current threshold (reference: log.h:61). */
extern int log_threshold;

/* Format and write one record (reference: log.h:63-64). */
void log_emit(int level, const char *subsys, const char *file, int line,
	const char *fmt, ...) __attribute__((format(printf, 5, 6)));

#define log_at(lvl, ...)                                                       \
	do {                                                                   \
		if ((lvl) >= log_threshold)                                    \
			log_emit((lvl), LOG_SUBSYS, __FILE__, __LINE__,        \
				__VA_ARGS__);                                  \
	} while (0)

#ifdef DEBUG
#define log_trace(...) log_at(LOG_TRACE, __VA_ARGS__)
#define log_debug(...) log_at(LOG_DEBUG, __VA_ARGS__)
#else
#define log_trace(...) ((void)0)
#define log_debug(...) ((void)0)
#endif
#define log_info(...) log_at(LOG_INFO, __VA_ARGS__)
#define log_warn(...) log_at(LOG_WARN, __VA_ARGS__)
#define log_error(...) log_at(LOG_ERROR, __VA_ARGS__)
#define log_fatal(...) log_at(LOG_FATAL, __VA_ARGS__)

/* Read the environment; idempotent; 0 or -1 (reference: log.h:83). */
int log_init(void);

/* Flush both sinks (reference: log.h:86). */
void log_fini(void);

#ifdef __cplusplus
}
#endif

#endif /* LOG_H */
