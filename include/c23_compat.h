/*
 * c23_compat.h -- the few C23 spellings phase2 code uses, for C11
 * compilers.  Provided so that code written against the phase2 headers
 * (include/c23_compat.h in Quantum-for-Life/phase2) compiles unchanged
 * against this library.
 */
#ifndef C23_COMPAT_H
#define C23_COMPAT_H

#include <stdbool.h>

#ifndef __cplusplus
#define nullptr ((void *)0)
#endif
#define stdc_count_ones_ul(v) (__builtin_popcountl(v))
#define unreachable() (__builtin_unreachable())

#ifndef static_assert
#define static_assert _Static_assert
#endif

#endif /* C23_COMPAT_H */
