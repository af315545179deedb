/*
 * memory_extern.c -- emits the external definitions of the C99 `inline`
 * helpers declared in the reference's src/src_c/memory.h (aligned_malloc,
 * aligned_malloc_64byte, aligned_free, lines 16-48).  In C99/C11 an `inline`
 * definition without `extern` provides no out-of-line symbol, so a build in
 * which the compiler declines to inline a call fails to link.  Declaring the
 * functions `extern` in exactly one translation unit is the standard fix; the
 * reference sources themselves stay unmodified.  TEST INFRASTRUCTURE ONLY.
 */
#include "memory.h"

extern void *aligned_malloc(size_t size, size_t alignment);
extern void *aligned_malloc_64byte(size_t size);
extern void aligned_free(void *ptr);
