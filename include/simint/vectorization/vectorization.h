#pragma once
/* Layout constants of the pair arrays.  The GPU engine keeps the padding of
 * the reference's 8-wide (AVX-512) build so that simint_multi_shellpair
 * objects have the same size and element positions
 * (skel/simint/vectorization/vectorization.h:71,81;
 * intrinsics_avx512.h:69).  Host callers also use SIMINT_ALLOC/SIMINT_FREE for
 * their work and output buffers (skel/test/test_eri.cpp:72-77). */
#include <stdlib.h>

#define SIMINT_SIMD_LEN 8
#define SIMINT_SIMD_ALIGN_DBL (SIMINT_SIMD_LEN*8)
#define SIMINT_SIMD_ALIGN_INT (SIMINT_SIMD_LEN*sizeof(int))
#define SIMINT_SIMD_ALIGN SIMINT_SIMD_ALIGN_DBL
#define SIMINT_SIMD_ROUND(x) (((x) + ((SIMINT_SIMD_LEN-1))) & (~(SIMINT_SIMD_LEN-1)))
#define SIMINT_NSHELL_SIMD (2*SIMINT_SIMD_LEN)

static inline void * simint_malloc_aligned(size_t size, size_t alignment)
{
    void * ptr = NULL;
    if(posix_memalign(&ptr, alignment, size) != 0)
        return NULL;
    return ptr;
}

static inline void simint_free_aligned(void * mem) { free(mem); }

#define SIMINT_ALLOC(x) simint_malloc_aligned((x), SIMINT_SIMD_ALIGN)
#define SIMINT_FREE(x) simint_free_aligned((x))
#define SIMINT_ALIGN_ARRAY_DBL __attribute__((aligned(SIMINT_SIMD_ALIGN_DBL)))
