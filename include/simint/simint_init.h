#pragma once
/* Library set-up and tear-down. */
#ifdef __cplusplus
extern "C" {
#endif

/* Replaces simint_init (skel/simint/simint_init.h:21, simint_init.c:4-8).
 * Idempotent.  Selects the CUDA device (the current one), uploads the Boys
 * grid and builds the per-class kernel table.  Not thread safe. */
void simint_init(void);

/* Replaces simint_finalize (skel/simint/simint_init.h:37, simint_init.c:11-15).
 * Idempotent.  Releases every device buffer the library cached. */
void simint_finalize(void);

#ifdef __cplusplus
}
#endif
