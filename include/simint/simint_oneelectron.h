#pragma once
/* One-electron integrals over contracted Cartesian shells: overlap, kinetic
 * energy and nuclear attraction (point charges).  Same prototypes as the
 * reference's skel/simint/simint_oneelectron.h:12-27; computed on the GPU
 * (one warp per shell pair).  Each call writes the ncart(a) x ncart(b) block,
 * row-major, Cartesians in the fixed lexicographic order (x descending, then
 * y; skel/simint/recur_lookup.c), whatever the ERI ordering, and returns 1,
 * or a negative SIMINT_B200_ERR_* code (simint_b200.h): am > 4 gives
 * SIMINT_B200_ERR_CLASS, no device SIMINT_B200_ERR_NODEVICE. */

#include "simint/shell/shell.h"

#ifdef __cplusplus
extern "C" {
#endif

/* skel/simint/simint_oneelectron.h:12-14 */
int simint_compute_overlap(struct simint_shell * a,
                           struct simint_shell * b,
                           double * integrals);

/* skel/simint/simint_oneelectron.h:16-18 */
int simint_compute_ke(struct simint_shell * a,
                      struct simint_shell * b,
                      double * integrals);

/* skel/simint/simint_oneelectron.h:21-26: -sum_C Z_C (a| 1/|r - C| |b) */
int simint_compute_potential(int ncenter,
                             double * Z, double * x, double * y, double * z,
                             struct simint_shell const * sh1,
                             struct simint_shell const * sh2,
                             double * integrals);

#ifdef __cplusplus
}
#endif
