#pragma once
/* Two-electron repulsion integrals over multi-shell-pairs. */
#include <stddef.h>
#include "simint/shell/shell.h"
#include "simint/ostei/ostei_config.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces simint_compute_eri (skel/simint/simint_eri.h:22-26,
 * simint_eri.c:4-11, ostei.c:10-23).
 * Computes (ab|cd) for every bra pair of P and ket pair of Q (the first
 * nshell12_clip pairs of each) on the GPU.  P, Q and integrals are host
 * memory.  The output is shell-quartet major (bra outer, ket inner), then
 * Cartesians a,b,c,d row major in the library's ordering.  Returns
 * P->nshell12_clip * Q->nshell12_clip, or -1 when the pair-level Schwarz test
 * screens everything (nothing is written).  work may be NULL: the GPU path
 * needs no host workspace.  A negative return other than -1 is an error
 * code (see simint_b200.h). */
int simint_compute_eri(struct simint_multi_shellpair const * P,
                       struct simint_multi_shellpair const * Q,
                       double screen_tol,
                       double * work,
                       double * integrals);

/* Replaces simint_compute_eri_deriv (skel/simint/simint_eri.h:39-44,
 * simint_eri.c:13-22, ostei.c:27-41).  deriv = 0 is simint_compute_eri;
 * deriv = 1 writes 12 gradient components per Cartesian quartet,
 * [Ax Ay Az Bx By Bz Cx Cy Cz Dx Dy Dz], innermost. */
int simint_compute_eri_deriv(int deriv,
                             struct simint_multi_shellpair const * P,
                             struct simint_multi_shellpair const * Q,
                             double screen_tol,
                             double * work,
                             double * integrals);

/* Replaces simint_eri_worksize / simint_eri_workmem
 * (skel/simint/simint_eri.h:53,62).  Same values as the reference
 * (computed from the same recurrence plan), so callers that size their
 * workspace with them keep working. */
size_t simint_eri_worksize(int derorder, int maxam);
size_t simint_eri_workmem(int derorder, int maxam);

#ifdef __cplusplus
}
#endif
