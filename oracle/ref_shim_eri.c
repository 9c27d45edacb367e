/*
 * TEST INFRASTRUCTURE ONLY.  The reference's Schwarz screening
 * (skel/simint/shell/shell_screen.c:48-223) calls simint_compute_eri on
 * uncontracted shells.  Inside the reference-built test library that call is
 * answered by the CPU oracle (oracle/ostei_oracle.c); the diagonal maxima it
 * takes do not depend on the Cartesian ordering.
 */
#include "simint/shell/shell.h"

int oracle_compute_eri(struct simint_multi_shellpair const * P,
                       struct simint_multi_shellpair const * Q,
                       double screen_tol, int deriv, int ordering, double * out);

int simint_compute_eri(struct simint_multi_shellpair const * P,
                       struct simint_multi_shellpair const * Q,
                       double screen_tol, double * work, double * integrals)
{
    (void)work;
    return oracle_compute_eri(P, Q, screen_tol, 0, 0, integrals);
}
