/*
 * TEST INFRASTRUCTURE ONLY.  Exposes the reference's Boys function
 * (skel/simint/boys/boys.h:84-92, scalar build) and its tables, compiled from
 * the reference sources by oracle/build_ref.py, so tests can pin our Boys grid
 * and evaluation against it.
 */
#include "simint/boys/boys.h"
#include "simint/boys/boys_longfac.h"

void ref_boys_F(double x, int n, double * F)
{
    boys_F_split(F, x, n);
}

double ref_boys_grid(int i, int n)
{
    return boys_shortgrid[i][n];
}

double ref_boys_longfac(int n)
{
    return boys_longfac[n];
}
