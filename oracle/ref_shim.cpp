/*
 * TEST INFRASTRUCTURE ONLY.  Glue that lets tests call the reference's own
 * long-double integral code (skel/test/ValeevRef.cpp, compiled from its
 * source by oracle/build_ref.py) through a plain C entry point.  Nothing
 * here is shipped or linked into libsimint_b200.so.
 *
 * ValeevRef.cpp needs two helpers that live in the reference's test harness
 * (skel/test/Common.cpp:14-33).  They are restated here: a Cartesian
 * exponent triple is valid when no exponent is negative, and the Psi4
 * iteration order steps (i,j,k) -> (i,j-1,k+1) while k < l-i, else
 * (i-1, l-i+1, 0), ending at (0,0,l).
 */
#include <array>
#include "test/ValeevRef.hpp"
#include "simint/shell/shell.h"

bool ValidGaussian(const std::array<int, 3> & g)
{
    return g[0] >= 0 && g[1] >= 0 && g[2] >= 0;
}

bool IterateGaussian(std::array<int, 3> & g)
{
    const int l = g[0] + g[1] + g[2];
    if(g[2] == l)
        return false;
    if(g[2] < l - g[0])
        g = {{g[0], g[1] - 1, g[2] + 1}};
    else
        g = {{g[0] - 1, l - g[0] + 1, 0}};
    return ValidGaussian(g);
}

extern "C" void ref_valeev_integrals(simint_shell const * A, int nA,
                                     simint_shell const * B, int nB,
                                     simint_shell const * C, int nC,
                                     simint_shell const * D, int nD,
                                     double * out, int deriv)
{
    static bool initialised = false;
    if(!initialised)
    {
        ValeevRef_Init();
        initialised = true;
    }
    ValeevRef_Integrals(A, nA, B, nB, C, nC, D, nD, out, deriv, false);
}
