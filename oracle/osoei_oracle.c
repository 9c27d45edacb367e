/*
 * CPU oracle for the one-electron integrals of the B200 Simint engine.
 *
 * TEST INFRASTRUCTURE ONLY.  A plain-C restatement of Simint's one-electron
 * integrals (overlap, kinetic energy, nuclear attraction over contracted
 * Cartesian shells), written from the reference's sources and loaded only by
 * tests/ as the checker.  The product never links or calls it.
 *
 * What it restates (reference paths relative to the simint-generator tree):
 *   - overlap       skel/simint/osoei/osoei_overlap.c:9-67 with the 1-D
 *                   Obara-Saika tables of osoei_terms.c:9-83
 *   - kinetic       skel/simint/osoei/osoei_ke.c:10-68, terms
 *                   osoei_terms.c:86-165 (T = Tx Sy Sz + Sx Ty Sz + Sx Sy Tz)
 *   - potential     skel/simint/osoei/osoei_potential.c:10-219: two-centre
 *                   Obara-Saika recursion over (a|b)^(m), base
 *                   (2 pi / p) exp(-mu AB^2) F_m(p PC^2), contracted with
 *                   -Z_C c_a c_b over every centre C
 *   - output order  the fixed lexicographic Cartesian order of
 *                   skel/simint/recur_lookup.c (x descending, then y), the
 *                   same for every ERI ordering option
 *
 * The recursion here is written over dense (a, b, m) tables indexed by level
 * offsets (one step direction per Cartesian: the first non-zero exponent);
 * the reference picks directions from its lookup table, which changes only
 * the rounding.
 */

#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "simint/shell/shell.h"

#ifdef ORACLE_LONG_DOUBLE
typedef long double real;
#define R_EXP expl
#define R_SQRT sqrtl
#else
typedef double real;
#define R_EXP exp
#define R_SQRT sqrt
#endif

#define NC1(l) ((((l) + 1) * ((l) + 2)) / 2)
#define OEI_MAXL 6                      /* per shell */
#define OEI_NLEV ((OEI_MAXL + 1) * (OEI_MAXL + 2) * (OEI_MAXL + 3) / 6)
#define PI_L 3.14159265358979323846264338327950288419716939937510582097494L

void oracle_boys(real x, int L, real * F);

static int oei_psi4(int i, int k, int l) { return ((l - i) * (l - i + 1)) / 2 + k; }
static int oei_lev(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
static int oei_g(const int g[3])
{
    const int l = g[0] + g[1] + g[2];
    return oei_lev(l) + oei_psi4(g[0], g[2], l);
}

static void oei_carts(int l, int (*out)[3])
{
    int n = 0;
    for(int i = l; i >= 0; i--)
        for(int j = l - i; j >= 0; j--)
        {
            out[n][0] = i; out[n][1] = j; out[n][2] = l - i - j;
            n++;
        }
}

/* 1-D overlap and kinetic tables S[d][i][j], T[d][i][j] of one primitive
 * pair, i <= la, j <= lb (osoei_terms.c:9-165) */
static void terms_1d(real a1, const double A[3], real a2, const double B[3], int la, int lb,
                     real S[3][OEI_MAXL + 1][OEI_MAXL + 1], real T[3][OEI_MAXL + 1][OEI_MAXL + 1])
{
    const real p = a1 + a2, oop = 1.0 / p, mu = a1 * a2 * oop, o2p = 0.5 * oop;
    for(int d = 0; d < 3; d++)
    {
        const real P = (a1 * A[d] + a2 * B[d]) * oop;
        const real PA = P - A[d], PB = P - B[d];
        const real AB = (real)A[d] - (real)B[d];
        S[d][0][0] = R_SQRT((real)PI_L * oop) * R_EXP(-mu * AB * AB);
        T[d][0][0] = S[d][0][0] * (a1 - 2.0 * a1 * a1 * (PA * PA + o2p));
        for(int i = 0; i <= la; i++)
            for(int j = 0; j <= lb; j++)
            {
                if(i == 0 && j == 0)
                    continue;
                if(j == 0)
                {
                    /* raise i */
                    real s = PA * S[d][i - 1][0];
                    real t = PA * T[d][i - 1][0];
                    if(i > 1)
                    {
                        s += (i - 1) * o2p * S[d][i - 2][0];
                    }
                    S[d][i][0] = s;
                    t += 2.0 * mu * s;
                    if(i > 1)
                        t += (i - 1) * o2p * T[d][i - 2][0] - a2 * oop * (i - 1) * S[d][i - 2][0];
                    T[d][i][0] = t;
                }
                else
                {
                    /* raise j */
                    real s = PB * S[d][i][j - 1];
                    real t = PB * T[d][i][j - 1];
                    if(i > 0)
                    {
                        s += i * o2p * S[d][i - 1][j - 1];
                        t += i * o2p * T[d][i - 1][j - 1];
                    }
                    if(j > 1)
                        s += (j - 1) * o2p * S[d][i][j - 2];
                    S[d][i][j] = s;
                    t += 2.0 * mu * s;
                    if(j > 1)
                        t += (j - 1) * o2p * T[d][i][j - 2] - a1 * oop * (j - 1) * S[d][i][j - 2];
                    T[d][i][j] = t;
                }
            }
    }
}

/* kind 0 overlap, 1 kinetic energy (osoei_overlap.c:36-64, osoei_ke.c:37-65) */
int oracle_oei_st(int kind, const struct simint_shell * A, const struct simint_shell * B, double * out)
{
    const int la = A->am, lb = B->am;
    if(la > OEI_MAXL || lb > OEI_MAXL)
        return -1;
    const int na = NC1(la), nb = NC1(lb);
    int ca[NC1(OEI_MAXL)][3], cb[NC1(OEI_MAXL)][3];
    oei_carts(la, ca);
    oei_carts(lb, cb);
    real acc[NC1(OEI_MAXL) * NC1(OEI_MAXL)];
    for(int k = 0; k < na * nb; k++)
        acc[k] = 0.0;
    const double Ax[3] = {A->x, A->y, A->z}, Bx[3] = {B->x, B->y, B->z};
    real S[3][OEI_MAXL + 1][OEI_MAXL + 1], T[3][OEI_MAXL + 1][OEI_MAXL + 1];
    for(int i = 0; i < A->nprim; i++)
        for(int j = 0; j < B->nprim; j++)
        {
            terms_1d(A->alpha[i], Ax, B->alpha[j], Bx, la, lb, S, T);
            const real c = (real)A->coef[i] * (real)B->coef[j];
            for(int u = 0; u < na; u++)
                for(int v = 0; v < nb; v++)
                {
                    const int x1 = ca[u][0], y1 = ca[u][1], z1 = ca[u][2];
                    const int x2 = cb[v][0], y2 = cb[v][1], z2 = cb[v][2];
                    real val;
                    if(kind == 0)
                        val = S[0][x1][x2] * S[1][y1][y2] * S[2][z1][z2];
                    else
                        val = T[0][x1][x2] * S[1][y1][y2] * S[2][z1][z2]
                            + S[0][x1][x2] * T[1][y1][y2] * S[2][z1][z2]
                            + S[0][x1][x2] * S[1][y1][y2] * T[2][z1][z2];
                    acc[u * nb + v] += c * val;
                }
        }
    for(int k = 0; k < na * nb; k++)
        out[k] = (double)acc[k];
    return 1;
}

/* nuclear attraction over ncenter point charges (osoei_potential.c:10-219) */
int oracle_oei_potential(int ncenter, const double * Z, const double * x, const double * y,
                         const double * z, const struct simint_shell * A,
                         const struct simint_shell * B, double * out)
{
    const int la = A->am, lb = B->am, L = la + lb;
    if(la > OEI_MAXL || lb > OEI_MAXL)
        return -1;
    const int na = NC1(la), nb = NC1(lb);
    const int nga = oei_lev(la + 1), ngb = oei_lev(lb + 1);
    /* W[(ga * ngb + gb) * (L + 1) + m] = (a|b)^(m) */
    real * W = (real *)malloc(sizeof(real) * (size_t)nga * ngb * (L + 1));
    real acc[NC1(OEI_MAXL) * NC1(OEI_MAXL)];
    for(int k = 0; k < na * nb; k++)
        acc[k] = 0.0;
    const double Ac[3] = {A->x, A->y, A->z}, Bc[3] = {B->x, B->y, B->z};
    real AB2 = 0.0;
    for(int d = 0; d < 3; d++)
        AB2 += ((real)Ac[d] - Bc[d]) * ((real)Ac[d] - Bc[d]);
    int cl[OEI_MAXL + 1][NC1(OEI_MAXL)][3];
    for(int l = 0; l <= (la > lb ? la : lb); l++)
        oei_carts(l, cl[l]);
    real F[2 * OEI_MAXL + 1];
#define WAT(ga, gb, m) W[((size_t)(ga) * ngb + (gb)) * (L + 1) + (m)]
    for(int c = 0; c < ncenter; c++)
        for(int i = 0; i < A->nprim; i++)
            for(int j = 0; j < B->nprim; j++)
            {
                const real a1 = A->alpha[i], a2 = B->alpha[j];
                const real p = a1 + a2, oop = 1.0 / p, mu = a1 * a2 * oop, o2p = 0.5 * oop;
                real PA[3], PB[3], PC[3], PC2 = 0.0;
                const double Cc[3] = {x[c], y[c], z[c]};
                for(int d = 0; d < 3; d++)
                {
                    const real P = (a1 * Ac[d] + a2 * Bc[d]) * oop;
                    PA[d] = P - Ac[d];
                    PB[d] = P - Bc[d];
                    PC[d] = P - Cc[d];
                    PC2 += PC[d] * PC[d];
                }
                oracle_boys(PC2 * p, L, F);
                const real base = 2.0 * (real)PI_L * oop * R_EXP(-mu * AB2);
                for(int m = 0; m <= L; m++)
                    WAT(0, 0, m) = base * F[m];
                /* (a|0)^(m), m <= L - |a| */
                for(int l = 1; l <= la; l++)
                    for(int t = 0; t < NC1(l); t++)
                    {
                        const int * g = cl[l][t];
                        const int d = g[0] ? 0 : (g[1] ? 1 : 2);
                        int g1[3] = {g[0], g[1], g[2]};
                        g1[d]--;
                        const int i1 = oei_g(g1);
                        int i2 = -1;
                        if(g1[d] > 0)
                        {
                            int g2[3] = {g1[0], g1[1], g1[2]};
                            g2[d]--;
                            i2 = oei_g(g2);
                        }
                        const int gi = oei_g(g);
                        for(int m = 0; m <= L - l; m++)
                        {
                            real v = PA[d] * WAT(i1, 0, m) - PC[d] * WAT(i1, 0, m + 1);
                            if(i2 >= 0)
                                v += g1[d] * o2p * (WAT(i2, 0, m) - WAT(i2, 0, m + 1));
                            WAT(gi, 0, m) = v;
                        }
                    }
                /* (a|b)^(m), m <= L - |a| - |b|: raise b */
                for(int lbb = 1; lbb <= lb; lbb++)
                    for(int lab = 0; lab <= la; lab++)
                        for(int tb = 0; tb < NC1(lbb); tb++)
                        {
                            const int * h = cl[lbb][tb];
                            const int d = h[0] ? 0 : (h[1] ? 1 : 2);
                            int h1[3] = {h[0], h[1], h[2]};
                            h1[d]--;
                            const int j1 = oei_g(h1);
                            int j2 = -1;
                            if(h1[d] > 0)
                            {
                                int h2[3] = {h1[0], h1[1], h1[2]};
                                h2[d]--;
                                j2 = oei_g(h2);
                            }
                            const int gj = oei_g(h);
                            for(int ta = 0; ta < NC1(lab); ta++)
                            {
                                const int * g = cl[lab][ta];
                                const int gi = oei_g(g);
                                int i1 = -1;
                                if(g[d] > 0)
                                {
                                    int g1[3] = {g[0], g[1], g[2]};
                                    g1[d]--;
                                    i1 = oei_g(g1);
                                }
                                for(int m = 0; m <= L - lab - lbb; m++)
                                {
                                    real v = PB[d] * WAT(gi, j1, m) - PC[d] * WAT(gi, j1, m + 1);
                                    if(i1 >= 0)
                                        v += g[d] * o2p * (WAT(i1, j1, m) - WAT(i1, j1, m + 1));
                                    if(j2 >= 0)
                                        v += h1[d] * o2p * (WAT(gi, j2, m) - WAT(gi, j2, m + 1));
                                    WAT(gi, gj, m) = v;
                                }
                            }
                        }
                const real f = -(real)Z[c] * (real)A->coef[i] * (real)B->coef[j];
                for(int u = 0; u < na; u++)
                    for(int v = 0; v < nb; v++)
                        acc[u * nb + v] += f * WAT(oei_lev(la) + u, oei_lev(lb) + v, 0);
            }
#undef WAT
    free(W);
    for(int k = 0; k < na * nb; k++)
        out[k] = (double)acc[k];
    return 1;
}
