/*
 * CPU oracle for the B200 Simint engine.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of Simint's
 * two-electron-integral algorithm, written from the reference's sources.  It
 * is loaded only by tests/, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg, always as the checker, never as the thing measured or
 * shipped.  The product (libsimint_b200.so) never links or calls it.
 *
 * What it restates (reference paths relative to the simint-generator tree):
 *   - pair precompute        skel/simint/shell/shell.c:425-582 (padding :538-570,
 *                            screen sort :37-128)
 *   - normalisation          skel/simint/shell/shell.c:248-278
 *   - screening values       skel/simint/shell/shell_screen.c:48-270
 *   - Boys function          skel/simint/boys/boys.h:14-92, boys_taylor.h:14-39,
 *                            boys_long.h:14-58
 *   - primitive set-up       generator/ostei/OSTEI_Writer.cpp:586-702
 *   - VRR (8-term step)      generator/ostei/Makowski.hpp:87-242,
 *                            OSTEI_VRR_Writer.cpp:33-130; centre order
 *                            OSTEI_VRR_Algorithm_Base.cpp:449-469
 *   - contraction            OSTEI_Writer.cpp:67-99 (deriv weights
 *                            OSTEIDeriv1_Writer.cpp:53-94)
 *   - HRR                    Makowski.hpp:17-82, OSTEI_HRR_Algorithm_Base.cpp:160-283,
 *                            OSTEI_HRR_Writer.cpp:22-101
 *   - deriv=1 formation      OSTEIDeriv1_Writer.cpp:334-537,
 *                            ostei_deriv1_generator.cpp:97-123
 *   - screening semantics    ostei.c:10-23, OSTEI_Writer.cpp:499-586: a bra
 *                            primitive is skipped when P.screen[i]*Q.screen_max
 *                            < tol^2, an 8-wide ket vector when its largest
 *                            P.screen[i]*Q.screen[j] < tol^2.
 *
 * It is deliberately generic and dense: every (e0|f0)^(m) of the class is
 * computed by the same per-element rule the reference's planner uses, so it
 * shares no code (and no generated plan) with the CUDA kernels.
 *
 * Two deliberate differences from the reference, both documented in the
 * product too: the bra primitive offsets follow the padded layout (the
 * reference's generated loop uses istart = iend, OSTEI_Writer.cpp:734, which
 * ignores the padding inserted after every 16 bra pairs); GAMESS-ordered
 * deriv=1 output is the Psi4 result permuted per centre (the reference indexes
 * it through the Psi4 table, OSTEIDeriv1_Writer.cpp:359-362).
 */

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

#include "simint/shell/shell.h"
#include "boys_grid.inc"

/* Arithmetic type of the integral evaluation (pair data, shells and
 * screening values stay double).  The oracle is built twice: double, and
 * with -DORACLE_LONG_DOUBLE long double -- the same algorithm evaluated with
 * 64-bit mantissas, which measures how far any double-precision evaluation
 * (this oracle's or the product's) is from the exact values on elements that
 * the recurrences compute with cancellation. */
#ifdef ORACLE_LONG_DOUBLE
typedef long double real;
#define R_EXP expl
#define R_SQRT sqrtl
#define R_POW powl
#define R_FMA fmal
#else
typedef double real;
#define R_EXP exp
#define R_SQRT sqrt
#define R_POW pow
#define R_FMA fma
#endif

#define NC(l) ((l) >= 0 ? (((l) + 1) * ((l) + 2)) / 2 : 0)
#define MAXLEV 24                       /* largest AM level handled */
#define SQRT_TWO_PI_52 5.91496717279561287782347843505365022963403204272156069835237
#define SQRT_TWO_TIMES_PI_52 24.739429451193148050228357586821944304008810699990039583

static const double norm_fac_tab[9] = {
    /* pi^(3/2) (2l-1)!! / 2^l, l = 0..8 (shell_constants.c:13-36) */
    5.568327996831707845, 2.784163998415853922, 4.176245997623780883,
    10.44061499405945221, 36.54215247920808273, 164.4396861564363723,
    904.4182738604000480, 5878.718780092600312, 44090.39085069450234
};

/* ------------------------------------------------------------------ */
/* Cartesian bookkeeping                                               */
/* ------------------------------------------------------------------ */

static int psi4_index(int i, int j, int k)
{
    int l = i + j + k;
    (void)j;
    return ((l - i) * (l - i + 1)) / 2 + k;
}

static const int gamess2[6][3] = {{2,0,0},{0,2,0},{0,0,2},{1,1,0},{1,0,1},{0,1,1}};
static const int gamess3[10][3] = {{3,0,0},{0,3,0},{0,0,3},{2,1,0},{2,0,1},
                                   {1,2,0},{0,2,1},{1,0,2},{0,1,2},{1,1,1}};

static int cart_index(const int g[3], int ordering)
{
    int l = g[0] + g[1] + g[2];
    if(ordering == 1 && (l == 2 || l == 3))
    {
        int n = NC(l);
        for(int t = 0; t < n; t++)
        {
            const int * h = (l == 2) ? gamess2[t] : gamess3[t];
            if(h[0] == g[0] && h[1] == g[1] && h[2] == g[2])
                return t;
        }
    }
    return psi4_index(g[0], g[1], g[2]);
}

/* flat index over all levels 0..l: offset of level l plus Psi4 position */
static int lev_off(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
static int gidx(const int g[3]) { return lev_off(g[0] + g[1] + g[2]) + psi4_index(g[0], g[1], g[2]); }

/* cart list of level l in Psi4 order */
static void level_carts(int l, int (*out)[3])
{
    int n = 0;
    for(int i = l; i >= 0; i--)
        for(int j = l - i; j >= 0; j--)
        {
            out[n][0] = i; out[n][1] = j; out[n][2] = l - i - j;
            n++;
        }
}

static int stepdir(const int g[3])
{
    int m = 1000;
    for(int t = 0; t < 3; t++)
        if(g[t] > 0 && g[t] < m) m = g[t];
    for(int t = 2; t >= 0; t--)
        if(g[t] == m) return t;
    return -1;
}

/* ------------------------------------------------------------------ */
/* Boys function                                                       */
/* ------------------------------------------------------------------ */

static real taylor_single(real x, int n)
{
    const int idx = (int)(10.0 * (x + 0.05));
    const real xi = (real)idx * 0.1;
    const real dx = xi - x;
    const double * g = &simint_b200_boys_grid_host[idx][n];
    return g[0] + dx * (g[1] + dx * ((1.0/2.0) * g[2] + dx * ((1.0/6.0) * g[3]
           + dx * ((1.0/24.0) * g[4] + dx * ((1.0/120.0) * g[5]
           + dx * ((1.0/720.0) * g[6] + dx * ((1.0/5040.0) * g[7])))))));
}

void oracle_boys(real x, int L, real * F)
{
    if(L < 4)
    {
        if(x < SIMINT_B200_BOYS_MAXX)
        {
            for(int n = 0; n <= L; n++)
                F[n] = taylor_single(x, n);
        }
        else
        {
            const real x1 = 1.0 / x;
            real x2 = R_SQRT(x1);
            for(int n = 0; n <= L; n++)
            {
                F[n] = simint_b200_boys_longfac_host[n] * x2;
                x2 *= x1;
            }
        }
        return;
    }
    if(x < SIMINT_B200_BOYS_MAXX)
        F[L] = taylor_single(x, L);
    else
        F[L] = simint_b200_boys_longfac_host[L] * R_POW(x, -((real)L + 0.5));
    const real x2 = 2.0 * x;
    const real ex = R_EXP(-x);
    for(int n = L - 1; n >= 0; n--)
        F[n] = (1.0 / (2.0 * n + 1)) * R_FMA(x2, F[n + 1], ex);
}

/* ------------------------------------------------------------------ */
/* Shells and pairs                                                    */
/* ------------------------------------------------------------------ */

void oracle_normalize_shells(int n, struct simint_shell * G)
{
    for(int s = 0; s < n; ++s)
    {
        const double am = (double)G[s].am;
        const double m = am + 1.5;
        const double m2 = 0.5 * m;
        double sum = 0.0;
        for(int j = 0; j < G[s].nprim; j++)
            for(int k = 0; k < G[s].nprim; k++)
            {
                const double a1 = G[s].alpha[j], c1 = G[s].coef[j];
                const double a2 = G[s].alpha[k], c2 = G[s].coef[k];
                sum += (c1 * c2 * pow(a1 * a2, m2)) / (pow(a1 + a2, m));
            }
        const double norm = 1.0 / sqrt(sum * norm_fac_tab[G[s].am]);
        for(int j = 0; j < G[s].nprim; ++j)
            G[s].coef[j] *= norm * pow(G[s].alpha[j], m2);
    }
}

static int same_shell(const struct simint_shell * A, const struct simint_shell * B)
{
    return A->nprim == B->nprim && A->ptr == B->ptr;
}

static int round8(int x) { return (x + 7) & ~7; }

int oracle_compute_eri(struct simint_multi_shellpair const * P,
                       struct simint_multi_shellpair const * Q,
                       double screen_tol, int deriv, int ordering, real * out);

static double prim_schwarz_one(const struct simint_shell * A, int i,
                               const struct simint_shell * B, int j);

/* number of padded primitive slots of a pair list (shell.c:356-382) */
static int padded_nprim(int npair, const struct simint_shell * AB)
{
    int nprim = 0, batch = 0;
    for(int p = 0; p < npair; p++)
    {
        const struct simint_shell * A = &AB[2 * p];
        const struct simint_shell * B = &AB[2 * p + 1];
        batch += same_shell(A, B) ? (A->nprim * (A->nprim + 1)) / 2 : A->nprim * B->nprim;
        if(((p + 1) % 16) == 0 || p + 1 >= npair)
        {
            nprim += round8(batch);
            batch = 0;
        }
    }
    return nprim;
}

static void sort_prims(struct simint_multi_shellpair * P, int lo, int hi)
{
    /* descending by screen value within one shell pair (shell.c:37-128 use a
     * quicksort; any order with descending screen values gives the same
     * set of primitives, only the summation order changes) */
    for(int a = lo + 1; a <= hi; a++)
    {
        int b = a;
        while(b > lo && P->screen[b - 1] < P->screen[b])
        {
#define SW(arr) { double t_ = P->arr[b - 1]; P->arr[b - 1] = P->arr[b]; P->arr[b] = t_; }
            SW(x) SW(y) SW(z) SW(PA_x) SW(PA_y) SW(PA_z) SW(PB_x) SW(PB_y) SW(PB_z)
            SW(alpha) SW(prefac) SW(screen) SW(alpha2) SW(beta2)
#undef SW
            b--;
        }
    }
}

void oracle_create_pair(int npair, const struct simint_shell * AB,
                        struct simint_multi_shellpair * P, int screen_method)
{
    const int nprim = padded_nprim(npair, AB);
    const int narr = 11 + (screen_method ? 1 : 0) + 2;
    const size_t memsize = (size_t)nprim * narr * sizeof(double)
                         + 3 * (size_t)npair * sizeof(double) + (size_t)npair * sizeof(int);
    char * mem = (char *)calloc(1, memsize + 64);
    P->ptr = mem;
    P->memsize = memsize;
    double * d = (double *)mem;
    double ** arrs[14] = {&P->x, &P->y, &P->z, &P->PA_x, &P->PA_y, &P->PA_z,
                          &P->PB_x, &P->PB_y, &P->PB_z, &P->alpha, &P->prefac,
                          &P->screen, &P->alpha2, &P->beta2};
    int c = 0;
    for(int t = 0; t < 14; t++)
    {
        if(t == 11 && !screen_method) { P->screen = NULL; continue; }
        *arrs[t] = d + (size_t)nprim * c++;
    }
    P->AB_x = d + (size_t)nprim * c;
    P->AB_y = P->AB_x + npair;
    P->AB_z = P->AB_y + npair;
    P->nprim12 = (int *)(P->AB_z + npair);

    P->nshell12 = npair;
    P->nshell12_clip = npair;
    P->nprim = 0;
    P->screen_max = 1.e99;   /* shell.c:434, only ever raised */
    int idx = 0;
    for(int p = 0; p < npair; p++)
    {
        const struct simint_shell * A = &AB[2 * p];
        const struct simint_shell * B = &AB[2 * p + 1];
        const int same = same_shell(A, B);
        const int start = idx;
        P->am1 = A->am;
        P->am2 = B->am;
        if(screen_method)
        {
            double mx = 0.0;
            int sidx = idx;
            for(int i = 0; i < A->nprim; i++)
                for(int j = 0; j < (same ? i + 1 : B->nprim); j++)
                {
                    double v;
                    if(screen_method == SIMINT_SCREEN_FASTSCHWARZ)
                    {
                        const double a = A->alpha[i], b = B->alpha[j];
                        const double pp = a + b, oop = 1.0 / pp, rho = (a * b) / pp;
                        const double Rx = A->x - B->x, Ry = A->y - B->y, Rz = A->z - B->z;
                        const double R2 = Rx * Rx + Ry * Ry + Rz * Rz;
                        v = SQRT_TWO_TIMES_PI_52 * pow(oop, 2.5) * exp(-2.0 * rho * R2);
                        v *= A->coef[i] * A->coef[i] * B->coef[j] * B->coef[j];
                    }
                    else
                        v = prim_schwarz_one(A, i, B, j);
                    P->screen[sidx++] = v;
                    if(v > mx) mx = v;
                }
            if(mx > P->screen_max) P->screen_max = mx;
        }
        const double Xab_x = A->x - B->x, Xab_y = A->y - B->y, Xab_z = A->z - B->z;
        const double Xab = Xab_x * Xab_x + Xab_y * Xab_y + Xab_z * Xab_z;
        for(int i = 0; i < A->nprim; ++i)
        {
            const double ai = A->alpha[i];
            const double AxAa = A->x * ai, AyAa = A->y * ai, AzAa = A->z * ai;
            const int jend = same ? i + 1 : B->nprim;
            for(int j = 0; j < jend; ++j)
            {
                const double aj = B->alpha[j];
                const double s = ai + aj, mu = ai * aj;
                P->prefac[idx] = A->coef[i] * B->coef[j] * exp(-Xab * mu / s) * SQRT_TWO_PI_52 / s;
                if(same && i != j) P->prefac[idx] *= 2.0;
                P->x[idx] = (AxAa + aj * B->x) / s;
                P->y[idx] = (AyAa + aj * B->y) / s;
                P->z[idx] = (AzAa + aj * B->z) / s;
                P->PA_x[idx] = P->x[idx] - A->x;
                P->PA_y[idx] = P->y[idx] - A->y;
                P->PA_z[idx] = P->z[idx] - A->z;
                P->PB_x[idx] = P->x[idx] - B->x;
                P->PB_y[idx] = P->y[idx] - B->y;
                P->PB_z[idx] = P->z[idx] - B->z;
                P->alpha[idx] = s;
                if(same && i != j) { P->alpha2[idx] = s; P->beta2[idx] = s; }
                else { P->alpha2[idx] = 2.0 * ai; P->beta2[idx] = 2.0 * aj; }
                ++idx;
            }
        }
        const int np = same ? (A->nprim * (A->nprim + 1)) / 2 : A->nprim * B->nprim;
        P->AB_x[p] = Xab_x; P->AB_y[p] = Xab_y; P->AB_z[p] = Xab_z;
        if(((p + 1) % 16) == 0 || p + 1 >= npair)
            while(idx < round8(idx))
            {
                P->alpha[idx] = 1.0; P->prefac[idx] = 0.0;
                P->x[idx] = P->y[idx] = P->z[idx] = 0.0;
                P->PA_x[idx] = P->PA_y[idx] = P->PA_z[idx] = 0.0;
                P->PB_x[idx] = P->PB_y[idx] = P->PB_z[idx] = 0.0;
                if(P->screen) P->screen[idx] = 0.0;
                P->alpha2[idx] = 1.0; P->beta2[idx] = 1.0;
                idx++;
            }
        P->nprim12[p] = np;
        P->nprim += np;
        if(screen_method)
            sort_prims(P, start, start + np - 1);
    }
}

void oracle_free_pair(struct simint_multi_shellpair * P)
{
    free(P->ptr);
    P->ptr = NULL;
    P->memsize = 0;
}

/* Schwarz value of one primitive pair: max over diagonal Cartesians of
 * |(ab|ab)| for the uncontracted shells (shell_screen.c:127-223). */
static double prim_schwarz_one(const struct simint_shell * A, int i,
                               const struct simint_shell * B, int j)
{
    struct simint_shell sh[2];
    sh[0] = *A; sh[1] = *B;
    sh[0].nprim = 1; sh[0].alpha = A->alpha + i; sh[0].coef = A->coef + i; sh[0].ptr = (void *)1;
    sh[1].nprim = 1; sh[1].alpha = B->alpha + j; sh[1].coef = B->coef + j; sh[1].ptr = (void *)2;
    struct simint_multi_shellpair P;
    oracle_create_pair(1, sh, &P, 0);
    const int n1 = NC(A->am), n2 = NC(B->am), n12 = n1 * n2;
    real * ints = (real *)malloc(sizeof(real) * n12 * n12);
    oracle_compute_eri(&P, &P, 0.0, 0, 0, ints);
    double mx = 0.0;
    for(int m = 0; m < n1; m++)
        for(int n = 0; n < n2; n++)
        {
            const double v = fabs((double)ints[m * n2 * n1 * n2 + m * n2 + n * n1 * n2 + n]);
            if(v > mx) mx = v;
        }
    free(ints);
    oracle_free_pair(&P);
    return mx;
}

double oracle_shellscreen_schwarz(const struct simint_shell * A, const struct simint_shell * B)
{
    struct simint_shell sh[2] = {*A, *B};
    struct simint_multi_shellpair P;
    oracle_create_pair(1, sh, &P, 0);
    const int n12 = NC(A->am) * NC(B->am);
    real * ints = (real *)malloc(sizeof(real) * n12 * n12);
    oracle_compute_eri(&P, &P, 0.0, 0, 0, ints);
    double mx = 0.0;
    for(int n = 0; n < n12 * n12; n++)
        if(fabs((double)ints[n]) > mx) mx = fabs((double)ints[n]);
    free(ints);
    oracle_free_pair(&P);
    return mx;
}

/* ------------------------------------------------------------------ */
/* Class set-up                                                        */
/* ------------------------------------------------------------------ */

typedef struct
{
    int am[4];
    int deriv;
    int missing;                 /* deriv=1: centre recovered by invariance */
    int ntarget;
    int tgt[8][4];               /* target AMs */
    int tgt_tag[8];              /* 0 untagged, 1..4 = 2a,2b,2c,2d */
    int brastep_j;               /* 1: bra moves I->J (tops (e,0)); 0: J->I */
    int ketstep_l;               /* 1: ket moves K->L (tops (f,0)); 0: L->K */
    int Emax, Fmax, L;
    int ket_first;               /* VRR reduces the ket centre first */
} ClassInfo;

static void class_setup(const int am[4], int deriv, ClassInfo * ci)
{
    memset(ci, 0, sizeof(*ci));
    memcpy(ci->am, am, sizeof(ci->am));
    ci->deriv = deriv;
    if(deriv == 0)
    {
        ci->ntarget = 1;
        memcpy(ci->tgt[0], am, sizeof(ci->am));
        ci->tgt_tag[0] = 0;
        ci->missing = -1;
    }
    else
    {
        int mx = am[0];
        for(int c = 1; c < 4; c++) if(am[c] > mx) mx = am[c];
        ci->missing = 0;
        while(am[ci->missing] != mx) ci->missing++;
        for(int c = 0; c < 4; c++)
        {
            if(c == ci->missing) continue;
            memcpy(ci->tgt[ci->ntarget], am, sizeof(ci->am));
            ci->tgt[ci->ntarget][c]++;
            ci->tgt_tag[ci->ntarget++] = c + 1;
            if(am[c] > 0)
            {
                memcpy(ci->tgt[ci->ntarget], am, sizeof(ci->am));
                ci->tgt[ci->ntarget][c]--;
                ci->tgt_tag[ci->ntarget++] = 0;
            }
        }
    }
    /* HRR directions from the lexicographically largest target
     * (OSTEI_HRR_Algorithm_Base.cpp:160-172) */
    int hi = 0;
    for(int t = 1; t < ci->ntarget; t++)
    {
        int cmp = 0;
        for(int c = 0; c < 4 && cmp == 0; c++)
            cmp = (ci->tgt[t][c] > ci->tgt[hi][c]) - (ci->tgt[t][c] < ci->tgt[hi][c]);
        if(cmp > 0) hi = t;
    }
    ci->brastep_j = ci->tgt[hi][0] >= ci->tgt[hi][1];
    ci->ketstep_l = ci->tgt[hi][2] >= ci->tgt[hi][3];
    ci->Emax = ci->Fmax = 0;
    for(int t = 0; t < ci->ntarget; t++)
    {
        const int e = ci->tgt[t][0] + ci->tgt[t][1];
        const int f = ci->tgt[t][2] + ci->tgt[t][3];
        if(e > ci->Emax) ci->Emax = e;
        if(f > ci->Fmax) ci->Fmax = f;
    }
    ci->L = ci->Emax + ci->Fmax;
    /* VRR centre order (OSTEI_VRR_Algorithm_Base.cpp:449-469): the ket centre
     * is reduced first unless it carries more AM than the bra centre. */
    ci->ket_first = ci->Fmax <= ci->Emax;
}

/* ------------------------------------------------------------------ */
/* Per primitive quartet: Boys + dense VRR                             */
/* ------------------------------------------------------------------ */

typedef struct
{
    real XP[3];      /* PA or PB, for the bra top centre */
    real XQ[3];      /* QC or QD, for the ket top centre */
    real aop_PQ[3], aoq_PQ[3];
    real a_over_p, a_over_q;         /* both negative, as in the reference */
    real one_over_2p, one_over_2q, one_over_2pq;
} PrimFactors;

/* V[(gE * nF + gF) * (L+1) + m] */
static void dense_vrr(const ClassInfo * ci, const PrimFactors * f, const real * F,
                      real * V, int nE, int nF)
{
    const int L = ci->L;
    const int LP = L + 1;
    int ce[MAXLEV * MAXLEV][3];
    int cf[MAXLEV * MAXLEV][3];
#define VV(ge, gf, m) V[((size_t)(ge) * nF + (gf)) * LP + (m)]
    VV(0, 0, 0) = F[0];
    for(int m = 0; m <= L; m++) VV(0, 0, m) = F[m];
    for(int el = 0; el <= ci->Emax; el++)
    {
        level_carts(el, ce);
        for(int fl = 0; fl <= ci->Fmax; fl++)
        {
            if(el == 0 && fl == 0) continue;
            level_carts(fl, cf);
            const int mmax = L - el - fl;
            for(int a = 0; a < NC(el); a++)
                for(int b = 0; b < NC(fl); b++)
                {
                    const int * ge = ce[a];
                    const int * gf = cf[b];
                    const int use_ket = (fl > 0) && (ci->ket_first || el == 0);
                    const int gE = gidx(ge), gF = gidx(gf);
                    if(use_ket)
                    {
                        const int x = stepdir(gf);
                        int f1[3] = {gf[0], gf[1], gf[2]}; f1[x]--;
                        int f2[3] = {gf[0], gf[1], gf[2]}; f2[x] -= 2;
                        int e1[3] = {ge[0], ge[1], ge[2]}; e1[x]--;
                        const int gF1 = gidx(f1);
                        const int have2 = f2[x] >= 0;
                        const int have6 = e1[x] >= 0;
                        const int gF2 = have2 ? gidx(f2) : 0;
                        const int gE1 = have6 ? gidx(e1) : 0;
                        const real c0 = (gf[x] - 1) == 1 ? f->one_over_2q : (real)(gf[x] - 1) * f->one_over_2q;
                        const real c2 = ge[x] == 1 ? f->one_over_2pq : (real)ge[x] * f->one_over_2pq;
                        for(int m = 0; m <= mmax; m++)
                        {
                            real t = f->XQ[x] * VV(gE, gF1, m);
                            t = R_FMA(f->aoq_PQ[x], VV(gE, gF1, m + 1), t);
                            if(have2)
                                t = R_FMA(c0, R_FMA(f->a_over_q, VV(gE, gF2, m + 1), VV(gE, gF2, m)), t);
                            if(have6)
                                t = R_FMA(c2, VV(gE1, gF1, m + 1), t);
                            VV(gE, gF, m) = t;
                        }
                    }
                    else
                    {
                        const int x = stepdir(ge);
                        int e1[3] = {ge[0], ge[1], ge[2]}; e1[x]--;
                        int e2[3] = {ge[0], ge[1], ge[2]}; e2[x] -= 2;
                        int f1[3] = {gf[0], gf[1], gf[2]}; f1[x]--;
                        const int gE1 = gidx(e1);
                        const int have2 = e2[x] >= 0;
                        const int have6 = f1[x] >= 0;
                        const int gE2 = have2 ? gidx(e2) : 0;
                        const int gF1 = have6 ? gidx(f1) : 0;
                        const real c0 = (ge[x] - 1) == 1 ? f->one_over_2p : (real)(ge[x] - 1) * f->one_over_2p;
                        const real c2 = gf[x] == 1 ? f->one_over_2pq : (real)gf[x] * f->one_over_2pq;
                        for(int m = 0; m <= mmax; m++)
                        {
                            real t = f->XP[x] * VV(gE1, gF, m);
                            t = R_FMA(f->aop_PQ[x], VV(gE1, gF, m + 1), t);
                            if(have2)
                                t = R_FMA(c0, R_FMA(f->a_over_p, VV(gE2, gF, m + 1), VV(gE2, gF, m)), t);
                            if(have6)
                                t = R_FMA(c2, VV(gE1, gF1, m + 1), t);
                            VV(gE, gF, m) = t;
                        }
                    }
                }
        }
    }
#undef VV
}

/* ------------------------------------------------------------------ */
/* HRR (one side)                                                      */
/* ------------------------------------------------------------------ */

/* top[gTop * ncol + col] holds the doublets with all AM on the top centre
 * (levels up to ta+tb).  right_step: 1 for I->J / K->L (tops (e,0), step on
 * the right function), 0 for J->I / L->K (tops (0,e), step on the left).
 * out[(psi4(A)*NC(tb) + psi4(B)) * ncol + col]. */
static void hrr_side(int right_step, int ta, int tb, const real X[3],
                     const real * top, int ncol, real * out)
{
    const int lt = ta + tb;
    const int nall = lev_off(lt + 1);
    const int nstep = right_step ? lev_off(tb + 1) : lev_off(ta + 1);
    real * H = (real *)malloc(sizeof(real) * (size_t)nall * nstep * ncol);
    int cs[MAXLEV * MAXLEV][3], co[MAXLEV * MAXLEV][3];
#define HH(gt, gs, c) H[((size_t)(gt) * nstep + (gs)) * ncol + (c)]
    /* H(gt, gs): gt indexes the function on the top centre, gs the one that
     * is stepped (B for right_step, A otherwise). */
    const int lo = right_step ? ta : tb;
    for(int l = lo; l <= lt; l++)
        for(int g = lev_off(l); g < lev_off(l + 1); g++)
            for(int c = 0; c < ncol; c++)
                HH(g, 0, c) = top[(size_t)g * ncol + c];
    const int sl_max = right_step ? tb : ta;
    for(int sl = 1; sl <= sl_max; sl++)
    {
        level_carts(sl, cs);
        for(int tl = lo; tl <= lt - sl; tl++)
        {
            level_carts(tl, co);
            for(int a = 0; a < NC(tl); a++)
                for(int b = 0; b < NC(sl); b++)
                {
                    const int * gt = co[a];
                    const int * gs = cs[b];
                    const int x = stepdir(gs);
                    int gsm[3] = {gs[0], gs[1], gs[2]}; gsm[x]--;
                    int gtp[3] = {gt[0], gt[1], gt[2]}; gtp[x]++;
                    const int it = gidx(gt), is = gidx(gs);
                    const int ism = gidx(gsm), itp = gidx(gtp);
                    for(int c = 0; c < ncol; c++)
                    {
                        if(right_step)   /* (a,b) = (a+1x, b-1x) + X (a, b-1x) */
                            HH(it, is, c) = R_FMA(X[x], HH(it, ism, c), HH(itp, ism, c));
                        else             /* (a,b) = (a-1x, b+1x) - X (a-1x, b) */
                            HH(it, is, c) = R_FMA(-X[x], HH(it, ism, c), HH(itp, ism, c));
                    }
                }
        }
    }
    /* gather the target block */
    int cA[MAXLEV * MAXLEV][3], cB[MAXLEV * MAXLEV][3];
    level_carts(ta, cA);
    level_carts(tb, cB);
    for(int a = 0; a < NC(ta); a++)
        for(int b = 0; b < NC(tb); b++)
        {
            const int it = right_step ? gidx(cA[a]) : gidx(cB[b]);
            const int is = right_step ? gidx(cB[b]) : gidx(cA[a]);
            for(int c = 0; c < ncol; c++)
                out[((size_t)a * NC(tb) + b) * ncol + c] = HH(it, is, c);
        }
#undef HH
    free(H);
}

/* full HRR: Acc[gE * nF + gF] -> target (ta tb | tc td), Psi4 order */
static void hrr_full(const ClassInfo * ci, const int t[4], const real AB[3], const real CD[3],
                     const real * Acc, int nE, int nF, real * out)
{
    const int fl_lo = ci->ketstep_l ? t[2] : t[3];
    const int fl_hi = t[2] + t[3];
    const int ncolF = lev_off(fl_hi + 1);
    (void)fl_lo;
    /* bra HRR for every ket column gF < ncolF */
    const int nbra = NC(t[0]) * NC(t[1]);
    real * top = (real *)malloc(sizeof(real) * (size_t)nE * ncolF);
    for(int e = 0; e < nE; e++)
        for(int f = 0; f < ncolF; f++)
            top[(size_t)e * ncolF + f] = Acc[(size_t)e * nF + f];
    real * bra = (real *)malloc(sizeof(real) * (size_t)nbra * ncolF);
    hrr_side(ci->brastep_j, t[0], t[1], AB, top, ncolF, bra);
    /* ket HRR: columns are the bra Cartesians */
    real * top2 = (real *)malloc(sizeof(real) * (size_t)ncolF * nbra);
    for(int f = 0; f < ncolF; f++)
        for(int b = 0; b < nbra; b++)
            top2[(size_t)f * nbra + b] = bra[(size_t)b * ncolF + f];
    const int nket = NC(t[2]) * NC(t[3]);
    real * ket = (real *)malloc(sizeof(real) * (size_t)nket * nbra);
    hrr_side(ci->ketstep_l, t[2], t[3], CD, top2, nbra, ket);
    for(int b = 0; b < nbra; b++)
        for(int k = 0; k < nket; k++)
            out[(size_t)b * nket + k] = ket[(size_t)k * nbra + b];
    free(top); free(bra); free(top2); free(ket);
}

/* ------------------------------------------------------------------ */
/* The ERI driver                                                      */
/* ------------------------------------------------------------------ */

static void pair_offsets(const struct simint_multi_shellpair * P, int * start)
{
    int idx = 0;
    for(int p = 0; p < P->nshell12; p++)
    {
        start[p] = idx;
        idx += P->nprim12[p];
        if(((p + 1) % 16) == 0 || p + 1 >= P->nshell12)
            idx = round8(idx);
    }
}

int oracle_compute_eri(struct simint_multi_shellpair const * P,
                       struct simint_multi_shellpair const * Q,
                       double screen_tol, int deriv, int ordering, real * out)
{
    const double tol2 = screen_tol * screen_tol;
    if(screen_tol > 0.0 && P->screen_max * Q->screen_max < tol2)
        return -1;
    const int check = (screen_tol > 0.0) && P->screen && Q->screen;
    const int am[4] = {P->am1, P->am2, Q->am1, Q->am2};
    ClassInfo ci;
    class_setup(am, deriv, &ci);
    const int nE = lev_off(ci.Emax + 1), nF = lev_off(ci.Fmax + 1);
    const int LP = ci.L + 1;
    real * V = (real *)malloc(sizeof(real) * (size_t)nE * nF * LP);
    real * Acc = (real *)malloc(sizeof(real) * 5 * (size_t)nE * nF);
    const int ncart = NC(am[0]) * NC(am[1]) * NC(am[2]) * NC(am[3]);
    const int nout = ncart * (deriv ? 12 : 1);
    real * tmp = (real *)malloc(sizeof(real) * 8 * (size_t)lev_off(ci.Emax + 2) * lev_off(ci.Fmax + 2));
    real * res[8];
    for(int t = 0; t < ci.ntarget; t++)
    {
        const int n = NC(ci.tgt[t][0]) * NC(ci.tgt[t][1]) * NC(ci.tgt[t][2]) * NC(ci.tgt[t][3]);
        res[t] = (real *)malloc(sizeof(real) * (size_t)n);
    }
    int * pst = (int *)malloc(sizeof(int) * (P->nshell12 + 1));
    int * qst = (int *)malloc(sizeof(int) * (Q->nshell12 + 1));
    pair_offsets(P, pst);
    pair_offsets(Q, qst);
    real F[64];
    const int bra_on_A = ci.brastep_j, ket_on_C = ci.ketstep_l;

    /* The reference's (ss|ss) kernel zeroes the screening values past the
     * last ket primitive before testing a partial vector
     * (skel/ostei_s_s_s_s.c): with a clipped ket list its vector test ends
     * at the clip. */
    int qclip_end = 0x7fffffff;
    if(!P->am1 && !P->am2 && !Q->am1 && !Q->am2 && Q->nshell12_clip < Q->nshell12 && Q->nshell12_clip > 0)
        qclip_end = qst[Q->nshell12_clip - 1] + Q->nprim12[Q->nshell12_clip - 1];
    for(int ab = 0; ab < P->nshell12_clip; ab++)
    for(int cd = 0; cd < Q->nshell12_clip; cd++)
    {
        memset(Acc, 0, sizeof(real) * 5 * (size_t)nE * nF);
        for(int i = pst[ab]; i < pst[ab] + P->nprim12[ab]; i++)
        {
            if(check && P->screen[i] * Q->screen_max < tol2)
                continue;
            for(int j = qst[cd]; j < qst[cd] + Q->nprim12[cd]; j++)
            {
                if(check)
                {
                    /* 8-wide vector test: [8*(j/8), 8*(j/8)+8) of the padded ket */
                    const int v0 = j & ~7;
                    double vmax = 0.0;
                    for(int jj = v0; jj < v0 + 8 && jj < qclip_end; jj++)
                    {
                        const double s = P->screen[i] * Q->screen[jj];
                        if(s > vmax) vmax = s;
                    }
                    if(vmax < tol2) continue;
                }
                const real pa = P->alpha[i], qa = Q->alpha[j];
                const real one_over_sum = 1.0 / (pa + qa);
                const real PQ[3] = {P->x[i] - Q->x[j], P->y[i] - Q->y[j], P->z[i] - Q->z[j]};
                real R2 = PQ[0] * PQ[0];
                R2 = R_FMA(PQ[1], PQ[1], R2);
                R2 = R_FMA(PQ[2], PQ[2], R2);
                const real alpha = (pa * qa) * one_over_sum;
                PrimFactors f;
                const real one_over_p = 1.0 / pa, one_over_q = 1.0 / qa;
                f.one_over_2p = 0.5 * one_over_p;
                f.one_over_2q = 0.5 * one_over_q;
                f.one_over_2pq = 0.5 * one_over_sum;
                f.a_over_p = -alpha * one_over_p;
                const real aoq = alpha * one_over_q;
                f.a_over_q = -aoq;
                for(int k = 0; k < 3; k++)
                {
                    f.aop_PQ[k] = f.a_over_p * PQ[k];
                    f.aoq_PQ[k] = aoq * PQ[k];
                }
                if(bra_on_A) { f.XP[0] = P->PA_x[i]; f.XP[1] = P->PA_y[i]; f.XP[2] = P->PA_z[i]; }
                else         { f.XP[0] = P->PB_x[i]; f.XP[1] = P->PB_y[i]; f.XP[2] = P->PB_z[i]; }
                if(ket_on_C) { f.XQ[0] = Q->PA_x[j]; f.XQ[1] = Q->PA_y[j]; f.XQ[2] = Q->PA_z[j]; }
                else         { f.XQ[0] = Q->PB_x[j]; f.XQ[1] = Q->PB_y[j]; f.XQ[2] = Q->PB_z[j]; }
                oracle_boys(R2 * alpha, ci.L, F);
                real prefac = R_SQRT(one_over_sum);
                prefac = (P->prefac[i] * Q->prefac[j]) * prefac;
                for(int n = 0; n <= ci.L; n++) F[n] *= prefac;
                dense_vrr(&ci, &f, F, V, nE, nF);
                const real w[5] = {1.0, P->alpha2[i], P->beta2[i], Q->alpha2[j], Q->beta2[j]};
                for(int tg = 0; tg < (deriv ? 5 : 1); tg++)
                {
                    real * A = Acc + (size_t)tg * nE * nF;
                    for(int e = 0; e < nE; e++)
                        for(int g = 0; g < nF; g++)
                            A[(size_t)e * nF + g] += (tg == 0) ? V[((size_t)e * nF + g) * LP]
                                                               : V[((size_t)e * nF + g) * LP] * w[tg];
                }
            }
        }
        const real AB[3] = {P->AB_x[ab], P->AB_y[ab], P->AB_z[ab]};
        const real CD[3] = {Q->AB_x[cd], Q->AB_y[cd], Q->AB_z[cd]};
        for(int t = 0; t < ci.ntarget; t++)
            hrr_full(&ci, ci.tgt[t], AB, CD, Acc + (size_t)ci.tgt_tag[t] * nE * nF, nE, nF, res[t]);

        real * o = out + ((size_t)ab * Q->nshell12_clip + cd) * nout;
        int ca[MAXLEV * MAXLEV][3], cb[MAXLEV * MAXLEV][3], cc[MAXLEV * MAXLEV][3], cdd[MAXLEV * MAXLEV][3];
        level_carts(am[0], ca); level_carts(am[1], cb); level_carts(am[2], cc); level_carts(am[3], cdd);
        for(int a = 0; a < NC(am[0]); a++)
        for(int b = 0; b < NC(am[1]); b++)
        for(int c = 0; c < NC(am[2]); c++)
        for(int d = 0; d < NC(am[3]); d++)
        {
            const int oi = ((cart_index(ca[a], ordering) * NC(am[1]) + cart_index(cb[b], ordering)) * NC(am[2])
                            + cart_index(cc[c], ordering)) * NC(am[3]) + cart_index(cdd[d], ordering);
            if(!deriv)
            {
                o[oi] = res[0][((a * NC(am[1]) + b) * NC(am[2]) + c) * NC(am[3]) + d];
                continue;
            }
            real g12[12];
            const int * gg[4] = {ca[a], cb[b], cc[c], cdd[d]};
            for(int t = 0; t < ci.ntarget; t++)
            {
                /* which centre and sign does this target serve? */
                int ctr = -1, plus = 0;
                for(int k = 0; k < 4; k++)
                    if(ci.tgt[t][k] != am[k]) { ctr = k; plus = ci.tgt[t][k] > am[k]; }
                (void)ctr; (void)plus;
            }
            for(int ctr = 0; ctr < 4; ctr++)
            {
                if(ctr == ci.missing) continue;
                int tp = -1, tm = -1;
                for(int t = 0; t < ci.ntarget; t++)
                {
                    if(ci.tgt[t][ctr] == am[ctr] + 1) tp = t;
                    if(ci.tgt[t][ctr] == am[ctr] - 1) tm = t;
                }
                for(int x = 0; x < 3; x++)
                {
                    int g[4][3];
                    for(int k = 0; k < 4; k++) memcpy(g[k], gg[k], sizeof(g[k]));
                    g[ctr][x]++;
                    const int * tt = ci.tgt[tp];
                    int idx = ((psi4_index(g[0][0], g[0][1], g[0][2]) * NC(tt[1]) + psi4_index(g[1][0], g[1][1], g[1][2])) * NC(tt[2])
                               + psi4_index(g[2][0], g[2][1], g[2][2])) * NC(tt[3]) + psi4_index(g[3][0], g[3][1], g[3][2]);
                    real v = res[tp][idx];
                    if(gg[ctr][x] > 0)
                    {
                        g[ctr][x] -= 2;
                        const int * tu = ci.tgt[tm];
                        idx = ((psi4_index(g[0][0], g[0][1], g[0][2]) * NC(tu[1]) + psi4_index(g[1][0], g[1][1], g[1][2])) * NC(tu[2])
                               + psi4_index(g[2][0], g[2][1], g[2][2])) * NC(tu[3]) + psi4_index(g[3][0], g[3][1], g[3][2]);
                        v -= gg[ctr][x] * res[tm][idx];
                    }
                    g12[ctr * 3 + x] = v;
                }
            }
            const int ms = ci.missing;
            for(int x = 0; x < 3; x++)
            {
                real s = 0.0;
                int first = 1;
                for(int ctr = 0; ctr < 4; ctr++)
                {
                    if(ctr == ms) continue;
                    if(first) { s = g12[ctr * 3 + x]; first = 0; }
                    else s += g12[ctr * 3 + x];
                }
                g12[ms * 3 + x] = -s;
            }
            memcpy(o + (size_t)oi * 12, g12, sizeof(g12));
        }
    }
    for(int t = 0; t < ci.ntarget; t++) free(res[t]);
    free(V); free(Acc); free(tmp); free(pst); free(qst);
    return P->nshell12_clip * Q->nshell12_clip;
}

/* Count of primitive quartets the reference evaluates for (P, Q) at this
 * tolerance (after bra and 8-wide ket vector screening). */
long long oracle_count_primq(struct simint_multi_shellpair const * P,
                             struct simint_multi_shellpair const * Q, double screen_tol)
{
    const double tol2 = screen_tol * screen_tol;
    if(screen_tol > 0.0 && P->screen_max * Q->screen_max < tol2)
        return 0;
    const int check = (screen_tol > 0.0) && P->screen && Q->screen;
    int * pst = (int *)malloc(sizeof(int) * (P->nshell12 + 1));
    int * qst = (int *)malloc(sizeof(int) * (Q->nshell12 + 1));
    pair_offsets(P, pst);
    pair_offsets(Q, qst);
    long long n = 0;
    for(int ab = 0; ab < P->nshell12_clip; ab++)
    for(int cd = 0; cd < Q->nshell12_clip; cd++)
    for(int i = pst[ab]; i < pst[ab] + P->nprim12[ab]; i++)
    {
        if(check && P->screen[i] * Q->screen_max < tol2) continue;
        for(int j = qst[cd]; j < qst[cd] + Q->nprim12[cd]; j++)
        {
            if(check)
            {
                const int v0 = j & ~7;
                double vmax = 0.0;
                for(int jj = v0; jj < v0 + 8; jj++)
                    if(P->screen[i] * Q->screen[jj] > vmax) vmax = P->screen[i] * Q->screen[jj];
                if(vmax < tol2) continue;
            }
            n++;
        }
    }
    free(pst); free(qst);
    return n;
}
