/* Driver of Simint's public C API: shells and shell-pair lists in, integrals
 * out.  TEST INFRASTRUCTURE ONLY.
 *
 * The same source is compiled
 *   - into every reference build under oracle/_ref/ (oracle/build_reflib.py),
 *     against that build's own headers: there it is the checker and the
 *     timed CPU baseline (OpenMP over rows, dynamic schedule, one work buffer
 *     per thread, as skel/test/benchmark_eri.cpp:135-216 does), and
 *   - against include/ and linked to libsimint_b200.so (tests/c_host.py):
 *     a C host that drives the B200 library through the very calls the
 *     reference's users make.
 * Only public API is used: simint_create_shell, simint_normalize_shells,
 * simint_create_multi_shellpair2, simint_shellscreen_schwarz,
 * simint_compute_eri_deriv, simint_ostei_workmem
 * (skel/simint/shell/shell.h, shell_screen.h, simint_eri.h). */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "simint/simint.h"
#include "simint/shell/shell_screen.h"

static struct simint_shell * g_sh = NULL;
static int g_nsh = 0;
static struct simint_multi_shellpair ** g_ps = NULL;
static int g_nps = 0, g_cps = 0;
/* Per pair-set handle: a copy of the screening values of an (s s) pair set
 * as created (NULL for other sets).  The reference's (ss|ss) kernel
 * (skel/ostei_s_s_s_s.c) writes zeros into Q.screen past the last ket
 * primitive when it tests a partial vector; with a clipped ket list
 * (nshell12_clip < nshell12) those are the next pairs' values, so a later
 * call that reaches further into the same list skips primitives it should
 * not.  rd_rows keeps the shared pair sets as created: rows that evaluate
 * into `out` run such calls on a private copy of the values, and timed runs
 * put the values back after the loop. */
static double ** g_scr0 = NULL;

static double wtime(void)
{
#ifdef _OPENMP
    return omp_get_wtime();
#else
    return 0.0;
#endif
}

int rd_simd_len(void) { return SIMINT_SIMD_LEN; }
int rd_max_am(void) { return SIMINT_OSTEI_MAXAM; }
int rd_max_der(void) { return SIMINT_OSTEI_MAXDER; }

void rd_init(void) { simint_init(); }

/* Shells from flat arrays (primitives of shell k at offset sum_{i<k} nprim[i]);
 * normalised with simint_normalize_shells when `normalize` is set. */
int rd_set_shells(int n, const int * am, const int * nprim, const double * xyz,
                  const double * alpha, const double * coef, int normalize)
{
    if(g_sh)
    {
        simint_free_shells(g_nsh, g_sh);
        free(g_sh);
    }
    g_sh = (struct simint_shell *)malloc(sizeof(struct simint_shell) * (size_t)(n > 0 ? n : 1));
    if(!g_sh)
        return -1;
    g_nsh = n;
    simint_initialize_shells(n, g_sh);
    size_t off = 0;
    for(int k = 0; k < n; k++)
    {
        simint_create_shell(nprim[k], am[k], xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2],
                            alpha + off, coef + off, &g_sh[k]);
        off += (size_t)nprim[k];
    }
    if(normalize)
        simint_normalize_shells(n, g_sh);
    return 0;
}

/* The (normalised) contraction coefficients, concatenated. */
void rd_get_coefs(double * out)
{
    size_t off = 0;
    for(int k = 0; k < g_nsh; k++)
    {
        memcpy(out + off, g_sh[k].coef, sizeof(double) * (size_t)g_sh[k].nprim);
        off += (size_t)g_sh[k].nprim;
    }
}

/* Contracted Schwarz value max |(ab|ab)| of each pair (pairs = 2*npair shell
 * indices), simint_shellscreen_schwarz. */
void rd_shell_schwarz(int npair, const int * pairs, double * out, int nthreads)
{
#ifdef _OPENMP
    #pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads > 0 ? nthreads : 1)
#endif
    for(int p = 0; p < npair; p++)
        out[p] = simint_shellscreen_schwarz(&g_sh[pairs[2 * p]], &g_sh[pairs[2 * p + 1]]);
}

/* Room for `need` handles. */
static int reserve_handles(int need)
{
    while(g_cps < need)
    {
        int nc = g_cps ? 2 * g_cps : 64;
        struct simint_multi_shellpair ** np =
            (struct simint_multi_shellpair **)realloc(g_ps, sizeof(*np) * (size_t)nc);
        if(!np)
            return -1;
        g_ps = np;
        double ** ns = (double **)realloc(g_scr0, sizeof(*ns) * (size_t)nc);
        if(!ns)
            return -1;
        g_scr0 = ns;
        g_cps = nc;
    }
    return 0;
}

/* Padded primitive slots of a pair set (the reference's layout: each batch
 * of SIMINT_NSHELL_SIMD pairs rounded up to SIMINT_SIMD_LEN). */
static int padded_slots(const struct simint_multi_shellpair * P)
{
    int idx = 0;
    for(int p = 0; p < P->nshell12; p++)
    {
        idx += P->nprim12[p];
        if(((p + 1) % SIMINT_NSHELL_SIMD) == 0 || p + 1 >= P->nshell12)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    return idx;
}

static double * screen_copy(const struct simint_multi_shellpair * P)
{
    if(P->am1 != 0 || P->am2 != 0 || !P->screen)
        return NULL;
    const size_t n = (size_t)padded_slots(P);
    double * c = (double *)malloc(sizeof(double) * (n ? n : 1));
    if(c)
        memcpy(c, P->screen, sizeof(double) * n);
    return c;
}

/* End (padded primitive index) of the last ket pair of a clipped (ss|ss)
 * call, or -1 when the call is not one. */
static int ssss_clip_end(const struct simint_multi_shellpair * P, const struct simint_multi_shellpair * Q)
{
    if(P->am1 || P->am2 || Q->am1 || Q->am2 || Q->nshell12_clip >= Q->nshell12 || Q->nshell12_clip <= 0)
        return -1;
    int idx = 0;
    for(int p = 0; p < Q->nshell12_clip; p++)
    {
        idx += Q->nprim12[p];
        if(((p + 1) % SIMINT_NSHELL_SIMD) == 0 && p + 1 < Q->nshell12_clip)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    return idx;
}

/* A multi shell pair over an explicit pair list; returns its handle. */
int rd_pairset(int npair, const int * pairs, int screen_method)
{
    if(reserve_handles(g_nps + 1) != 0)
        return -1;
    struct simint_shell * AB = (struct simint_shell *)malloc(sizeof(struct simint_shell) * 2 * (size_t)npair);
    struct simint_multi_shellpair * P = (struct simint_multi_shellpair *)malloc(sizeof(*P));
    if(!AB || !P)
    {
        free(AB);
        free(P);
        return -1;
    }
    for(int p = 0; p < npair; p++)
    {
        AB[2 * p] = g_sh[pairs[2 * p]];
        AB[2 * p + 1] = g_sh[pairs[2 * p + 1]];
    }
    simint_initialize_multi_shellpair(P);
    simint_create_multi_shellpair2(npair, AB, P, screen_method);
    free(AB);
    g_ps[g_nps] = P;
    g_scr0[g_nps] = screen_copy(P);
    return g_nps++;
}

/* Many single-pair sets at once (one per pair), OpenMP over pairs; handles
 * are first, first+1, ... (returns first). */
int rd_pairsets_single(int npair, const int * pairs, int screen_method, int nthreads)
{
    if(reserve_handles(g_nps + npair) != 0)
        return -1;
    const int first = g_nps;
#ifdef _OPENMP
    #pragma omp parallel for schedule(dynamic, 8) num_threads(nthreads > 0 ? nthreads : 1)
#endif
    for(int p = 0; p < npair; p++)
    {
        struct simint_shell AB[2];
        AB[0] = g_sh[pairs[2 * p]];
        AB[1] = g_sh[pairs[2 * p + 1]];
        struct simint_multi_shellpair * P = (struct simint_multi_shellpair *)malloc(sizeof(*P));
        simint_initialize_multi_shellpair(P);
        simint_create_multi_shellpair2(1, AB, P, screen_method);
        g_ps[first + p] = P;
        g_scr0[first + p] = NULL;        /* one pair: never clipped */
    }
    g_nps += npair;
    return first;
}

/* nset pair sets at once (set s: counts[s] pairs, consecutive in `pairs`),
 * OpenMP over sets; handles first, first+1, ... (returns first). */
int rd_pairsets_multi(int nset, const int * counts, const int * pairs, int screen_method, int nthreads)
{
    if(reserve_handles(g_nps + nset) != 0)
        return -1;
    const int first = g_nps;
    long long * start = (long long *)malloc(sizeof(long long) * (size_t)(nset + 1));
    start[0] = 0;
    for(int s = 0; s < nset; s++)
        start[s + 1] = start[s] + counts[s];
#ifdef _OPENMP
    #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
#endif
    for(int s = 0; s < nset; s++)
    {
        const int n = counts[s];
        struct simint_shell * AB = (struct simint_shell *)malloc(sizeof(struct simint_shell) * 2 * (size_t)(n > 0 ? n : 1));
        for(int p = 0; p < n; p++)
        {
            AB[2 * p] = g_sh[pairs[2 * (start[s] + p)]];
            AB[2 * p + 1] = g_sh[pairs[2 * (start[s] + p) + 1]];
        }
        struct simint_multi_shellpair * P = (struct simint_multi_shellpair *)malloc(sizeof(*P));
        simint_initialize_multi_shellpair(P);
        simint_create_multi_shellpair2(n, AB, P, screen_method);
        free(AB);
        g_ps[first + s] = P;
        g_scr0[first + s] = screen_copy(P);
    }
    free(start);
    g_nps += nset;
    return first;
}

void rd_pairsets_free(void)
{
    for(int k = 0; k < g_nps; k++)
    {
        simint_free_multi_shellpair(g_ps[k]);
        free(g_ps[k]);
        free(g_scr0[k]);
        g_scr0[k] = NULL;
    }
    g_nps = 0;
}

int rd_pairset_info(int h, int * nshell12, int * nprim, double * screen_max)
{
    if(h < 0 || h >= g_nps)
        return -1;
    *nshell12 = g_ps[h]->nshell12;
    *nprim = g_ps[h]->nprim;
    *screen_max = g_ps[h]->screen_max;
    return 0;
}

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static long long row_size(const struct simint_multi_shellpair * P,
                          const struct simint_multi_shellpair * Q, int deriv)
{
    return (long long)P->nshell12_clip * Q->nshell12_clip * ncart(P->am1) * ncart(P->am2)
           * ncart(Q->am1) * ncart(Q->am2) * (deriv ? 12 : 1);
}

/* Primitive quartets that simint_compute_eri(P, Q, tol) evaluates: the
 * generated kernels' pair-level test (ostei.c:16-19), bra-primitive test
 * (OSTEI_Writer.cpp:507) and SIMD-vector ket test (OSTEI_Writer.cpp:570-586)
 * over ket batches of SIMINT_NSHELL_SIMD pairs (:480-486, 716), restated. */
static long long count_primq(const struct simint_multi_shellpair * P,
                             const struct simint_multi_shellpair * Q, double tol)
{
    const double tol2 = tol * tol;
    const int check = tol > 0.0 && P->screen && Q->screen;
    if(tol > 0.0 && P->screen_max * Q->screen_max < tol2)
        return 0;
    /* the (ss|ss) kernel tests the vector at the clip with zeros past it */
    const int cend = ssss_clip_end(P, Q);
    const int qend = cend >= 0 ? cend : 0x7fffffff;
    long long n = 0;
    int istart = 0;
    for(int ab = 0; ab < P->nshell12_clip; ++ab)
    {
        const int iend = istart + P->nprim12[ab];
        int jstart = 0;
        for(int cd = 0; cd < Q->nshell12_clip; cd += SIMINT_NSHELL_SIMD)
        {
            const int nb = (cd + SIMINT_NSHELL_SIMD > Q->nshell12_clip) ? Q->nshell12_clip - cd
                                                                       : SIMINT_NSHELL_SIMD;
            int jend = jstart;
            for(int k = 0; k < nb; k++)
                jend += Q->nprim12[cd + k];
            for(int i = istart; i < iend; ++i)
            {
                if(check && P->screen[i] * Q->screen_max < tol2)
                    continue;
                for(int j = jstart; j < jend; j += SIMINT_SIMD_LEN)
                {
                    if(check)
                    {
                        double vmax = 0.0;
                        for(int l = 0; l < SIMINT_SIMD_LEN && j + l < qend; l++)
                        {
                            const double v = P->screen[i] * Q->screen[j + l];
                            vmax = v > vmax ? v : vmax;
                        }
                        if(vmax < tol2)
                            continue;
                    }
                    n += (jend - j < SIMINT_SIMD_LEN) ? jend - j : SIMINT_SIMD_LEN;
                }
            }
            jstart = SIMINT_SIMD_ROUND(jend);
        }
        istart = iend;
    }
    return n;
}

/* Evaluate rows: row r is simint_compute_eri_deriv(deriv, P[bh[r]], Q[kh[r]]
 * clipped to kc[r] ket pairs (kc <= 0: all), tol).  With `out`, row r's
 * integrals go to out + off[r] (zeros where the call returns -1); without,
 * each thread writes into its own scratch (timing).  ret[r] and primq[r]
 * (primitive quartets evaluated) are filled when non-NULL.  OpenMP over rows
 * with `nthreads` threads, dynamic schedule.  Returns the wall seconds of
 * the loop (0 without OpenMP). */
double rd_rows(int nrow, const int * bh, const int * kh, const int * kc, int deriv, double tol,
               int nthreads, double * out, const long long * off, int * ret, long long * primq)
{
    long long maxsz = 1;
    if(!out)
        for(int r = 0; r < nrow; r++)
        {
            struct simint_multi_shellpair Q = *g_ps[kh[r]];
            if(kc[r] > 0 && kc[r] < Q.nshell12)
                Q.nshell12_clip = kc[r];
            const long long s = row_size(g_ps[bh[r]], &Q, deriv);
            maxsz = s > maxsz ? s : maxsz;
        }
    if(primq)
        for(int r = 0; r < nrow; r++)
        {
            struct simint_multi_shellpair Q = *g_ps[kh[r]];
            if(kc[r] > 0 && kc[r] < Q.nshell12)
                Q.nshell12_clip = kc[r];
            primq[r] = count_primq(g_ps[bh[r]], &Q, tol);
        }
    const int nt = nthreads > 0 ? nthreads : 1;
    const size_t wsz = simint_ostei_workmem(deriv, SIMINT_OSTEI_MAXAM) + 64;
    double t0 = 0.0, t1 = 0.0;
#ifdef _OPENMP
    #pragma omp parallel num_threads(nt)
#endif
    {
        double * work = (double *)SIMINT_ALLOC(wsz);
        double * scratch = out ? NULL : (double *)SIMINT_ALLOC(sizeof(double) * (size_t)maxsz);
        double * scr = NULL;             /* private screening values (see g_scr0) */
        size_t scr_cap = 0;
#ifdef _OPENMP
        #pragma omp barrier
        #pragma omp master
#endif
        t0 = wtime();
#ifdef _OPENMP
        #pragma omp for schedule(dynamic)
#endif
        for(int r = 0; r < nrow; r++)
        {
            struct simint_multi_shellpair Q = *g_ps[kh[r]];
            if(kc[r] > 0 && kc[r] < Q.nshell12)
                Q.nshell12_clip = kc[r];
            const struct simint_multi_shellpair * P = g_ps[bh[r]];
            const int cend = (out && g_scr0[kh[r]] && tol > 0.0) ? ssss_clip_end(P, &Q) : -1;
            if(cend >= 0)
            {
                /* the whole array: a library may read every slot */
                const size_t n = (size_t)padded_slots(&Q);
                if(n > scr_cap)
                {
                    free(scr);
                    scr = (double *)malloc(sizeof(double) * n);
                    scr_cap = scr ? n : 0;
                }
                if(scr)
                {
                    memcpy(scr, g_scr0[kh[r]], sizeof(double) * n);
                    Q.screen = scr;
                }
            }
            double * dst = out ? out + off[r] : scratch;
            const int rc = simint_compute_eri_deriv(deriv, P, &Q, tol, work, dst);
            if(rc < 0 && out)
                memset(dst, 0, sizeof(double) * (size_t)row_size(P, &Q, deriv));
            if(ret)
                ret[r] = rc;
        }
#ifdef _OPENMP
        #pragma omp master
#endif
        t1 = wtime();
        SIMINT_FREE(work);
        if(scratch)
            SIMINT_FREE(scratch);
        free(scr);
    }
    if(!out && tol > 0.0)
    {
        /* timed runs call the reference as it is: put back what its (ss|ss)
         * kernel overwrote (each (s s) ket set once) */
        char * done = (char *)calloc((size_t)(g_nps > 0 ? g_nps : 1), 1);
        for(int r = 0; r < nrow && done; r++)
        {
            const struct simint_multi_shellpair * Q = g_ps[kh[r]];
            if(g_scr0[kh[r]] && Q->screen && !done[kh[r]])
            {
                memcpy(Q->screen, g_scr0[kh[r]], sizeof(double) * (size_t)padded_slots(Q));
                done[kh[r]] = 1;
            }
        }
        free(done);
    }
    return t1 - t0;
}
