/*
 * TEST INFRASTRUCTURE ONLY: the timed CPU baseline.
 *
 * Runs the oracle the way the reference's own benchmark drives its library
 * (skel/test/benchmark_eri.cpp:135-216): one multi-shell-pair per bra shell
 * pair, the whole ket list as Q, OpenMP dynamic scheduling over the bra
 * pairs, every thread with its own output buffer.
 */
#include <omp.h>
#include <stdlib.h>
#include "simint/shell/shell.h"

int oracle_compute_eri(struct simint_multi_shellpair const * P,
                       struct simint_multi_shellpair const * Q,
                       double screen_tol, int deriv, int ordering, double * out);

/* Returns wall seconds; out_checksum receives the sum of all outputs. */
double oracle_bench_omp(int nbra, struct simint_multi_shellpair const * Plist,
                        struct simint_multi_shellpair const * Q,
                        double screen_tol, int deriv, int nthreads, int nout_per_bra,
                        double * out_checksum)
{
    if(nthreads > 0)
        omp_set_num_threads(nthreads);
    double total = 0.0;
    const double t0 = omp_get_wtime();
    #pragma omp parallel reduction(+:total)
    {
        double * buf = (double *)malloc(sizeof(double) * (size_t)nout_per_bra);
        #pragma omp for schedule(dynamic)
        for(int b = 0; b < nbra; b++)
        {
            int r = oracle_compute_eri(&Plist[b], Q, screen_tol, deriv, 0, buf);
            if(r > 0)
                for(int k = 0; k < nout_per_bra; k++)
                    total += buf[k];
        }
        free(buf);
    }
    const double t1 = omp_get_wtime();
    if(out_checksum)
        *out_checksum = total;
    return t1 - t0;
}

long long oracle_count_primq(struct simint_multi_shellpair const * P,
                             struct simint_multi_shellpair const * Q, double screen_tol);

/* Time a list of independent (P_k, Q_k) calls, OpenMP dynamic over k (the
 * way a QC code would thread simint_compute_eri calls).  Returns wall
 * seconds; *nprimq gets the primitive quartets the calls evaluate. */
double oracle_bench_rows(int n, struct simint_multi_shellpair const * const * Plist,
                         struct simint_multi_shellpair const * const * Qlist,
                         double screen_tol, int nthreads, long long * nprimq,
                         double * out_checksum)
{
    if(nthreads > 0)
        omp_set_num_threads(nthreads);
    long long npq = 0;
    for(int k = 0; k < n; k++)
        npq += oracle_count_primq(Plist[k], Qlist[k], screen_tol);
    double total = 0.0;
    const double t0 = omp_get_wtime();
    #pragma omp parallel reduction(+:total)
    {
        double * buf = NULL;
        size_t cap = 0;
        #pragma omp for schedule(dynamic)
        for(int k = 0; k < n; k++)
        {
            const struct simint_multi_shellpair * P = Plist[k];
            const struct simint_multi_shellpair * Q = Qlist[k];
            const int nc = ((P->am1 + 1) * (P->am1 + 2) / 2) * ((P->am2 + 1) * (P->am2 + 2) / 2)
                         * ((Q->am1 + 1) * (Q->am1 + 2) / 2) * ((Q->am2 + 1) * (Q->am2 + 2) / 2);
            const size_t need = (size_t)P->nshell12_clip * Q->nshell12_clip * nc;
            if(need > cap)
            {
                free(buf);
                buf = (double *)malloc(sizeof(double) * need);
                cap = need;
            }
            if(oracle_compute_eri(P, Q, screen_tol, 0, 0, buf) > 0)
                for(size_t i = 0; i < need; i++)
                    total += buf[i];
        }
        free(buf);
    }
    const double t1 = omp_get_wtime();
    if(nprimq)
        *nprimq = npq;
    if(out_checksum)
        *out_checksum = total;
    return t1 - t0;
}
