// Gaussian-product fill of a multi-shell-pair on the GPU.
//
// simint_fill_multi_shellpair2 (skel/simint/shell/shell.c:425-582) computes,
// for every primitive pair (i, j) of every shell pair of a list, the
// Gaussian-product quantities (P, P-A, P-B, a+b, the prefactor, 2a, 2b), the
// shell pair's A-B and primitive count, pads every group of 16 shell pairs
// to a multiple of 8 slots, and -- with screening -- the primitive screening
// value of each pair, after which the primitive pairs of each shell pair are
// sorted by decreasing screening value (shell.c:37-128).  Here every shell
// pair is one device thread that writes its slots into a device block with
// the layout of the host allocation (one copy back fills every array); the
// Schwarz values (shell_screen.c:127-223: the largest diagonal element of
// (ab|ab) of the two uncontracted primitives) come from the same launch's
// single-primitive records, run through the class kernel as one task list
// (pair_diag_max), and a second kernel scatters them and sorts each shell
// pair's slots with the reference's stable insertion sort.
//
// The arithmetic is the host fill's, operation for operation, in IEEE
// round-to-nearest without contraction (__dmul_rn and friends), so every
// array equals the host fill bit for bit except the prefactor and the
// screening values, which go through exp (and pow for the fast Schwarz
// bound): CUDA's exp and glibc's may differ in the last bit.

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "simint/simint.h"
#include "simint_b200.h"
#include "runtime.h"

#define FILL_SQRT_TWO_PI_52 5.91496717279561287782347843505365022963403204272156069835237
#define FILL_SQRT_TWO_TIMES_PI_52 24.739429451193148050228357586821944304008810699990039583

namespace {

// One shell pair of the list: centres, primitive counts, whether it is a
// shell with itself (i >= j triangle only), its first padded slot, its first
// primitive pair in fill order, the end of the padding after it (group ends
// only), and the offset of alpha_A, coef_A, alpha_B, coef_B in the flat array.
struct FillPair
{
    double A[3], B[3];
    int na, nb, same, slot0, ibase, pad_end, off, pad;
};

// Device pointers of the arrays, at the host allocation's offsets.
struct FillOut
{
    double *x, *y, *z, *pax, *pay, *paz, *pbx, *pby, *pbz, *alpha, *prefac, *screen, *a2, *b2;
    double *abx, *aby, *abz;
    int * nprim12;
};

// Single-primitive pair set of every primitive pair (the Schwarz launch):
// packed records, starts, counts and A-B as the kernels read them.
struct SingleSet
{
    double * rec;
    int *start, *nprim;
    double * AB;
    int n, npad;
};

} // namespace

__global__ void k_pair_fill(const FillPair * __restrict__ pr, const double * __restrict__ flat, int npair,
                            int method, FillOut o, SingleSet s1)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s < npair)
    {
        const FillPair p = pr[s];
        const double * aA = flat + p.off;
        const double * cA = aA + p.na;
        const double * aB = cA + p.na;
        const double * cB = aB + p.nb;
        const double abx = __dsub_rn(p.A[0], p.B[0]);
        const double aby = __dsub_rn(p.A[1], p.B[1]);
        const double abz = __dsub_rn(p.A[2], p.B[2]);
        const double Xab = __dadd_rn(__dadd_rn(__dmul_rn(abx, abx), __dmul_rn(aby, aby)), __dmul_rn(abz, abz));
        int idx = p.slot0, item = p.ibase;
        for(int i = 0; i < p.na; i++)
        {
            const double ai = aA[i], ci = cA[i];
            const double AxAa = __dmul_rn(p.A[0], ai), AyAa = __dmul_rn(p.A[1], ai), AzAa = __dmul_rn(p.A[2], ai);
            const int jend = p.same ? i + 1 : p.nb;
            for(int j = 0; j < jend; j++, idx++, item++)
            {
                const double aj = aB[j], cj = cB[j];
                const double sum = __dadd_rn(ai, aj), mul = __dmul_rn(ai, aj);
                const double e = exp(__ddiv_rn(__dmul_rn(-Xab, mul), sum));
                const double pf1 = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(ci, cj), e), FILL_SQRT_TWO_PI_52), sum);
                const bool dbl = p.same && i != j;
                const double x = __ddiv_rn(__dadd_rn(AxAa, __dmul_rn(aj, p.B[0])), sum);
                const double y = __ddiv_rn(__dadd_rn(AyAa, __dmul_rn(aj, p.B[1])), sum);
                const double z = __ddiv_rn(__dadd_rn(AzAa, __dmul_rn(aj, p.B[2])), sum);
                const double pax = __dsub_rn(x, p.A[0]), pay = __dsub_rn(y, p.A[1]), paz = __dsub_rn(z, p.A[2]);
                const double pbx = __dsub_rn(x, p.B[0]), pby = __dsub_rn(y, p.B[1]), pbz = __dsub_rn(z, p.B[2]);
                o.x[idx] = x; o.y[idx] = y; o.z[idx] = z;
                o.pax[idx] = pax; o.pay[idx] = pay; o.paz[idx] = paz;
                o.pbx[idx] = pbx; o.pby[idx] = pby; o.pbz[idx] = pbz;
                o.alpha[idx] = sum;
                o.prefac[idx] = dbl ? __dmul_rn(pf1, 2.0) : pf1;
                o.a2[idx] = dbl ? sum : __dmul_rn(2.0, ai);
                o.b2[idx] = dbl ? sum : __dmul_rn(2.0, aj);
                if(method == SIMINT_SCREEN_FASTSCHWARZ)
                {
                    // shell.c:455-472
                    const double rho = __ddiv_rn(mul, sum);
                    const double oop = __ddiv_rn(1.0, sum);
                    double g = __dmul_rn(__dmul_rn(FILL_SQRT_TWO_TIMES_PI_52, pow(oop, 2.5)),
                                         exp(__dmul_rn(__dmul_rn(-2.0, rho), Xab)));
                    g = __dmul_rn(g, __dmul_rn(__dmul_rn(__dmul_rn(ci, ci), cj), cj));
                    o.screen[idx] = g;
                }
                else if(method == SIMINT_SCREEN_SCHWARZ)
                {
                    // the primitive pair as a single-primitive shell pair of
                    // two distinct shells: no doubling, 2a and 2b
                    double * r = s1.rec + (size_t)item * SB_REC;
                    r[0] = sum; r[1] = pf1;
                    r[2] = x; r[3] = y; r[4] = z;
                    r[5] = pax; r[6] = pay; r[7] = paz;
                    r[8] = pbx; r[9] = pby; r[10] = pbz;
                    r[11] = __dmul_rn(2.0, ai); r[12] = __dmul_rn(2.0, aj);
                    r[13] = 0.0; r[14] = 0.0; r[15] = INFINITY;
                    s1.start[item] = item;
                    s1.nprim[item] = 1;
                    s1.AB[3 * (size_t)item + 0] = abx;
                    s1.AB[3 * (size_t)item + 1] = aby;
                    s1.AB[3 * (size_t)item + 2] = abz;
                }
            }
        }
        // padding after a group of 16 shell pairs (shell.c:538-570)
        for(; idx < p.pad_end; idx++)
        {
            o.alpha[idx] = 1.0;
            o.prefac[idx] = 0.0;
            o.x[idx] = o.y[idx] = o.z[idx] = 0.0;
            o.pax[idx] = o.pay[idx] = o.paz[idx] = 0.0;
            o.pbx[idx] = o.pby[idx] = o.pbz[idx] = 0.0;
            if(o.screen)
                o.screen[idx] = 0.0;
            o.a2[idx] = 1.0;
            o.b2[idx] = 1.0;
        }
        o.abx[s] = abx; o.aby[s] = aby; o.abz[s] = abz;
        o.nprim12[s] = p.same ? (p.na * (p.na + 1)) / 2 : p.na * p.nb;
    }
    // padded slots of the single-primitive set (its last group only)
    if(method == SIMINT_SCREEN_SCHWARZ && s == 0)
        for(int k = s1.n; k < s1.npad; k++)
        {
            double * r = s1.rec + (size_t)k * SB_REC;
            r[0] = 1.0;
            for(int f = 1; f <= 10; f++)
                r[f] = 0.0;
            r[11] = 1.0; r[12] = 1.0;
            r[13] = 0.0; r[14] = 0.0; r[15] = INFINITY;
        }
}

// Schwarz values into the screen array (method 1), then each shell pair's
// slots in decreasing screening value: the reference's stable insertion sort
// (shell.c:37-128), swapping all fourteen primitive arrays.
__global__ void k_pair_sort(const FillPair * __restrict__ pr, int npair, const double * __restrict__ dmax,
                            FillOut o)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if(s >= npair)
        return;
    const FillPair p = pr[s];
    const int np = p.same ? (p.na * (p.na + 1)) / 2 : p.na * p.nb;
    const int lo = p.slot0;
    if(dmax)
        for(int k = 0; k < np; k++)
            o.screen[lo + k] = dmax[p.ibase + k];
    double * arr[14] = {o.x, o.y, o.z, o.pax, o.pay, o.paz, o.pbx, o.pby, o.pbz,
                        o.alpha, o.prefac, o.screen, o.a2, o.b2};
    for(int a = lo + 1; a < lo + np; a++)
        for(int b = a; b > lo && o.screen[b - 1] < o.screen[b]; b--)
            for(int v = 0; v < 14; v++)
            {
                const double t = arr[v][b - 1];
                arr[v][b - 1] = arr[v][b];
                arr[v][b] = t;
            }
}

namespace sb200 {

static int g_pair_fill_mode = -1;

int pair_fill_mode()
{
    if(g_pair_fill_mode < 0)
    {
        const char * v = getenv("SIMINT_B200_PAIR_FILL");
        g_pair_fill_mode = SIMINT_B200_PAIR_FILL_AUTO;
        if(v && !strcmp(v, "host"))
            g_pair_fill_mode = SIMINT_B200_PAIR_FILL_HOST;
        else if(v && !strcmp(v, "gpu"))
            g_pair_fill_mode = SIMINT_B200_PAIR_FILL_GPU;
    }
    return g_pair_fill_mode;
}

// Fill P (allocated by simint_allocate_multi_shellpair2 for the same list)
// on the device.  Returns 0, or a negative SIMINT_B200_ERR_* with P's arrays
// unspecified.
int gpu_fill_multi_shellpair2(int npair, const simint_shell * AB, simint_multi_shellpair * P, int screen_method)
{
    if(npair <= 0)
        return SIMINT_B200_ERR_ARG;
    init_tables();
    if(ensure_device() < 0)
        return SIMINT_B200_ERR_NODEVICE;
    Workspace & w = workspace();
    if(!w.stream && cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess)
    {
        set_error("cudaStreamCreate failed");
        return SIMINT_B200_ERR_CUDA;
    }
    cudaStream_t st = w.stream;
    // the shell-pair table and the flat exponent / coefficient array
    std::vector<FillPair> pr(npair);
    std::vector<double> flat;
    int idx = 0, item = 0;
    for(int s = 0; s < npair; s++)
    {
        const simint_shell * A = &AB[2 * s];
        const simint_shell * B = &AB[2 * s + 1];
        FillPair & p = pr[s];
        p.A[0] = A->x; p.A[1] = A->y; p.A[2] = A->z;
        p.B[0] = B->x; p.B[1] = B->y; p.B[2] = B->z;
        p.na = A->nprim; p.nb = B->nprim;
        p.same = compare_shell(A, B);
        p.slot0 = idx;
        p.ibase = item;
        p.off = (int)flat.size();
        p.pad = 0;
        flat.insert(flat.end(), A->alpha, A->alpha + A->nprim);
        flat.insert(flat.end(), A->coef, A->coef + A->nprim);
        flat.insert(flat.end(), B->alpha, B->alpha + B->nprim);
        flat.insert(flat.end(), B->coef, B->coef + B->nprim);
        const int np = p.same ? (p.na * (p.na + 1)) / 2 : p.na * p.nb;
        idx += np;
        item += np;
        if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= npair)
            idx = SIMINT_SIMD_ROUND(idx);
        p.pad_end = idx;
    }
    const int n = item;
    const char * base = (const char *)P->ptr;
    const size_t used = (size_t)((const char *)(P->nprim12 + npair) - base);
    const int method = screen_method;
    if(method && !P->screen)
    {
        set_error("pair set allocated without a screen array");
        return SIMINT_B200_ERR_ARG;
    }
    // device memory: block, pair table, flat array, single-primitive set
    const int npad1 = SIMINT_SIMD_ROUND(n);
    const size_t szBlock = (used + 255) & ~(size_t)255;
    const size_t szPr = ((size_t)npair * sizeof(FillPair) + 255) & ~(size_t)255;
    const size_t szFlat = (flat.size() * sizeof(double) + 255) & ~(size_t)255;
    const bool schwarz = method == SIMINT_SCREEN_SCHWARZ;
    const size_t szRec = schwarz ? (size_t)npad1 * SB_REC * sizeof(double) : 0;
    const size_t szInt = schwarz ? (((size_t)n * sizeof(int) + 255) & ~(size_t)255) : 0;
    const size_t szAB = schwarz ? (((size_t)n * 3 * sizeof(double) + 255) & ~(size_t)255) : 0;
    const size_t szMax = schwarz ? (((size_t)n * sizeof(double) + 255) & ~(size_t)255) : 0;
    const size_t total = szBlock + szPr + szFlat + szRec + 2 * szInt + szAB + szMax;
    char * d = nullptr;
    if(cudaMallocAsync((void **)&d, total, st) != cudaSuccess)
    {
        cudaGetLastError();
        set_error("out of device memory in the pair fill");
        return SIMINT_B200_ERR_CUDA;
    }
    char * dblock = d;
    FillPair * dpr = (FillPair *)(d + szBlock);
    double * dflat = (double *)(d + szBlock + szPr);
    char * q = d + szBlock + szPr + szFlat;
    SingleSet s1;
    s1.rec = (double *)q; q += szRec;
    s1.start = (int *)q; q += szInt;
    s1.nprim = (int *)q; q += szInt;
    s1.AB = (double *)q; q += szAB;
    double * dmax = schwarz ? (double *)q : nullptr;
    s1.n = n;
    s1.npad = npad1;
    auto at = [&](const void * a) { return a ? dblock + ((const char *)a - base) : nullptr; };
    FillOut o;
    o.x = (double *)at(P->x); o.y = (double *)at(P->y); o.z = (double *)at(P->z);
    o.pax = (double *)at(P->PA_x); o.pay = (double *)at(P->PA_y); o.paz = (double *)at(P->PA_z);
    o.pbx = (double *)at(P->PB_x); o.pby = (double *)at(P->PB_y); o.pbz = (double *)at(P->PB_z);
    o.alpha = (double *)at(P->alpha); o.prefac = (double *)at(P->prefac);
    o.screen = method ? (double *)at(P->screen) : nullptr;
    o.a2 = (double *)at(P->alpha2); o.b2 = (double *)at(P->beta2);
    o.abx = (double *)at(P->AB_x); o.aby = (double *)at(P->AB_y); o.abz = (double *)at(P->AB_z);
    o.nprim12 = (int *)at(P->nprim12);
    int rc = 0;
    cudaMemcpyAsync(dpr, pr.data(), (size_t)npair * sizeof(FillPair), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dflat, flat.data(), flat.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    // the host vectors must outlive the copies from pageable memory
    cudaStreamSynchronize(st);
    k_pair_fill<<<(unsigned)((npair + 127) / 128), 128, 0, st>>>(dpr, dflat, npair, method, o, s1);
    count_launch(1);
    if(schwarz && n > 0)
    {
        PairSetDev d1;
        d1.prim = s1.rec;
        d1.pstart = s1.start;
        d1.nprim = s1.nprim;
        d1.AB = s1.AB;
        d1.screen_max = 1.e99;
        d1.npair = n;
        rc = pair_diag_max(d1, AB[0].am, AB[1].am, n, dmax, st);
    }
    if(rc == 0 && method)
    {
        k_pair_sort<<<(unsigned)((npair + 127) / 128), 128, 0, st>>>(dpr, npair, dmax, o);
        count_launch(1);
    }
    if(rc == 0)
        cudaMemcpyAsync(P->ptr, dblock, used, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(d, st);
    cudaError_t e = cudaStreamSynchronize(st);
    if(e == cudaSuccess)
        e = cudaGetLastError();
    if(rc == 0 && e != cudaSuccess)
    {
        set_error(std::string("CUDA error in the pair fill: ") + cudaGetErrorString(e));
        rc = SIMINT_B200_ERR_CUDA;
    }
    if(rc != 0)
        return rc;
    P->nshell12 = npair;
    P->nshell12_clip = npair;
    P->nprim = n;
    P->screen_max = 1.e99;     // shell.c:434 (only ever raised)
    P->am1 = AB[2 * (npair - 1)].am;
    P->am2 = AB[2 * (npair - 1) + 1].am;
    return 0;
}

} // namespace sb200

extern "C" int simint_b200_set_pair_fill(int mode)
{
    if(mode != SIMINT_B200_PAIR_FILL_AUTO && mode != SIMINT_B200_PAIR_FILL_HOST && mode != SIMINT_B200_PAIR_FILL_GPU)
        return SIMINT_B200_ERR_ARG;
    sb200::g_pair_fill_mode = mode;
    return 0;
}

extern "C" int simint_b200_get_pair_fill(void) { return sb200::pair_fill_mode(); }
