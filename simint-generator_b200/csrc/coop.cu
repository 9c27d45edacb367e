// CTA-cooperative ERI kernel for large AM classes and for deriv=1.
//
// One CTA computes one shell quartet at a time (grid-stride over tasks).
// The primitive loop is sequential; inside a primitive quartet the dense
// Obara-Saika VRR runs as anti-diagonal wavefronts: the (e|f) block of bra
// level e and ket level f depends only on blocks of e+f-1 and e+f-2
// ((e,f-1), (e,f-2), (e-1,f-1) for a ket step; (e-1,0), (e-2,0) for a bra
// step), so every element of wavefront s = e+f is independent and the CTA's
// threads share them; three rolling wavefront buffers live in shared memory
// and one __syncthreads separates wavefronts.  The per-element rule is the
// reference planner's (centre order OSTEI_VRR_Algorithm_Base.cpp:449-469,
// xyz choice Makowski.hpp:113-117, 8-term step Makowski.hpp:87-242).
// Top quartets (m = 0, levels of the HRR targets) are added to per-tag
// accumulators in shared memory as they are produced (deriv weights of
// OSTEIDeriv1_Writer.cpp:53-94).  The HRR (OSTEI_HRR_Algorithm_Base.cpp:
// 160-283) runs once per shell quartet, bra side column-parallel and ket
// side row-parallel, with working arrays in an L2-resident global scratch;
// deriv=1 components are formed by translational invariance
// (OSTEIDeriv1_Writer.cpp:334-537).

#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "simint_b200.h"
#include "runtime.h"
#include "cartinfo.cuh"

#define CMAXL 10
#define CMAXB 12            // blocks per wavefront (levels 0..E, <= CMAXL+1)
#define CMAXS 21            // wavefronts (Emax + Fmax + 1)

struct CoopClass
{
    int am[4];
    int deriv, missing, ntarget, ntag;
    int tgt[8][4];
    int tgt_tag[8];
    int brastep_j, ketstep_l;
    int Emax, Fmax, L, ket_first;
    // wavefront layout: block (e, s-e) of wavefront s at buf + boff[e][f]
    int boff[CMAXL][CMAXL];
    int wsize;                 // doubles per wavefront buffer
    int welem[CMAXS];          // elements in wavefront s
    // accumulators: tag t covers bra levels [elo, ehi], ket levels [flo, fhi]
    int elo[5], ehi[5], flo[5], fhi[5];
    int acc_off[5];            // offset of tag t in the accumulator array
    int acc_nf[5];             // ket columns of tag t (carts of levels flo..fhi)
    int acc_size;
    // global scratch: per thread H (hrr_side_col), per CTA bra stage + results
    int h_per_thread;
    int cta_bra, cta_res[8], cta_size;
    int ordering;
    int smem_doubles;
};

__device__ __forceinline__ int c_lev_off(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
__device__ __forceinline__ int c_nc(int l) { return ((l + 1) * (l + 2)) / 2; }

// Cartesian position in the output ordering, from the shared-memory table
__device__ __forceinline__ int ci_index(const CartInfo * __restrict__ ci, int g, int ordering)
{
    const CartInfo & c = ci[g];
    const int l = c.lev;
    if(ordering == SIMINT_B200_ORDERING_GAMESS && (l == 2 || l == 3))
    {
        const int i = c.ijk[0], j = c.ijk[1], k = c.ijk[2];
        if(l == 2)
            return i == 2 ? 0 : j == 2 ? 1 : k == 2 ? 2 : (i == 1 && j == 1) ? 3 : i == 1 ? 4 : 5;
        return i == 3 ? 0 : j == 3 ? 1 : k == 3 ? 2 : (i == 2 && j == 1) ? 3 : i == 2 ? 4
             : (i == 1 && j == 2) ? 5 : j == 2 ? 6 : (i == 1 && k == 2) ? 7 : k == 2 ? 8 : 9;
    }
    return c.pos;
}

// one side of the HRR for one column, working array H in global scratch
// (same recurrence as the oracle's hrr_side)
template<typename SRC, typename DST>
__device__ void coop_hrr_col(const CartInfo * __restrict__ ci, int right_step, int ta, int tb,
                             double X0, double X1, double X2, SRC src, DST dst,
                             double * __restrict__ H)
{
    const int lt = ta + tb;
    const int nstep = right_step ? c_lev_off(tb + 1) : c_lev_off(ta + 1);
    const int lo = right_step ? ta : tb;
    for(int g = c_lev_off(lo); g < c_lev_off(lt + 1); g++)
        H[g * nstep] = src(g);
    const int sl_max = right_step ? tb : ta;
    for(int sl = 1; sl <= sl_max; sl++)
        for(int tl = lo; tl <= lt - sl; tl++)
            for(int it = c_lev_off(tl); it < c_lev_off(tl + 1); it++)
                for(int is = c_lev_off(sl); is < c_lev_off(sl + 1); is++)
                {
                    const int x = ci[is].dir;
                    const int ism = ci[is].m1[x];
                    const int itp = ci[it].p1[x];
                    const double a = H[it * nstep + ism];
                    const double b = H[itp * nstep + ism];
                    const double X = x == 0 ? X0 : (x == 1 ? X1 : X2);
                    H[it * nstep + is] = right_step ? fma(X, a, b) : fma(-X, a, b);
                }
    for(int a = 0; a < c_nc(ta); a++)
        for(int b = 0; b < c_nc(tb); b++)
        {
            const int gA = c_lev_off(ta) + a, gB = c_lev_off(tb) + b;
            const int it = right_step ? gA : gB;
            const int is = right_step ? gB : gA;
            dst(a * c_nc(tb) + b, H[it * nstep + is]);
        }
}

template<int MODE>
__global__ void __launch_bounds__(128) k_coop(const KernArgs a, const CoopClass gc,
                                              double * __restrict__ gscr)
{
    extern __shared__ double sm[];
    __shared__ CartInfo ci[CI_NCART];
    for(int k = threadIdx.x; k < CI_NCART; k += blockDim.x)
        ci[k] = c_cartinfo[k];
    __syncthreads();
    double * wave = sm;                         // 3 * wsize
    double * acc = sm + 3 * gc.wsize;           // acc_size
    const int L = gc.L;
    const int tid = threadIdx.x;
    const int nth = blockDim.x;
    double * Hth = gscr + ((size_t)blockIdx.x * nth + tid) * gc.h_per_thread;
    double * cta = gscr + (size_t)gridDim.x * nth * gc.h_per_thread + (size_t)blockIdx.x * gc.cta_size;

    for(long long t = blockIdx.x; t < a.ntask; t += gridDim.x)
    {
        int iP, iQ;
        long long off;
        task_of<MODE>(a, t, iP, iQ, off);
        QuartetCtx c;
        make_ctx(a, iP, iQ, c);
        for(int k = tid; k < gc.acc_size; k += nth)
            acc[k] = 0.0;
        __syncthreads();
        for(int i = c.bi0; i < c.bi1; ++i)
        {
            const BraPrim bp = load_bra_prim(c, i);
            if(c.check && bp.skip)
                continue;
            for(int j = c.kj0; j < c.kj1; ++j)
            {
                PrimSetup s;
                if(!prim_setup(c, bp, j, s))
                    continue;
                // Boys F_0..F_L times the prefactor: thread m <= L writes (ss|ss)^(m)
                if(tid <= L)
                {
                    double F[24];
                    if(L < 4)
                    {
                        if(s.T >= 0.0 && s.T < 36.5)
                        {
                            const int idx = (int)(10.0 * (s.T + 0.05));
                            const double dx = (double)idx * 0.1 - s.T;
                            F[tid] = boys_taylor(c.boys + idx * 32 + tid, dx);
                        }
                        else
                        {
                            const double x1 = 1.0 / s.T;
                            double x2 = sqrt(x1);
                            for(int n = 0; n < tid; n++)
                                x2 *= x1;
                            F[tid] = c.boys[SB_BOYS_LONGFAC_OFF + tid] * x2;
                        }
                    }
                    else
                    {
                        if(s.T >= 0.0 && s.T < 36.5)
                        {
                            const int idx = (int)(10.0 * (s.T + 0.05));
                            const double dx = (double)idx * 0.1 - s.T;
                            F[L] = boys_taylor(c.boys + idx * 32 + L, dx);
                        }
                        else
                            F[L] = c.boys[SB_BOYS_LONGFAC_OFF + L] * pow(s.T, -((double)L + 0.5));
                        const double x2 = 2.0 * s.T;
                        const double ex = exp(-s.T);
                        for(int n = L - 1; n >= tid; n--)
                            F[n] = (1.0 / (2.0 * n + 1.0)) * fma(x2, F[n + 1], ex);
                    }
                    wave[tid] = F[tid] * s.prefac;      // block (0,0), wavefront 0
                }
                const double XP0 = gc.brastep_j ? s.PAx : s.PBx, XP1 = gc.brastep_j ? s.PAy : s.PBy,
                             XP2 = gc.brastep_j ? s.PAz : s.PBz;
                const double XQ0 = gc.ketstep_l ? s.QCx : s.QDx, XQ1 = gc.ketstep_l ? s.QCy : s.QDy,
                             XQ2 = gc.ketstep_l ? s.QCz : s.QDz;
#define SEL3(x, a, b, c) ((x) == 0 ? (a) : ((x) == 1 ? (b) : (c)))
#define WTAG(tg) ((tg) == 0 ? 1.0 : ((tg) == 1 ? s.c2a : ((tg) == 2 ? s.c2b : ((tg) == 3 ? s.c2c : s.c2d))))
                // (ss|ss) is a top when both target sides are s
                if(tid == 0)
                    for(int tg = 0; tg < gc.ntag; tg++)
                        if(gc.elo[tg] == 0 && gc.flo[tg] == 0 && gc.ehi[tg] >= 0 && gc.fhi[tg] >= 0)
                            acc[gc.acc_off[tg]] += WTAG(tg) * wave[0];
                __syncthreads();
                for(int sfront = 1; sfront <= gc.Emax + gc.Fmax; sfront++)
                {
                    double * cur = wave + (sfront % 3) * gc.wsize;
                    const double * w1 = wave + ((sfront + 2) % 3) * gc.wsize;   // s-1
                    const double * w2 = wave + ((sfront + 1) % 3) * gc.wsize;   // s-2
                    const int mlen = L - sfront + 1;                            // m = 0..L-s
                    const int e0 = max(0, sfront - gc.Fmax), e1 = min(gc.Emax, sfront);
                    for(int q = tid; q < gc.welem[sfront]; q += nth)
                    {
                        // locate block (e, f) holding flat element q
                        int e = e0, rem = q;
                        for(; e <= e1; e++)
                        {
                            const int nblk = c_nc(e) * c_nc(sfront - e) * mlen;
                            if(rem < nblk) break;
                            rem -= nblk;
                        }
                        const int f = sfront - e;
                        const int m = rem % mlen;
                        const int pp = rem / mlen;
                        const int pe = pp / c_nc(f), pf = pp - pe * c_nc(f);
                        const int gE = c_lev_off(e) + pe, gF = c_lev_off(f) + pf;
                        const bool use_ket = (f > 0) && (gc.ket_first || e == 0);
                        double v;
                        if(use_ket)
                        {
                            const int x = ci[gF].dir;
                            const int gF1 = ci[gF].m1[x];
                            const int nfx = ci[gF].ijk[x];
                            const int gE1 = ci[gE].m1[x];
                            const int mlen1 = mlen + 1, mlen2 = mlen + 2;
                            // (e, f-1) in s-1
                            const double * b1 = w1 + gc.boff[e][f - 1] + (pe * c_nc(f - 1) + ci[gF1].pos) * mlen1;
                            v = SEL3(x, XQ0, XQ1, XQ2) * b1[m];
                            v = fma(SEL3(x, s.aoqPQx, s.aoqPQy, s.aoqPQz), b1[m + 1], v);
                            if(nfx >= 2)
                            {
                                const int gF2 = ci[gF].m2;
                                const double * b2 = w2 + gc.boff[e][f - 2] + (pe * c_nc(f - 2) + ci[gF2].pos) * mlen2;
                                v = fma((double)(nfx - 1) * s.oo2q, fma(s.a_over_q, b2[m + 1], b2[m]), v);
                            }
                            if(gE1 >= 0)
                            {
                                const double * b3 = w2 + gc.boff[e - 1][f - 1]
                                                    + (ci[gE1].pos * c_nc(f - 1) + ci[gF1].pos) * mlen2;
                                v = fma((double)ci[gE].ijk[x] * s.oo2pq, b3[m + 1], v);
                            }
                        }
                        else
                        {
                            const int x = ci[gE].dir;
                            const int gE1 = ci[gE].m1[x];
                            const int nex = ci[gE].ijk[x];
                            const int gF1 = ci[gF].m1[x];
                            const int mlen1 = mlen + 1, mlen2 = mlen + 2;
                            const double * b1 = w1 + gc.boff[e - 1][f] + (ci[gE1].pos * c_nc(f) + pf) * mlen1;
                            v = SEL3(x, XP0, XP1, XP2) * b1[m];
                            v = fma(SEL3(x, s.aopPQx, s.aopPQy, s.aopPQz), b1[m + 1], v);
                            if(nex >= 2)
                            {
                                const int gE2 = ci[gE].m2;
                                const double * b2 = w2 + gc.boff[e - 2][f] + (ci[gE2].pos * c_nc(f) + pf) * mlen2;
                                v = fma((double)(nex - 1) * s.oo2p, fma(s.a_over_p, b2[m + 1], b2[m]), v);
                            }
                            if(gF1 >= 0)
                            {
                                const double * b3 = w2 + gc.boff[e - 1][f - 1]
                                                    + (ci[gE1].pos * c_nc(f - 1) + ci[gF1].pos) * mlen2;
                                v = fma((double)ci[gF].ijk[x] * s.oo2pq, b3[m + 1], v);
                            }
                        }
                        cur[gc.boff[e][f] + pp * mlen + m] = v;
                        if(m == 0)
                            for(int tg = 0; tg < gc.ntag; tg++)
                                if(e >= gc.elo[tg] && e <= gc.ehi[tg] && f >= gc.flo[tg] && f <= gc.fhi[tg])
                                {
                                    const int re = gE - c_lev_off(gc.elo[tg]);
                                    const int rf = gF - c_lev_off(gc.flo[tg]);
                                    acc[gc.acc_off[tg] + re * gc.acc_nf[tg] + rf] += (tg == 0 ? v : v * WTAG(tg));
                                }
                    }
                    __syncthreads();
                }
            }
        }
        // HRR: bra side per ket column, ket side per bra row
        for(int ti = 0; ti < gc.ntarget; ti++)
        {
            const int * tt = gc.tgt[ti];
            const int tg = gc.tgt_tag[ti];
            const int ncolF = c_lev_off(tt[2] + tt[3] + 1);
            const int nbra = c_nc(tt[0]) * c_nc(tt[1]);
            const int nket = c_nc(tt[2]) * c_nc(tt[3]);
            double * bra = cta + gc.cta_bra;
            const int flo = gc.flo[tg], elo = gc.elo[tg];
            for(int col = tid; col < ncolF; col += nth)
            {
                if(col < c_lev_off(flo))
                    continue;     // ket levels below the accumulated range are never read
                coop_hrr_col(ci, gc.brastep_j, tt[0], tt[1], c.AB[0], c.AB[1], c.AB[2],
                             [&](int g) { return acc[gc.acc_off[tg] + (g - c_lev_off(elo)) * gc.acc_nf[tg]
                                                     + (col - c_lev_off(flo))]; },
                             [&](int r, double v) { bra[r * ncolF + col] = v; }, Hth);
            }
            __syncthreads();
            double * res = cta + gc.cta_res[ti];
            for(int r = tid; r < nbra; r += nth)
                coop_hrr_col(ci, gc.ketstep_l, tt[2], tt[3], c.CD[0], c.CD[1], c.CD[2],
                             [&](int g) { return bra[r * ncolF + g]; },
                             [&](int k, double v) { res[r * nket + k] = v; }, Hth);
            __syncthreads();
        }
        // output (ordering permutation; deriv=1 formation)
        double * o = a.out + off;
        const int * am = gc.am;
        const int n0 = c_nc(am[0]), n1 = c_nc(am[1]), n2 = c_nc(am[2]), n3 = c_nc(am[3]);
        const int nall = n0 * n1 * n2 * n3;
        for(int idx = tid; idx < nall; idx += nth)
        {
            const int pd = idx % n3, pc = (idx / n3) % n2, pb = (idx / (n3 * n2)) % n1, pa = idx / (n3 * n2 * n1);
            const int ga = c_lev_off(am[0]) + pa, gb = c_lev_off(am[1]) + pb;
            const int gcc = c_lev_off(am[2]) + pc, gd = c_lev_off(am[3]) + pd;
            const int oi = ((ci_index(ci, ga, gc.ordering) * n1 + ci_index(ci, gb, gc.ordering)) * n2
                            + ci_index(ci, gcc, gc.ordering)) * n3 + ci_index(ci, gd, gc.ordering);
            if(gc.deriv == 0)
            {
                o[oi] = cta[gc.cta_res[0] + idx];
                continue;
            }
            const int gg[4] = {ga, gb, gcc, gd};
            double g12[12];
            for(int ctr = 0; ctr < 4; ctr++)
            {
                if(ctr == gc.missing)
                    continue;
                int tp = -1, tm = -1;
                for(int t2 = 0; t2 < gc.ntarget; t2++)
                {
                    if(gc.tgt[t2][ctr] == am[ctr] + 1) tp = t2;
                    if(gc.tgt[t2][ctr] == am[ctr] - 1) tm = t2;
                }
                for(int x = 0; x < 3; x++)
                {
                    int h[4] = {gg[0], gg[1], gg[2], gg[3]};
                    h[ctr] = ci[gg[ctr]].p1[x];
                    const int * tp_am = gc.tgt[tp];
                    int r = ((ci[h[0]].pos * c_nc(tp_am[1]) + ci[h[1]].pos) * c_nc(tp_am[2])
                             + ci[h[2]].pos) * c_nc(tp_am[3]) + ci[h[3]].pos;
                    double v = cta[gc.cta_res[tp] + r];
                    const int nx = ci[gg[ctr]].ijk[x];
                    if(nx > 0)
                    {
                        h[ctr] = ci[gg[ctr]].m1[x];
                        const int * tm_am = gc.tgt[tm];
                        r = ((ci[h[0]].pos * c_nc(tm_am[1]) + ci[h[1]].pos) * c_nc(tm_am[2])
                             + ci[h[2]].pos) * c_nc(tm_am[3]) + ci[h[3]].pos;
                        v -= nx * cta[gc.cta_res[tm] + r];
                    }
                    g12[ctr * 3 + x] = v;
                }
            }
            for(int x = 0; x < 3; x++)
            {
                double sm3 = 0.0;
                bool first = true;
                for(int ctr = 0; ctr < 4; ctr++)
                {
                    if(ctr == gc.missing)
                        continue;
                    sm3 = first ? g12[ctr * 3 + x] : sm3 + g12[ctr * 3 + x];
                    first = false;
                }
                g12[gc.missing * 3 + x] = -sm3;
            }
            for(int k = 0; k < 12; k++)
                o[(size_t)oi * 12 + k] = g12[k];
        }
        __syncthreads();
    }
}

namespace sb200 {

static int lev_off_h(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
static int nc_h(int l) { return ((l + 1) * (l + 2)) / 2; }

static bool coop_setup(const int am[4], int deriv, CoopClass & g)
{
    memset(&g, 0, sizeof(g));
    memcpy(g.am, am, sizeof(g.am));
    g.deriv = deriv;
    g.missing = -1;
    if(deriv == 0)
    {
        g.ntarget = 1;
        memcpy(g.tgt[0], am, sizeof(g.am));
        g.ntag = 1;
    }
    else
    {
        const int mx = *std::max_element(am, am + 4);
        g.missing = (int)(std::find(am, am + 4, mx) - am);
        for(int c = 0; c < 4; c++)
        {
            if(c == g.missing) continue;
            memcpy(g.tgt[g.ntarget], am, sizeof(g.am));
            g.tgt[g.ntarget][c]++;
            g.tgt_tag[g.ntarget++] = c + 1;
            if(am[c] > 0)
            {
                memcpy(g.tgt[g.ntarget], am, sizeof(g.am));
                g.tgt[g.ntarget][c]--;
                g.tgt_tag[g.ntarget++] = 0;
            }
        }
        g.ntag = 5;
    }
    int hi = 0;
    for(int t = 1; t < g.ntarget; t++)
        if(std::lexicographical_compare(g.tgt[hi], g.tgt[hi] + 4, g.tgt[t], g.tgt[t] + 4))
            hi = t;
    g.brastep_j = g.tgt[hi][0] >= g.tgt[hi][1];
    g.ketstep_l = g.tgt[hi][2] >= g.tgt[hi][3];
    for(int t = 0; t < g.ntarget; t++)
    {
        g.Emax = std::max(g.Emax, g.tgt[t][0] + g.tgt[t][1]);
        g.Fmax = std::max(g.Fmax, g.tgt[t][2] + g.tgt[t][3]);
    }
    if(g.Emax >= CMAXL || g.Fmax >= CMAXL || g.Emax + g.Fmax >= CMAXS)
        return false;
    g.L = g.Emax + g.Fmax;
    g.ket_first = g.Fmax <= g.Emax;
    // wavefront layout
    g.wsize = g.L + 1;
    for(int s = 0; s <= g.L; s++)
    {
        int off = 0;
        for(int e = std::max(0, s - g.Fmax); e <= std::min(g.Emax, s); e++)
        {
            g.boff[e][s - e] = off;
            off += nc_h(e) * nc_h(s - e) * (g.L - s + 1);
        }
        g.welem[s] = off;
        g.wsize = std::max(g.wsize, off);
    }
    // accumulator ranges per tag from its targets (top levels of the HRR)
    for(int tg = 0; tg < 5; tg++)
    {
        g.elo[tg] = 1000; g.ehi[tg] = -1; g.flo[tg] = 1000; g.fhi[tg] = -1;
    }
    for(int t = 0; t < g.ntarget; t++)
    {
        const int * tt = g.tgt[t];
        const int tg = g.tgt_tag[t];
        const int elo = g.brastep_j ? tt[0] : tt[1], ehi = tt[0] + tt[1];
        const int flo = g.ketstep_l ? tt[2] : tt[3], fhi = tt[2] + tt[3];
        g.elo[tg] = std::min(g.elo[tg], elo); g.ehi[tg] = std::max(g.ehi[tg], ehi);
        g.flo[tg] = std::min(g.flo[tg], flo); g.fhi[tg] = std::max(g.fhi[tg], fhi);
    }
    int off = 0;
    for(int tg = 0; tg < g.ntag; tg++)
    {
        if(g.ehi[tg] < 0)
        {
            g.elo[tg] = g.flo[tg] = 1;  // empty range
            g.ehi[tg] = g.fhi[tg] = 0;
            g.acc_nf[tg] = 0;
            g.acc_off[tg] = off;
            continue;
        }
        g.acc_off[tg] = off;
        g.acc_nf[tg] = lev_off_h(g.fhi[tg] + 1) - lev_off_h(g.flo[tg]);
        off += (lev_off_h(g.ehi[tg] + 1) - lev_off_h(g.elo[tg])) * g.acc_nf[tg];
    }
    g.acc_size = off;
    g.smem_doubles = 3 * g.wsize + g.acc_size;
    // global scratch
    int hmax = 0, bramax = 0, cres = 0;
    for(int t = 0; t < g.ntarget; t++)
    {
        const int * tt = g.tgt[t];
        const int nall = lev_off_h(tt[0] + tt[1] + 1);
        const int nstep = g.brastep_j ? lev_off_h(tt[1] + 1) : lev_off_h(tt[0] + 1);
        const int nall2 = lev_off_h(tt[2] + tt[3] + 1);
        const int nstep2 = g.ketstep_l ? lev_off_h(tt[3] + 1) : lev_off_h(tt[2] + 1);
        hmax = std::max(hmax, std::max(nall * nstep, nall2 * nstep2));
        bramax = std::max(bramax, nc_h(tt[0]) * nc_h(tt[1]) * nall2);
    }
    g.h_per_thread = hmax;
    g.cta_bra = 0;
    cres = bramax;
    for(int t = 0; t < g.ntarget; t++)
    {
        g.cta_res[t] = cres;
        cres += nc_h(g.tgt[t][0]) * nc_h(g.tgt[t][1]) * nc_h(g.tgt[t][2]) * nc_h(g.tgt[t][3]);
    }
    g.cta_size = cres;
    g.ordering = ordering();
    return true;
}

bool coop_supported(const int am[4], int deriv)
{
    CoopClass g;
    if(!coop_setup(am, deriv, g))
        return false;
    return g.smem_doubles * 8 <= 200 * 1024;
}

int launch_coop(KernArgs & a, const int req[4], int deriv, int mode, cudaStream_t stream)
{
    CoopClass g;
    if(!coop_setup(req, deriv, g) || g.smem_doubles * 8 > 200 * 1024)
    {
        set_error("class outside the cooperative kernel's range");
        return SIMINT_B200_ERR_CLASS;
    }
    upload_cart_info();
    a.swapB = a.swapK = a.pq = 0;
    a.oidx = nullptr;
    const int threads = 128;
    const size_t smem = (size_t)g.smem_doubles * sizeof(double);
    static bool attr_set[3] = {false, false, false};
    if(!attr_set[mode])
    {
        if(mode == 0) cudaFuncSetAttribute(k_coop<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if(mode == 1) cudaFuncSetAttribute(k_coop<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if(mode == 2) cudaFuncSetAttribute(k_coop<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        attr_set[mode] = true;
    }
    const int per_sm = std::max(1, std::min(8, (int)((220 * 1024) / std::max<size_t>(smem, 1))));
    long long grid = std::min<long long>(a.ntask, 148LL * per_sm);
    grid = std::max<long long>(grid, 1);
    const size_t scratch = ((size_t)grid * threads * g.h_per_thread + (size_t)grid * g.cta_size) * sizeof(double);
    Workspace & w = workspace();
    if(!w.dscratch.reserve(scratch))
    {
        set_error("out of device memory for cooperative-kernel scratch");
        return SIMINT_B200_ERR_CUDA;
    }
    if(mode == 0)
        k_coop<0><<<(unsigned)grid, threads, smem, stream>>>(a, g, (double *)w.dscratch.ptr);
    else if(mode == 1)
        k_coop<1><<<(unsigned)grid, threads, smem, stream>>>(a, g, (double *)w.dscratch.ptr);
    else
        k_coop<2><<<(unsigned)grid, threads, smem, stream>>>(a, g, (double *)w.dscratch.ptr);
    count_launch(1);
    return 0;
}

} // namespace sb200
