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
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "simint_b200.h"
#include "runtime.h"
#include "cartinfo.cuh"
#include "gen/boys_grid.inc"

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
    // per process (the attribute holds for every device the kernel runs on
    // in this context); idempotent, so concurrent first calls are harmless
    static std::once_flag attr_once[3];
    std::call_once(attr_once[mode], [mode] {
        if(mode == 0) cudaFuncSetAttribute(k_coop<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if(mode == 1) cudaFuncSetAttribute(k_coop<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if(mode == 2) cudaFuncSetAttribute(k_coop<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    });
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

// ===========================================================================
// Entry point that allocates nothing.
//
// Some callers cannot allocate device memory: code running inside a
// framework that owns the whole device pool (it hands out buffers but
// forbids cudaMalloc), code called while a memory pool is being captured or
// frozen, or hosts that must never trigger a cudaMalloc/cudaFree (an
// implicit device synchronisation) on their hot path.  For them the
// cooperative kernel can run with every working array in memory that exists
// from load time: its global scratch, the Boys tables and an identity ket
// order live in file-scope static device arrays of fixed size.  The caller
// provides the packed pair data and the output in its own device buffers.
// ===========================================================================

#define NOALLOC_SCRATCH_DOUBLES (4 * 1024 * 1024)   // 32 MiB of scratch per device
#define NOALLOC_MAX_KETS (1 << 20)                  // identity ket order, 4 MiB
#define NOALLOC_MAX_DEV 64

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];
static __device__ __align__(256) int g_noalloc_kord[NOALLOC_MAX_KETS];
static __device__ __align__(256) double g_noalloc_boys[366 * 32 + 32];

__global__ void k_noalloc_iota(int * p, int n)
{
    for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        p[i] = i;
}

namespace {

struct NoallocDev
{
    int ready = 0;
    double * scratch = nullptr;
    int * kord = nullptr;
    double * boys = nullptr;
};

NoallocDev g_noalloc[NOALLOC_MAX_DEV];
std::mutex g_noalloc_mutex;
CartInfo g_noalloc_cart[CI_NCART];

// Packed layout of one pair set (the same records simint_compute_eri
// uploads, see ostei_device.cuh), computed without allocating.
size_t noalloc_layout(const simint_multi_shellpair * P, sb200::PackedLayout & L)
{
    int idx = 0;
    for(int p = 0; p < P->nshell12; p++)
    {
        idx += P->nprim12[p];
        if(((p + 1) % SIMINT_NSHELL_SIMD) == 0 || p + 1 >= P->nshell12)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    L.npad = idx;
    L.npair = P->nshell12;
    L.off_rec = 0;
    L.off_start = (size_t)idx * SB_REC * sizeof(double);
    L.off_nprim = L.off_start + ((P->nshell12 * sizeof(int) + 255) & ~(size_t)255);
    L.off_AB = L.off_nprim + ((P->nshell12 * sizeof(int) + 255) & ~(size_t)255);
    return L.off_AB + 3 * (size_t)P->nshell12 * sizeof(double);
}

// Per-device set-up: resolve the static arrays' device addresses, upload
// the Boys and Cartesian tables, fill the identity ket order.
int noalloc_setup(int dev)
{
    NoallocDev & d = g_noalloc[dev];
    if(d.ready)
        return 0;
    if(cudaGetSymbolAddress((void **)&d.scratch, g_noalloc_scratch) != cudaSuccess ||
       cudaGetSymbolAddress((void **)&d.kord, g_noalloc_kord) != cudaSuccess ||
       cudaGetSymbolAddress((void **)&d.boys, g_noalloc_boys) != cudaSuccess)
    {
        cudaGetLastError();
        return SIMINT_B200_ERR_CUDA;
    }
    if(cudaMemcpyToSymbol(g_noalloc_boys, simint_b200_boys_grid_host, sizeof(double) * 366 * 32) != cudaSuccess ||
       cudaMemcpyToSymbol(g_noalloc_boys, simint_b200_boys_longfac_host, sizeof(double) * 32,
                          sizeof(double) * 366 * 32) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    cart_table_fill(g_noalloc_cart);
    if(cudaMemcpyToSymbol(c_cartinfo, g_noalloc_cart, sizeof(CartInfo) * CI_NCART) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    k_noalloc_iota<<<256, 256>>>(d.kord, NOALLOC_MAX_KETS);
    if(cudaDeviceSynchronize() != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    if(cudaFuncSetAttribute(k_coop<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    d.ready = 1;
    return 0;
}

} // namespace

extern "C" size_t simint_b200_packed_size(struct simint_multi_shellpair const * P)
{
    if(!P)
        return 0;
    sb200::PackedLayout L;
    return noalloc_layout(P, L);
}

extern "C" int simint_b200_pack(struct simint_multi_shellpair const * P, void * dst, size_t cap)
{
    if(!P || !dst)
        return SIMINT_B200_ERR_ARG;
    sb200::PackedLayout L;
    const size_t need = noalloc_layout(P, L);
    if(cap < need)
        return SIMINT_B200_ERR_ARG;
    char * base = (char *)dst;
    double * rec = (double *)(base + L.off_rec);
    int * start = (int *)(base + L.off_start);
    int idx = 0;
    for(int p = 0; p < P->nshell12; p++)
    {
        start[p] = idx;
        idx += P->nprim12[p];
        if(((p + 1) % SIMINT_NSHELL_SIMD) == 0 || p + 1 >= P->nshell12)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    const bool has_screen = P->screen != nullptr;
    for(int s = 0; s < L.npad; s++)
    {
        double * r = rec + (size_t)s * SB_REC;
        r[0] = P->alpha[s]; r[1] = P->prefac[s];
        r[2] = P->x[s]; r[3] = P->y[s]; r[4] = P->z[s];
        r[5] = P->PA_x[s]; r[6] = P->PA_y[s]; r[7] = P->PA_z[s];
        r[8] = P->PB_x[s]; r[9] = P->PB_y[s]; r[10] = P->PB_z[s];
        r[11] = P->alpha2 ? P->alpha2[s] : 0.0;
        r[12] = P->beta2 ? P->beta2[s] : 0.0;
        const double sc = has_screen ? P->screen[s] : 0.0;
        r[13] = sc;
        r[15] = has_screen ? sqrt(sc > 0.0 ? sc : 0.0) : INFINITY;
    }
    for(int g = 0; g < L.npad; g += 8)
    {
        double m = 0.0;
        for(int s = g; s < g + 8 && s < L.npad; s++)
            m = fmax(m, rec[(size_t)s * SB_REC + 13]);
        for(int s = g; s < g + 8 && s < L.npad; s++)
            rec[(size_t)s * SB_REC + 14] = m;
    }
    memcpy(base + L.off_nprim, P->nprim12, P->nshell12 * sizeof(int));
    double * ab = (double *)(base + L.off_AB);
    for(int p = 0; p < P->nshell12; p++)
    {
        ab[3 * p + 0] = P->AB_x[p];
        ab[3 * p + 1] = P->AB_y[p];
        ab[3 * p + 2] = P->AB_z[p];
    }
    return 0;
}

extern "C" long long simint_b200_noalloc_scratch_bytes(void)
{
    return (long long)NOALLOC_SCRATCH_DOUBLES * (long long)sizeof(double);
}

extern "C" int simint_b200_compute_eri_noalloc(int deriv,
                                              struct simint_multi_shellpair const * P, const void * dev_P,
                                              struct simint_multi_shellpair const * Q, const void * dev_Q,
                                              double screen_tol, double * dev_integrals, void * stream)
{
    if(!P || !Q || !dev_P || !dev_Q || !dev_integrals || deriv < 0 || deriv > 1)
        return SIMINT_B200_ERR_ARG;
    const double tol2 = screen_tol * screen_tol;
    if(screen_tol > 0.0 && P->screen_max * Q->screen_max < tol2)
        return -1;
    const long long ntask = (long long)P->nshell12_clip * Q->nshell12_clip;
    if(ntask == 0)
        return 0;
    if(Q->nshell12_clip > NOALLOC_MAX_KETS)
        return SIMINT_B200_ERR_ARG;
    const int req[4] = {P->am1, P->am2, Q->am1, Q->am2};
    for(int k = 0; k < 4; k++)
        if(req[k] < 0 || req[k] > SIMINT_OSTEI_MAXAM)
            return SIMINT_B200_ERR_CLASS;
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEV)
        return SIMINT_B200_ERR_NODEVICE;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mutex);
        const int rc = noalloc_setup(dev);
        if(rc != 0)
            return rc;
    }
    const NoallocDev & d = g_noalloc[dev];
    CoopClass g;
    if(!sb200::coop_setup(req, deriv, g) || g.smem_doubles * 8 > 200 * 1024)
        return SIMINT_B200_ERR_CLASS;
    const int threads = 128;
    const long long per_cta = (long long)threads * g.h_per_thread + g.cta_size;
    const long long max_cta = NOALLOC_SCRATCH_DOUBLES / per_cta;
    if(max_cta < 1)
        return SIMINT_B200_ERR_ARG;        // one CTA's scratch exceeds the static array
    const int per_sm = std::max(1, std::min(8, (int)((220 * 1024) / std::max<size_t>((size_t)g.smem_doubles * 8, 1))));
    long long grid = std::min<long long>(ntask, 148LL * per_sm);
    grid = std::max<long long>(1, std::min(grid, max_cta));
    sb200::PackedLayout LP, LQ;
    noalloc_layout(P, LP);
    noalloc_layout(Q, LQ);
    KernArgs a;
    memset(&a, 0, sizeof(a));
    a.P = sb200::device_view((const char *)dev_P, LP, P->screen_max);
    a.Q = sb200::device_view((const char *)dev_Q, LQ, Q->screen_max);
    a.kord = d.kord;
    a.ntask = ntask;
    a.nQ = Q->nshell12_clip;
    a.nQc = a.nQ;
    a.check = (screen_tol > 0.0) && P->screen && Q->screen;
    a.tol2 = tol2;
    a.out = dev_integrals;
    a.nout = g.am[0] >= 0 ? (((req[0] + 1) * (req[0] + 2) / 2) * ((req[1] + 1) * (req[1] + 2) / 2)
                             * ((req[2] + 1) * (req[2] + 2) / 2) * ((req[3] + 1) * (req[3] + 2) / 2)
                             * (deriv ? 12 : 1)) : 0;
    a.boys = d.boys;
    const size_t smem = (size_t)g.smem_doubles * sizeof(double);
    k_coop<0><<<(unsigned)grid, threads, smem, (cudaStream_t)stream>>>(a, g, d.scratch);
    if(cudaGetLastError() != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    return (int)ntask;
}
