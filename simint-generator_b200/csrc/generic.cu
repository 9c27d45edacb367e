// Generic ERI kernel: any AM class up to SIMINT_OSTEI_MAXAM, deriv 0 and 1.
//
// This is the table-driven fallback for classes that have no straight-line
// kernel (their VRR/HRR state does not fit in registers) and for the
// deriv=1 path.  One thread computes one shell quartet with the dense
// Obara-Saika scheme: every (e0|f0)^(m) of the class by the per-element
// rule of the reference planner (centre order OSTEI_VRR_Algorithm_Base.cpp:
// 449-469, xyz choice Makowski.hpp:113-117, 8-term step Makowski.hpp:
// 87-242), contraction with the deriv weights (OSTEIDeriv1_Writer.cpp:53-94),
// HRR bra then ket (OSTEI_HRR_Algorithm_Base.cpp:160-283), deriv formation
// by translational invariance (OSTEIDeriv1_Writer.cpp:334-537).
//
// Working arrays live in a device scratch buffer, interleaved across
// threads (element k of thread t at k*stride + t) so that a warp's accesses
// coalesce.  The grid is sized so the scratch fits the buffer; threads loop
// over tasks.

#include <cuda_runtime.h>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "simint_b200.h"
#include "runtime.h"

#define GMAXL 10                 // Cartesian levels handled by the tables
#define GNCART 286               // lev_off(GMAXL + 1)

struct CartInfo
{
    signed char ijk[3];
    signed char lev, pos, dir;   // AM level, Psi4 position, recursion direction
    short m1[3];                 // flat index of g - 1_x (or -1)
    short m2;                    // flat index of g - 2_dir (or -1)
    short p1[3];                 // flat index of g + 1_x (or -1)
};

__constant__ CartInfo c_cart[GNCART];

struct GenClass
{
    int am[4];
    int deriv, missing, ntarget, ntag;
    int tgt[8][4];
    int tgt_tag[8];
    int brastep_j, ketstep_l;
    int Emax, Fmax, L, ket_first;
    int nE, nF;
    int vbase[GMAXL][GMAXL];
    int vsize;
    int off_acc, off_H, off_bra, off_H2, off_res[8];
    int scratch;                 // doubles per thread
    int ordering;
};

__device__ __forceinline__ int g_lev_off(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
__device__ __forceinline__ int g_nc(int l) { return ((l + 1) * (l + 2)) / 2; }

__device__ __forceinline__ int g_cart_index(int g, int ordering)
{
    const CartInfo & c = c_cart[g];
    const int l = c.lev;
    if(ordering == SIMINT_B200_ORDERING_GAMESS && (l == 2 || l == 3))
    {
        const int i = c.ijk[0], j = c.ijk[1], k = c.ijk[2];
        if(l == 2)
        {
            if(i == 2) return 0;
            if(j == 2) return 1;
            if(k == 2) return 2;
            if(i == 1 && j == 1) return 3;
            if(i == 1) return 4;
            return 5;
        }
        // l == 3: xxx yyy zzz xxy xxz xyy yyz xzz yzz xyz
        if(i == 3) return 0;
        if(j == 3) return 1;
        if(k == 3) return 2;
        if(i == 2 && j == 1) return 3;
        if(i == 2) return 4;
        if(i == 1 && j == 2) return 5;
        if(j == 2) return 6;
        if(i == 1 && k == 2) return 7;
        if(k == 2) return 8;
        return 9;
    }
    return c.pos;
}

#define SCR(k) scr[(size_t)(k) * stride + tid]

// one side of the HRR for one column (see oracle hrr_side): tops on the
// top centre with levels lo..lt in src(g), output target (ta, tb) block
template<typename SRC, typename DST>
__device__ void hrr_side_col(int right_step, int ta, int tb, const double X[3],
                             SRC src, DST dst, double * __restrict__ scr, int offH,
                             size_t stride, int tid)
{
    const int lt = ta + tb;
    const int nstep = right_step ? g_lev_off(tb + 1) : g_lev_off(ta + 1);
    const int lo = right_step ? ta : tb;
    for(int g = g_lev_off(lo); g < g_lev_off(lt + 1); g++)
        SCR(offH + g * nstep) = src(g);
    const int sl_max = right_step ? tb : ta;
    for(int sl = 1; sl <= sl_max; sl++)
        for(int tl = lo; tl <= lt - sl; tl++)
            for(int it = g_lev_off(tl); it < g_lev_off(tl + 1); it++)
                for(int is = g_lev_off(sl); is < g_lev_off(sl + 1); is++)
                {
                    const int x = c_cart[is].dir;
                    const int ism = c_cart[is].m1[x];
                    const int itp = c_cart[it].p1[x];
                    const double a = SCR(offH + it * nstep + ism);
                    const double b = SCR(offH + itp * nstep + ism);
                    SCR(offH + it * nstep + is) = right_step ? fma(X[x], a, b) : fma(-X[x], a, b);
                }
    for(int a = 0; a < g_nc(ta); a++)
        for(int b = 0; b < g_nc(tb); b++)
        {
            const int gA = g_lev_off(ta) + a, gB = g_lev_off(tb) + b;
            const int it = right_step ? gA : gB;
            const int is = right_step ? gB : gA;
            dst(a * g_nc(tb) + b, SCR(offH + it * nstep + is));
        }
}

template<int MODE>
__global__ void __launch_bounds__(128) k_generic(const KernArgs a, const GenClass gc,
                                                 double * __restrict__ scr, size_t stride)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if((size_t)tid >= stride)
        return;
    const int L = gc.L;
    const int nF = gc.nF;
    for(long long t = tid; t < a.ntask; t += (long long)stride)
    {
        int iP, iQ;
        long long off;
        task_of<MODE>(a, t, iP, iQ, off);
        QuartetCtx c;
        make_ctx(a, iP, iQ, c);
        for(int k = 0; k < gc.ntag * gc.nE * nF; k++)
            SCR(gc.off_acc + k) = 0.0;
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
                double F[24];
                // Boys, L < 4 from the grid per order, else top order + recursion
                if(L < 4)
                {
                    if(s.T >= 0.0 && s.T < 36.5)
                    {
                        const int idx = (int)(10.0 * (s.T + 0.05));
                        const double dx = (double)idx * 0.1 - s.T;
                        for(int n = 0; n <= L; n++)
                            F[n] = boys_taylor(c.boys + idx * 32 + n, dx);
                    }
                    else
                    {
                        const double x1 = 1.0 / s.T;
                        double x2 = sqrt(x1);
                        for(int n = 0; n <= L; n++)
                        {
                            F[n] = c.boys[SB_BOYS_LONGFAC_OFF + n] * x2;
                            x2 *= x1;
                        }
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
                    for(int n = L - 1; n >= 0; n--)
                        F[n] = (1.0 / (2.0 * n + 1.0)) * fma(x2, F[n + 1], ex);
                }
                for(int n = 0; n <= L; n++)
                    F[n] *= s.prefac;
                const double XP[3] = {gc.brastep_j ? s.PAx : s.PBx, gc.brastep_j ? s.PAy : s.PBy,
                                      gc.brastep_j ? s.PAz : s.PBz};
                const double XQ[3] = {gc.ketstep_l ? s.QCx : s.QDx, gc.ketstep_l ? s.QCy : s.QDy,
                                      gc.ketstep_l ? s.QCz : s.QDz};
                const double aop[3] = {s.aopPQx, s.aopPQy, s.aopPQz};
                const double aoq[3] = {s.aoqPQx, s.aoqPQy, s.aoqPQz};
#define VV(gE, gF, m) SCR(gc.vbase[c_cart[gE].lev][c_cart[gF].lev] + \
        (c_cart[gE].pos * g_nc(c_cart[gF].lev) + c_cart[gF].pos) * (L - c_cart[gE].lev - c_cart[gF].lev + 1) + (m))
                for(int m = 0; m <= L; m++)
                    VV(0, 0, m) = F[m];
                for(int eL = 0; eL <= gc.Emax; eL++)
                    for(int fL = 0; fL <= gc.Fmax; fL++)
                    {
                        if(eL == 0 && fL == 0)
                            continue;
                        const int mmax = L - eL - fL;
                        const bool use_ket = (fL > 0) && (gc.ket_first || eL == 0);
                        for(int gE = g_lev_off(eL); gE < g_lev_off(eL + 1); gE++)
                            for(int gF = g_lev_off(fL); gF < g_lev_off(fL + 1); gF++)
                            {
                                if(use_ket)
                                {
                                    const int x = c_cart[gF].dir;
                                    const int gF1 = c_cart[gF].m1[x];
                                    const int gF2 = (c_cart[gF].ijk[x] >= 2) ? c_cart[gF].m2 : -1;
                                    const int gE1 = c_cart[gE].m1[x];
                                    const double c0 = (double)(c_cart[gF].ijk[x] - 1) * s.oo2q;
                                    const double c2 = (double)c_cart[gE].ijk[x] * s.oo2pq;
                                    for(int m = 0; m <= mmax; m++)
                                    {
                                        double v = XQ[x] * VV(gE, gF1, m);
                                        v = fma(aoq[x], VV(gE, gF1, m + 1), v);
                                        if(gF2 >= 0)
                                            v = fma(c0, fma(s.a_over_q, VV(gE, gF2, m + 1), VV(gE, gF2, m)), v);
                                        if(gE1 >= 0)
                                            v = fma(c2, VV(gE1, gF1, m + 1), v);
                                        VV(gE, gF, m) = v;
                                    }
                                }
                                else
                                {
                                    const int x = c_cart[gE].dir;
                                    const int gE1 = c_cart[gE].m1[x];
                                    const int gE2 = (c_cart[gE].ijk[x] >= 2) ? c_cart[gE].m2 : -1;
                                    const int gF1 = c_cart[gF].m1[x];
                                    const double c0 = (double)(c_cart[gE].ijk[x] - 1) * s.oo2p;
                                    const double c2 = (double)c_cart[gF].ijk[x] * s.oo2pq;
                                    for(int m = 0; m <= mmax; m++)
                                    {
                                        double v = XP[x] * VV(gE1, gF, m);
                                        v = fma(aop[x], VV(gE1, gF, m + 1), v);
                                        if(gE2 >= 0)
                                            v = fma(c0, fma(s.a_over_p, VV(gE2, gF, m + 1), VV(gE2, gF, m)), v);
                                        if(gF1 >= 0)
                                            v = fma(c2, VV(gE1, gF1, m + 1), v);
                                        VV(gE, gF, m) = v;
                                    }
                                }
                            }
                    }
                const double w[5] = {1.0, s.c2a, s.c2b, s.c2c, s.c2d};
                for(int tg = 0; tg < gc.ntag; tg++)
                    for(int gE = 0; gE < gc.nE; gE++)
                        for(int gF = 0; gF < nF; gF++)
                        {
                            const double v = VV(gE, gF, 0);
                            SCR(gc.off_acc + (tg * gc.nE + gE) * nF + gF) += (tg == 0) ? v : v * w[tg];
                        }
#undef VV
            }
        }
        // HRR for every target
        for(int ti = 0; ti < gc.ntarget; ti++)
        {
            const int * tt = gc.tgt[ti];
            const int tg = gc.tgt_tag[ti];
            const int ncolF = g_lev_off(tt[2] + tt[3] + 1);
            const int nbra = g_nc(tt[0]) * g_nc(tt[1]);
            const int nket = g_nc(tt[2]) * g_nc(tt[3]);
            const int accb = gc.off_acc + tg * gc.nE * nF;
            for(int col = 0; col < ncolF; col++)
                hrr_side_col(gc.brastep_j, tt[0], tt[1], c.AB,
                             [&](int g) { return SCR(accb + g * nF + col); },
                             [&](int r, double v) { SCR(gc.off_bra + r * ncolF + col) = v; },
                             scr, gc.off_H, stride, tid);
            const int offr = gc.off_res[ti];
            for(int r = 0; r < nbra; r++)
                hrr_side_col(gc.ketstep_l, tt[2], tt[3], c.CD,
                             [&](int g) { return SCR(gc.off_bra + r * ncolF + g); },
                             [&](int k, double v) { SCR(offr + r * nket + k) = v; },
                             scr, gc.off_H2, stride, tid);
        }
        // output
        double * o = a.out + off;
        const int * am = gc.am;
        const int n1 = g_nc(am[1]), n2 = g_nc(am[2]), n3 = g_nc(am[3]);
        for(int ga = g_lev_off(am[0]); ga < g_lev_off(am[0] + 1); ga++)
        for(int gb = g_lev_off(am[1]); gb < g_lev_off(am[1] + 1); gb++)
        for(int gcc = g_lev_off(am[2]); gcc < g_lev_off(am[2] + 1); gcc++)
        for(int gd = g_lev_off(am[3]); gd < g_lev_off(am[3] + 1); gd++)
        {
            const int oi = ((g_cart_index(ga, gc.ordering) * n1 + g_cart_index(gb, gc.ordering)) * n2
                            + g_cart_index(gcc, gc.ordering)) * n3 + g_cart_index(gd, gc.ordering);
            const int gg[4] = {ga, gb, gcc, gd};
            if(gc.deriv == 0)
            {
                const int r = ((c_cart[ga].pos * n1 + c_cart[gb].pos) * n2 + c_cart[gcc].pos) * n3 + c_cart[gd].pos;
                o[oi] = SCR(gc.off_res[0] + r);
                continue;
            }
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
                    h[ctr] = c_cart[gg[ctr]].p1[x];
                    const int * tp_am = gc.tgt[tp];
                    int r = ((c_cart[h[0]].pos * g_nc(tp_am[1]) + c_cart[h[1]].pos) * g_nc(tp_am[2])
                             + c_cart[h[2]].pos) * g_nc(tp_am[3]) + c_cart[h[3]].pos;
                    double v = SCR(gc.off_res[tp] + r);
                    const int nx = c_cart[gg[ctr]].ijk[x];
                    if(nx > 0)
                    {
                        h[ctr] = c_cart[gg[ctr]].m1[x];
                        const int * tm_am = gc.tgt[tm];
                        r = ((c_cart[h[0]].pos * g_nc(tm_am[1]) + c_cart[h[1]].pos) * g_nc(tm_am[2])
                             + c_cart[h[2]].pos) * g_nc(tm_am[3]) + c_cart[h[3]].pos;
                        v -= nx * SCR(gc.off_res[tm] + r);
                    }
                    g12[ctr * 3 + x] = v;
                }
            }
            for(int x = 0; x < 3; x++)
            {
                double sm = 0.0;
                bool first = true;
                for(int ctr = 0; ctr < 4; ctr++)
                {
                    if(ctr == gc.missing)
                        continue;
                    sm = first ? g12[ctr * 3 + x] : sm + g12[ctr * 3 + x];
                    first = false;
                }
                g12[gc.missing * 3 + x] = -sm;
            }
            for(int k = 0; k < 12; k++)
                o[(size_t)oi * 12 + k] = g12[k];
        }
    }
}

namespace sb200 {

static int lev_off_h(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
static int nc_h(int l) { return ((l + 1) * (l + 2)) / 2; }

// Once per device, under a lock (concurrent first calls from several host
// threads).
static void upload_cart_table()
{
    static std::mutex m;
    static std::vector<char> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(m);
    if((int)done.size() > dev && done[dev])
        return;
    std::vector<CartInfo> t(GNCART);
    std::vector<std::array<int, 3>> cs;
    auto flat = [](int i, int j, int k) -> int {
        if(i < 0 || j < 0 || k < 0) return -1;
        const int l = i + j + k;
        if(l > GMAXL) return -1;
        return lev_off_h(l) + ((l - i) * (l - i + 1)) / 2 + k;
    };
    for(int l = 0; l <= GMAXL; l++)
    {
        carts(l, cs);
        for(size_t p = 0; p < cs.size(); p++)
        {
            CartInfo & c = t[lev_off_h(l) + p];
            const int i = cs[p][0], j = cs[p][1], k = cs[p][2];
            c.ijk[0] = i; c.ijk[1] = j; c.ijk[2] = k;
            c.lev = l;
            c.pos = (signed char)p;
            int dir = -1, mn = 1000;
            for(int x = 0; x < 3; x++)
                if(cs[p][x] > 0 && cs[p][x] < mn) mn = cs[p][x];
            for(int x = 2; x >= 0; x--)
                if(cs[p][x] == mn) { dir = x; break; }
            c.dir = dir;
            c.m1[0] = flat(i - 1, j, k); c.m1[1] = flat(i, j - 1, k); c.m1[2] = flat(i, j, k - 1);
            c.p1[0] = flat(i + 1, j, k); c.p1[1] = flat(i, j + 1, k); c.p1[2] = flat(i, j, k + 1);
            int q[3] = {i, j, k};
            if(dir >= 0) q[dir] -= 2;
            c.m2 = dir >= 0 ? flat(q[0], q[1], q[2]) : -1;
        }
    }
    cudaMemcpyToSymbol(c_cart, t.data(), sizeof(CartInfo) * GNCART);
    if((int)done.size() <= dev)
        done.resize(dev + 1, 0);
    done[dev] = 1;
}

static bool setup_class(const int am[4], int deriv, GenClass & g)
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
        int mx = *std::max_element(am, am + 4);
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
    if(g.Emax >= GMAXL || g.Fmax >= GMAXL)
        return false;
    g.L = g.Emax + g.Fmax;
    g.ket_first = g.Fmax <= g.Emax;
    g.nE = lev_off_h(g.Emax + 1);
    g.nF = lev_off_h(g.Fmax + 1);
    int off = 0;
    for(int e = 0; e <= g.Emax; e++)
        for(int f = 0; f <= g.Fmax; f++)
        {
            g.vbase[e][f] = off;
            off += nc_h(e) * nc_h(f) * (g.L - e - f + 1);
        }
    g.vsize = off;
    g.off_acc = off;
    off += g.ntag * g.nE * g.nF;
    int hmax = 0, h2max = 0, bramax = 0;
    for(int t = 0; t < g.ntarget; t++)
    {
        const int * tt = g.tgt[t];
        const int nall = lev_off_h(tt[0] + tt[1] + 1);
        const int nstep = g.brastep_j ? lev_off_h(tt[1] + 1) : lev_off_h(tt[0] + 1);
        hmax = std::max(hmax, nall * nstep);
        const int nall2 = lev_off_h(tt[2] + tt[3] + 1);
        const int nstep2 = g.ketstep_l ? lev_off_h(tt[3] + 1) : lev_off_h(tt[2] + 1);
        h2max = std::max(h2max, nall2 * nstep2);
        bramax = std::max(bramax, nc_h(tt[0]) * nc_h(tt[1]) * nall2);
    }
    g.off_H = off; off += hmax;
    g.off_H2 = off; off += h2max;
    g.off_bra = off; off += bramax;
    for(int t = 0; t < g.ntarget; t++)
    {
        g.off_res[t] = off;
        off += nc_h(g.tgt[t][0]) * nc_h(g.tgt[t][1]) * nc_h(g.tgt[t][2]) * nc_h(g.tgt[t][3]);
    }
    g.scratch = off;
    g.ordering = ordering();
    return true;
}

int launch_generic(KernArgs & a, const int req[4], const UniqueMap & u, int deriv, int mode,
                   cudaStream_t stream)
{
    (void)u;
    GenClass g;
    if(!setup_class(req, deriv, g))
    {
        set_error("class outside the generic kernel's range");
        return SIMINT_B200_ERR_CLASS;
    }
    upload_cart_table();
    // the generic kernel works on the requested class directly
    a.swapB = a.swapK = a.pq = 0;
    a.oidx = nullptr;
    // threads: enough to fill the GPU, bounded by a 2 GiB scratch budget
    const size_t budget = (size_t)2 << 30;
    size_t nthr = budget / ((size_t)g.scratch * sizeof(double));
    nthr = std::min<size_t>(nthr, 148 * 1024);
    nthr = std::min<size_t>(nthr, (size_t)a.ntask);
    nthr = std::max<size_t>(nthr, 1);
    Workspace & w = workspace();
    if(!w.dscratch.reserve(nthr * g.scratch * sizeof(double)))
    {
        set_error("out of device memory for generic-kernel scratch");
        return SIMINT_B200_ERR_CUDA;
    }
    const int threads = 128;
    const unsigned blocks = (unsigned)((nthr + threads - 1) / threads);
    if(mode == 0)
        k_generic<0><<<blocks, threads, 0, stream>>>(a, g, (double *)w.dscratch.ptr, nthr);
    else if(mode == 1)
        k_generic<1><<<blocks, threads, 0, stream>>>(a, g, (double *)w.dscratch.ptr, nthr);
    else
        k_generic<2><<<blocks, threads, 0, stream>>>(a, g, (double *)w.dscratch.ptr, nthr);
    count_launch(1);
    return 0;
}

} // namespace sb200
