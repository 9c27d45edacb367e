// CTA-cooperative ERI kernel, table-driven (v2): large AM classes, deriv 0/1.
//
// One CTA computes one shell quartet at a time.  Per class the host builds
// (once) a table of work items: one item per Cartesian pair (e-cart, f-cart)
// of every needed (e|f) block of the dense Obara-Saika VRR, holding the
// shared-memory offsets of its sources, the recursion direction and the
// integer factors of the reference's 8-term step (Makowski.hpp:87-242,
// centre order OSTEI_VRR_Algorithm_Base.cpp:449-469).  Blocks are grouped
// into anti-diagonal wavefronts s = e+f (a block depends only on s-1 and
// s-2) and each block keeps only the auxiliary orders m it really feeds.
//
// Surviving primitive quartets (the reference's screening tests) are
// compacted in order and processed B at a time: a thread owns an item and
// runs it for all B primitive quartets and all its m values, so one
// __syncthreads per wavefront serves B primitive quartets and every thread
// has B*m independent FMA chains.  Top quartets are summed into per-tag
// accumulators by the owning thread (deriv weights of
// OSTEIDeriv1_Writer.cpp:53-94).  After the primitive loop the HRR
// (OSTEI_HRR_Algorithm_Base.cpp:160-283) runs level by level over all
// columns (bra side) and rows (ket side) in shared memory; deriv=1 components
// are formed by translational invariance (OSTEIDeriv1_Writer.cpp:334-537).

#include <cuda_runtime.h>
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "simint_b200.h"
#include "runtime.h"
#include "cartinfo.cuh"

#define C2_MAXL 10
#define C2_MAXS 20
#define C2_NCOEF 24
#define C2_THREADS 256

struct C2Params
{
    int am[4];
    int deriv, missing, ntarget, ntag, L, B;
    int tgt[6][4];
    int tgt_tag[6];
    int brastep_j, ketstep_l;
    int Emax, Fmax;
    int elo[5], ehi[5], flo[5], fhi[5], acc_off[5], acc_nf[5], acc_size;
    int wsize;                    // doubles per (wave, batch entry)
    int smax;                     // last wavefront
    int wstart[C2_MAXS + 2];      // item range of wavefront s: [wstart[s], wstart[s+1])
    const int4 * items;           // 2 x int4 per item
    int off_acc, off_coef, off_surv, off_hrr;   // shared-memory layout (doubles)
    int hrr_layer;                // doubles per HRR layer buffer
    int smem_doubles;
    int ordering;
    int res_size;                 // deriv 1: doubles of all target results per CTA
    int res_off[6];
};

// item layout
//   a = {dst, src1, src2, src3}                 (offsets of the m = 0 slot)
//   b = {x | ket << 2 | nA << 3 | nB << 8 | mlen << 16,  gE | gF << 16,  tagmask, 0}

__device__ __forceinline__ int c2_lev_off(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
__device__ __forceinline__ int c2_nc(int l) { return ((l + 1) * (l + 2)) / 2; }

__device__ __forceinline__ int c2_index(const CartInfo * __restrict__ ci, int g, int ordering)
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

// coefficient slots of one primitive quartet in shared memory
enum { K_XP0, K_XP1, K_XP2, K_XQ0, K_XQ1, K_XQ2, K_AOP0, K_AOP1, K_AOP2, K_AOQ0, K_AOQ1, K_AOQ2,
       K_AP, K_AQ, K_O2P, K_O2Q, K_O2PQ, K_W1, K_W2, K_W3, K_W4 };

// One side of the HRR for every column at once, layer by layer in shared
// memory.  in(g, col) gives the tops (functions on the top centre, levels
// lo..lt); out(r, col, v) receives the (ta tb) block.
template<typename IN, typename OUT>
__device__ void c2_hrr_side(const CartInfo * __restrict__ ci, int right_step, int ta, int tb, int ncol,
                            double X0, double X1, double X2, IN in, OUT out,
                            double * __restrict__ L0, double * __restrict__ L1)
{
    const int lt = ta + tb;
    const int lo = right_step ? ta : tb;
    const int sl_max = right_step ? tb : ta;
    const int tid = threadIdx.x, nth = blockDim.x;
    // layer 0: tops, index (gt - lev_off(lo)) * ncol + col
    const int n0 = (c2_lev_off(lt + 1) - c2_lev_off(lo)) * ncol;
    for(int k = tid; k < n0; k += nth)
    {
        const int col = k % ncol, gt = c2_lev_off(lo) + k / ncol;
        L0[k] = in(gt, col);
    }
    __syncthreads();
    double * src = L0;
    double * dst = L1;
    for(int sl = 1; sl <= sl_max; sl++)
    {
        // layer sl: (gt in levels lo..lt-sl) x (gs in level sl) x col
        const int ngt = c2_lev_off(lt - sl + 1) - c2_lev_off(lo);
        const int ngtp = c2_lev_off(lt - sl + 2) - c2_lev_off(lo);   // previous layer's gt range
        const int nsl = c2_nc(sl), nslm = c2_nc(sl - 1);
        const int n = ngt * nsl * ncol;
        for(int k = tid; k < n; k += nth)
        {
            const int col = k % ncol;
            const int r = k / ncol;
            const int ps = r % nsl, it = c2_lev_off(lo) + r / nsl;
            const int is = c2_lev_off(sl) + ps;
            const int x = ci[is].dir;
            const int ism = ci[is].m1[x];
            const int itp = ci[it].p1[x];
            const int pm = ci[ism].pos;
            const double a = src[(((it - c2_lev_off(lo)) * nslm) + pm) * ncol + col];
            const double b = src[(((itp - c2_lev_off(lo)) * nslm) + pm) * ncol + col];
            const double X = x == 0 ? X0 : (x == 1 ? X1 : X2);
            dst[k] = right_step ? fma(X, a, b) : fma(-X, a, b);
            (void)ngtp;
        }
        __syncthreads();
        double * t = src; src = dst; dst = t;
    }
    // the last layer holds gt at level (right ? ta : tb), gs at level sl_max
    const int na = c2_nc(ta), nb = c2_nc(tb);
    const int nsl = c2_nc(sl_max);
    for(int k = tid; k < na * nb * ncol; k += nth)
    {
        const int col = k % ncol, r = k / ncol;
        const int pa = r / nb, pb = r % nb;
        const int pt = right_step ? pa : pb, ps = right_step ? pb : pa;
        out(r, col, src[(pt * nsl + ps) * ncol + col]);
    }
    __syncthreads();
}

template<int MODE, bool MIXED>
__global__ void __launch_bounds__(C2_THREADS) k_coop2(const KernArgs a, const C2Params p,
                                                     double * __restrict__ gres)
{
    extern __shared__ double sm[];
    __shared__ CartInfo ci[CI_NCART];
    __shared__ int s_cnt;
    for(int k = threadIdx.x; k < CI_NCART; k += blockDim.x)
        ci[k] = c_cartinfo[k];
    const int tid = threadIdx.x, nth = blockDim.x;
    const int B = p.B, L = p.L, W = p.wsize;
    double * wave = sm;
    double * acc = sm + p.off_acc;
    double * coef = sm + p.off_coef;
    int * surv = (int *)(sm + p.off_surv);
    double * res = gres + (size_t)blockIdx.x * p.res_size;
    __syncthreads();

    for(long long t = blockIdx.x; t < a.ntask; t += gridDim.x)
    {
        int iP, iQ;
        long long off;
        task_of<MODE>(a, t, iP, iQ, off);
        QuartetCtx c;
        make_ctx(a, iP, iQ, c);
        for(int k = tid; k < p.acc_size; k += nth)
            acc[k] = 0.0;
        const int ni = c.bi1 - c.bi0, nj = c.kj1 - c.kj0;
        const int ncand = ni * nj;
        for(int k0 = 0; k0 < ncand; k0 += nth)
        {
            // ordered compaction of the surviving primitive quartets k0..k0+nth
            if(tid == 0)
                s_cnt = 0;
            __syncthreads();
            const int k = k0 + tid;
            bool ok = false;
            if(k < ncand)
            {
                const int i = c.bi0 + k / nj, j = c.kj0 + k % nj;
                const BraPrim bp = load_bra_prim(c, i);
                ok = !(c.check && (bp.skip || !prim_survives(c, bp, j)));
            }
            const unsigned ball = __ballot_sync(0xffffffffu, ok);
            const int lane = tid & 31, warp = tid >> 5;
            __shared__ int wcount[C2_THREADS / 32];
            if(lane == 0)
                wcount[warp] = __popc(ball);
            __syncthreads();
            int base = 0;
            for(int w = 0; w < warp; w++)
                base += wcount[w];
            if(ok)
                surv[base + __popc(ball & ((1u << lane) - 1))] = k;
            if(tid == nth - 1)
            {
                int tot = 0;
                for(int w = 0; w < nth / 32; w++)
                    tot += wcount[w];
                s_cnt = tot;
            }
            __syncthreads();
            const int nsurv = s_cnt;
            for(int b0 = 0; b0 < nsurv; b0 += B)
            {
                const int nb = min(B, nsurv - b0);
                // set-up and Boys of the batch: one thread per primitive quartet
                if(tid < nb)
                {
                    const int kk = surv[b0 + tid];
                    const int i = c.bi0 + kk / nj, j = c.kj0 + kk % nj;
                    const BraPrim bp = load_bra_prim(c, i);
                    PrimSetup s;
                    prim_setup(c, bp, j, s);
                    double * cf = coef + tid * C2_NCOEF;
                    cf[K_XP0] = p.brastep_j ? s.PAx : s.PBx;
                    cf[K_XP1] = p.brastep_j ? s.PAy : s.PBy;
                    cf[K_XP2] = p.brastep_j ? s.PAz : s.PBz;
                    cf[K_XQ0] = p.ketstep_l ? s.QCx : s.QDx;
                    cf[K_XQ1] = p.ketstep_l ? s.QCy : s.QDy;
                    cf[K_XQ2] = p.ketstep_l ? s.QCz : s.QDz;
                    cf[K_AOP0] = s.aopPQx; cf[K_AOP1] = s.aopPQy; cf[K_AOP2] = s.aopPQz;
                    cf[K_AOQ0] = s.aoqPQx; cf[K_AOQ1] = s.aoqPQy; cf[K_AOQ2] = s.aoqPQz;
                    cf[K_AP] = s.a_over_p; cf[K_AQ] = s.a_over_q;
                    cf[K_O2P] = s.oo2p; cf[K_O2Q] = s.oo2q; cf[K_O2PQ] = s.oo2pq;
                    cf[K_W1] = s.c2a; cf[K_W2] = s.c2b; cf[K_W3] = s.c2c; cf[K_W4] = s.c2d;
                    double F[24];
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
                    double * w0 = wave + tid * W;           // wavefront 0 = block (0,0)
                    for(int n = 0; n <= L; n++)
                        w0[n] = F[n] * s.prefac;
                }
                __syncthreads();
                // (ss|ss) top (only when a tag's range starts at s on both sides), in order
                if(tid == 0)
                    for(int bb = 0; bb < nb; bb++)
                        for(int tg = 0; tg < p.ntag; tg++)
                            if(p.elo[tg] == 0 && p.flo[tg] == 0 && p.ehi[tg] >= 0)
                                acc[p.acc_off[tg]] += (tg == 0 ? 1.0 : coef[bb * C2_NCOEF + K_W1 + tg - 1]) * wave[bb * W];
                for(int sf = 1; sf <= p.smax; sf++)
                {
                    double * cur = wave + (sf % 3) * B * W;
                    const double * w1 = wave + ((sf + 2) % 3) * B * W;
                    const double * w2 = wave + ((sf + 1) % 3) * B * W;
                    for(int it = p.wstart[sf] + tid; it < p.wstart[sf + 1]; it += nth)
                    {
                        const int4 ia = __ldg(p.items + 2 * it);
                        const int4 ib = __ldg(p.items + 2 * it + 1);
                        const int x = ib.x & 3;
                        const bool ket = (ib.x >> 2) & 1;
                        const int nA = (ib.x >> 3) & 31, nB = (ib.x >> 8) & 255;
                        const int mlen = ib.x >> 16;
                        const int gE = ib.y & 0xffff, gF = ib.y >> 16;
                        for(int bb = 0; bb < nb; bb++)
                        {
                            const double * cf = coef + bb * C2_NCOEF;
                            const double X = cf[(ket ? K_XQ0 : K_XP0) + x];
                            const double Y = cf[(ket ? K_AOQ0 : K_AOP0) + x];
                            const double Z = cf[ket ? K_AQ : K_AP];
                            const double HA = (double)nA * cf[ket ? K_O2Q : K_O2P];
                            const double HB = (double)nB * cf[K_O2PQ];
                            const double * s1 = w1 + bb * W + ia.y;
                            const double * s2 = w2 + bb * W + ia.z;
                            const double * s3 = w2 + bb * W + ia.w;
                            double * d = cur + bb * W + ia.x;
                            for(int m = 0; m < mlen; m++)
                            {
                                double v = X * s1[m];
                                v = fma(Y, s1[m + 1], v);
                                if(ia.z >= 0)
                                    v = fma(HA, fma(Z, s2[m + 1], s2[m]), v);
                                if(ia.w >= 0)
                                    v = fma(HB, s3[m + 1], v);
                                d[m] = v;
                            }
                            // tops: added primitive quartet by primitive quartet, in order
                            if(ib.z)
                            {
                                const double v0 = d[0];
                                for(int tg = 0; tg < p.ntag; tg++)
                                    if((ib.z >> tg) & 1)
                                    {
                                        const int re = gE - c2_lev_off(p.elo[tg]);
                                        const int rf = gF - c2_lev_off(p.flo[tg]);
                                        acc[p.acc_off[tg] + re * p.acc_nf[tg] + rf] += (tg == 0 ? v0 : v0 * cf[K_W1 + tg - 1]);
                                    }
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            __syncthreads();      // s_cnt and wcount are reused by the next chunk
        }
        // ---------------- HRR ----------------
        double * L0 = sm + p.off_hrr;
        double * L1 = L0 + p.hrr_layer;
        double * o = a.out + off;
        const int * am = p.am;
        const int n1 = c2_nc(am[1]), n2 = c2_nc(am[2]), n3 = c2_nc(am[3]);
        for(int ti = 0; ti < p.ntarget; ti++)
        {
            const int * tt = p.tgt[ti];
            const int tg = p.tgt_tag[ti];
            const int klo = p.ketstep_l ? tt[2] : tt[3];
            const int ncol = c2_lev_off(tt[2] + tt[3] + 1) - c2_lev_off(klo);
            const int nbra = c2_nc(tt[0]) * c2_nc(tt[1]);
            const int nket = c2_nc(tt[2]) * c2_nc(tt[3]);
            double * mid = sm + p.off_hrr + 2 * p.hrr_layer;     // (ab | f) for all columns
            const int accb = p.acc_off[tg], accnf = p.acc_nf[tg];
            const int e0 = c2_lev_off(p.elo[tg]), f0 = c2_lev_off(p.flo[tg]), fk = c2_lev_off(klo);
            c2_hrr_side(ci, p.brastep_j, tt[0], tt[1], ncol, c.AB[0], c.AB[1], c.AB[2],
                        [&](int g, int col) { return acc[accb + (g - e0) * accnf + (fk + col - f0)]; },
                        [&](int r, int col, double v) { mid[r * ncol + col] = v; }, L0, L1);
            const int kl = c2_lev_off(klo);
            double * resd = res + p.res_off[ti];
            c2_hrr_side(ci, p.ketstep_l, tt[2], tt[3], nbra, c.CD[0], c.CD[1], c.CD[2],
                        [&](int g, int row) { return mid[row * ncol + (g - kl)]; },
                        [&](int r, int row, double v) {
                            if(p.deriv == 0)
                            {
                                // r indexes the ket (c,d) block, row the bra (a,b)
                                const int pa = row / n1, pb = row % n1, pc = r / n3, pd = r % n3;
                                const int oi = ((c2_index(ci, c2_lev_off(am[0]) + pa, p.ordering) * n1
                                                 + c2_index(ci, c2_lev_off(am[1]) + pb, p.ordering)) * n2
                                                + c2_index(ci, c2_lev_off(am[2]) + pc, p.ordering)) * n3
                                               + c2_index(ci, c2_lev_off(am[3]) + pd, p.ordering);
                                o[oi] = v;
                            }
                            else
                                resd[row * nket + r] = v;
                        }, L0, L1);
        }
        if(p.deriv == 1)
        {
            __syncthreads();
            const int n0 = c2_nc(am[0]);
            for(int idx = tid; idx < n0 * n1 * n2 * n3; idx += nth)
            {
                const int pd = idx % n3, pc = (idx / n3) % n2, pb = (idx / (n3 * n2)) % n1, pa = idx / (n3 * n2 * n1);
                const int gg[4] = {c2_lev_off(am[0]) + pa, c2_lev_off(am[1]) + pb, c2_lev_off(am[2]) + pc,
                                   c2_lev_off(am[3]) + pd};
                const int oi = ((c2_index(ci, gg[0], p.ordering) * n1 + c2_index(ci, gg[1], p.ordering)) * n2
                                + c2_index(ci, gg[2], p.ordering)) * n3 + c2_index(ci, gg[3], p.ordering);
                double g12[12];
                for(int ctr = 0; ctr < 4; ctr++)
                {
                    if(ctr == p.missing)
                        continue;
                    int tp = -1, tm = -1;
                    for(int t2 = 0; t2 < p.ntarget; t2++)
                    {
                        if(p.tgt[t2][ctr] == am[ctr] + 1) tp = t2;
                        if(p.tgt[t2][ctr] == am[ctr] - 1) tm = t2;
                    }
                    for(int x = 0; x < 3; x++)
                    {
                        int h[4] = {gg[0], gg[1], gg[2], gg[3]};
                        h[ctr] = ci[gg[ctr]].p1[x];
                        const int * ta = p.tgt[tp];
                        int r = ((ci[h[0]].pos * c2_nc(ta[1]) + ci[h[1]].pos) * c2_nc(ta[2]) + ci[h[2]].pos)
                                * c2_nc(ta[3]) + ci[h[3]].pos;
                        double v = res[p.res_off[tp] + r];
                        const int nx = ci[gg[ctr]].ijk[x];
                        if(nx > 0)
                        {
                            h[ctr] = ci[gg[ctr]].m1[x];
                            const int * tb = p.tgt[tm];
                            r = ((ci[h[0]].pos * c2_nc(tb[1]) + ci[h[1]].pos) * c2_nc(tb[2]) + ci[h[2]].pos)
                                * c2_nc(tb[3]) + ci[h[3]].pos;
                            v -= nx * res[p.res_off[tm] + r];
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
                        if(ctr == p.missing)
                            continue;
                        sm3 = first ? g12[ctr * 3 + x] : sm3 + g12[ctr * 3 + x];
                        first = false;
                    }
                    g12[p.missing * 3 + x] = -sm3;
                }
                for(int k = 0; k < 12; k++)
                    o[(size_t)oi * 12 + k] = g12[k];
            }
        }
        __syncthreads();
    }
}

namespace sb200 {

static int lo_h(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
static int nc2(int l) { return ((l + 1) * (l + 2)) / 2; }

static int c2_stepdir(int i, int j, int k)
{
    const int e[3] = {i, j, k};
    int mn = 1000;
    for(int x = 0; x < 3; x++)
        if(e[x] > 0 && e[x] < mn) mn = e[x];
    for(int x = 2; x >= 0; x--)
        if(e[x] == mn) return x;
    return -1;
}

struct C2Host
{
    bool ok = false;
    C2Params p;
    std::vector<int4> items;
    std::map<int, int4 *> dev_items;     // per device
};

static bool c2_build(const int am[4], int deriv, int forceB, C2Host & h)
{
    C2Params & p = h.p;
    memset(&p, 0, sizeof(p));
    memcpy(p.am, am, sizeof(p.am));
    p.deriv = deriv;
    p.missing = -1;
    if(deriv == 0)
    {
        p.ntarget = 1;
        memcpy(p.tgt[0], am, sizeof(p.am));
        p.ntag = 1;
    }
    else
    {
        const int mx = *std::max_element(am, am + 4);
        p.missing = (int)(std::find(am, am + 4, mx) - am);
        for(int c = 0; c < 4; c++)
        {
            if(c == p.missing) continue;
            memcpy(p.tgt[p.ntarget], am, sizeof(p.am));
            p.tgt[p.ntarget][c]++;
            p.tgt_tag[p.ntarget++] = c + 1;
            if(am[c] > 0)
            {
                memcpy(p.tgt[p.ntarget], am, sizeof(p.am));
                p.tgt[p.ntarget][c]--;
                p.tgt_tag[p.ntarget++] = 0;
            }
        }
        p.ntag = 5;
    }
    int hi = 0;
    for(int t = 1; t < p.ntarget; t++)
        if(std::lexicographical_compare(p.tgt[hi], p.tgt[hi] + 4, p.tgt[t], p.tgt[t] + 4))
            hi = t;
    p.brastep_j = p.tgt[hi][0] >= p.tgt[hi][1];
    p.ketstep_l = p.tgt[hi][2] >= p.tgt[hi][3];
    int E = 0, F = 0;
    for(int t = 0; t < p.ntarget; t++)
    {
        E = std::max(E, p.tgt[t][0] + p.tgt[t][1]);
        F = std::max(F, p.tgt[t][2] + p.tgt[t][3]);
    }
    if(E >= C2_MAXL || F >= C2_MAXL || E + F > C2_MAXS)
        return false;
    p.Emax = E;
    p.Fmax = F;
    p.L = E + F;
    const bool ket_first = F <= E;
    for(int tg = 0; tg < 5; tg++)
    {
        p.elo[tg] = 1000; p.ehi[tg] = -1; p.flo[tg] = 1000; p.fhi[tg] = -1;
    }
    for(int t = 0; t < p.ntarget; t++)
    {
        const int * tt = p.tgt[t];
        const int tg = p.tgt_tag[t];
        p.elo[tg] = std::min(p.elo[tg], p.brastep_j ? tt[0] : tt[1]);
        p.ehi[tg] = std::max(p.ehi[tg], tt[0] + tt[1]);
        p.flo[tg] = std::min(p.flo[tg], p.ketstep_l ? tt[2] : tt[3]);
        p.fhi[tg] = std::max(p.fhi[tg], tt[2] + tt[3]);
    }
    int off = 0;
    for(int tg = 0; tg < p.ntag; tg++)
    {
        p.acc_off[tg] = off;
        if(p.ehi[tg] < 0)
        {
            p.elo[tg] = p.flo[tg] = 1;
            p.ehi[tg] = p.fhi[tg] = 0;
            p.acc_nf[tg] = 0;
            continue;
        }
        p.acc_nf[tg] = lo_h(p.fhi[tg] + 1) - lo_h(p.flo[tg]);
        off += (lo_h(p.ehi[tg] + 1) - lo_h(p.elo[tg])) * p.acc_nf[tg];
    }
    p.acc_size = off;
    // auxiliary orders each block feeds (block level, conservative)
    int mneed[C2_MAXL][C2_MAXL];
    for(int e = 0; e < C2_MAXL; e++)
        for(int f = 0; f < C2_MAXL; f++)
            mneed[e][f] = -1;
    for(int tg = 0; tg < p.ntag; tg++)
        for(int e = p.elo[tg]; e <= p.ehi[tg]; e++)
            for(int f = p.flo[tg]; f <= p.fhi[tg]; f++)
                mneed[e][f] = std::max(mneed[e][f], 0);
    for(int s = E + F; s >= 1; s--)
        for(int e = std::min(E, s); e >= 0 && s - e <= F; e--)
        {
            const int f = s - e;
            const int m = mneed[e][f];
            if(m < 0)
                continue;
            const bool ket = f > 0 && (ket_first || e == 0);
            if(ket)
            {
                mneed[e][f - 1] = std::max(mneed[e][f - 1], m + 1);
                if(f >= 2) mneed[e][f - 2] = std::max(mneed[e][f - 2], m + 1);
                if(e >= 1) mneed[e - 1][f - 1] = std::max(mneed[e - 1][f - 1], m + 1);
            }
            else
            {
                mneed[e - 1][f] = std::max(mneed[e - 1][f], m + 1);
                if(e >= 2) mneed[e - 2][f] = std::max(mneed[e - 2][f], m + 1);
                if(f >= 1) mneed[e - 1][f - 1] = std::max(mneed[e - 1][f - 1], m + 1);
            }
        }
    mneed[0][0] = std::max(mneed[0][0], 0);
    if(mneed[0][0] > p.L)
        return false;
    // block offsets inside a wavefront buffer; (0,0) holds m = 0..L
    int boff[C2_MAXL][C2_MAXL];
    p.wsize = p.L + 1;
    for(int s = 1; s <= E + F; s++)
    {
        int o = 0;
        for(int e = std::max(0, s - F); e <= std::min(E, s); e++)
        {
            const int f = s - e;
            boff[e][f] = o;
            if(mneed[e][f] >= 0)
                o += nc2(e) * nc2(f) * (mneed[e][f] + 1);
        }
        p.wsize = std::max(p.wsize, o);
    }
    boff[0][0] = 0;
    auto slot = [&](int e, int f, int ge, int gf) {   // offset of the m = 0 slot
        const int pe = ge - lo_h(e), pf = gf - lo_h(f);
        return boff[e][f] + (pe * nc2(f) + pf) * (mneed[e][f] + 1);
    };
    auto flat = [](int i, int j, int k) { return ci_flat(i, j, k); };
    h.items.clear();
    p.smax = 0;
    for(int s = 1; s <= E + F; s++)
    {
        p.wstart[s] = (int)h.items.size() / 2;
        for(int e = std::max(0, s - F); e <= std::min(E, s); e++)
        {
            const int f = s - e;
            if(mneed[e][f] < 0)
                continue;
            p.smax = s;
            const bool ket = f > 0 && (ket_first || e == 0);
            for(int ie = e; ie >= 0; ie--)
                for(int je = e - ie; je >= 0; je--)
                    for(int i_f = f; i_f >= 0; i_f--)
                        for(int jf = f - i_f; jf >= 0; jf--)
                        {
                            const int ke = e - ie - je, kf = f - i_f - jf;
                            const int gE = flat(ie, je, ke), gF = flat(i_f, jf, kf);
                            const int E3[3] = {ie, je, ke}, F3[3] = {i_f, jf, kf};
                            int4 ia, ib;
                            int x, nA, nB;
                            ia.x = slot(e, f, gE, gF);
                            if(ket)
                            {
                                x = c2_stepdir(i_f, jf, kf);
                                int f1[3] = {F3[0], F3[1], F3[2]}; f1[x]--;
                                const int gF1 = flat(f1[0], f1[1], f1[2]);
                                ia.y = slot(e, f - 1, gE, gF1);
                                nA = F3[x] - 1;
                                if(F3[x] >= 2)
                                {
                                    int f2[3] = {F3[0], F3[1], F3[2]}; f2[x] -= 2;
                                    ia.z = slot(e, f - 2, gE, flat(f2[0], f2[1], f2[2]));
                                }
                                else
                                    ia.z = -1;
                                nB = E3[x];
                                if(E3[x] >= 1)
                                {
                                    int e1[3] = {E3[0], E3[1], E3[2]}; e1[x]--;
                                    ia.w = slot(e - 1, f - 1, flat(e1[0], e1[1], e1[2]), gF1);
                                }
                                else
                                    ia.w = -1;
                            }
                            else
                            {
                                x = c2_stepdir(ie, je, ke);
                                int e1[3] = {E3[0], E3[1], E3[2]}; e1[x]--;
                                const int gE1 = flat(e1[0], e1[1], e1[2]);
                                ia.y = slot(e - 1, f, gE1, gF);
                                nA = E3[x] - 1;
                                if(E3[x] >= 2)
                                {
                                    int e2[3] = {E3[0], E3[1], E3[2]}; e2[x] -= 2;
                                    ia.z = slot(e - 2, f, flat(e2[0], e2[1], e2[2]), gF);
                                }
                                else
                                    ia.z = -1;
                                nB = F3[x];
                                if(F3[x] >= 1)
                                {
                                    int f1[3] = {F3[0], F3[1], F3[2]}; f1[x]--;
                                    ia.w = slot(e - 1, f - 1, gE1, flat(f1[0], f1[1], f1[2]));
                                }
                                else
                                    ia.w = -1;
                            }
                            int mask = 0;
                            for(int tg = 0; tg < p.ntag; tg++)
                                if(e >= p.elo[tg] && e <= p.ehi[tg] && f >= p.flo[tg] && f <= p.fhi[tg])
                                    mask |= 1 << tg;
                            ib.x = x | ((ket ? 1 : 0) << 2) | (std::max(nA, 0) << 3) | (nB << 8)
                                 | ((mneed[e][f] + 1) << 16);
                            ib.y = gE | (gF << 16);
                            ib.z = mask;
                            ib.w = 0;
                            h.items.push_back(ia);
                            h.items.push_back(ib);
                        }
        }
    }
    p.wstart[E + F + 1] = (int)h.items.size() / 2;
    for(int s = p.smax + 1; s <= E + F + 1; s++)
        p.wstart[s] = p.wstart[E + F + 1];
    // HRR layer size: the largest layer of either side, over targets
    int hl = 0, midmax = 0;
    for(int t = 0; t < p.ntarget; t++)
    {
        const int * tt = p.tgt[t];
        const int klo = p.ketstep_l ? tt[2] : tt[3];
        const int ncol = lo_h(tt[2] + tt[3] + 1) - lo_h(klo);
        const int nbra = nc2(tt[0]) * nc2(tt[1]);
        auto side = [&](int right, int ta, int tb, int ncl) {
            const int lt = ta + tb, lo = right ? ta : tb, slm = right ? tb : ta;
            int mx = (lo_h(lt + 1) - lo_h(lo)) * ncl;
            for(int sl = 1; sl <= slm; sl++)
                mx = std::max(mx, (lo_h(lt - sl + 1) - lo_h(lo)) * nc2(sl) * ncl);
            return mx;
        };
        hl = std::max(hl, side(p.brastep_j, tt[0], tt[1], ncol));
        hl = std::max(hl, side(p.ketstep_l, tt[2], tt[3], nbra));
        midmax = std::max(midmax, nbra * ncol);
    }
    p.hrr_layer = hl;
    // shared memory: [waves | acc | coef | surv] and the HRR [L0 | L1 | mid] reuses waves
    p.B = forceB > 0 ? forceB : 4;
    for(;;)
    {
        const int waves = 3 * p.B * p.wsize;
        p.off_acc = std::max(waves, 2 * hl + midmax);
        p.off_coef = p.off_acc + p.acc_size;
        p.off_surv = p.off_coef + p.B * C2_NCOEF;
        p.smem_doubles = p.off_surv + C2_THREADS / 2 + 1;
        if(p.smem_doubles * 8 <= 200 * 1024 || p.B == 1)
            break;
        p.B /= 2;
    }
    p.off_hrr = 0;
    p.ordering = 0;
    int ro = 0;
    for(int t = 0; t < p.ntarget; t++)
    {
        p.res_off[t] = ro;
        if(deriv)
            ro += nc2(p.tgt[t][0]) * nc2(p.tgt[t][1]) * nc2(p.tgt[t][2]) * nc2(p.tgt[t][3]);
    }
    p.res_size = std::max(ro, 1);
    return p.smem_doubles * 8 <= 200 * 1024;
}

static std::mutex g_c2_mutex;
static std::map<std::array<int, 6>, C2Host> g_c2;

static C2Host * c2_get(const int am[4], int deriv, int forceB = 0)
{
    std::lock_guard<std::mutex> lk(g_c2_mutex);
    std::array<int, 6> key = {am[0], am[1], am[2], am[3], deriv, forceB};
    auto it = g_c2.find(key);
    if(it == g_c2.end())
    {
        C2Host h;
        h.ok = c2_build(am, deriv, forceB, h);
        if(h.ok && forceB > 0 && h.p.B != forceB)
            h.ok = false;          // that batch size does not fit shared memory
        it = g_c2.emplace(key, std::move(h)).first;
    }
    return &it->second;
}

bool coop2_supported(const int am[4], int deriv, int forceB)
{
    return c2_get(am, deriv, forceB)->ok;
}

int launch_coop2(KernArgs & a, const int req[4], int deriv, int mode, int prec, cudaStream_t stream,
                 int forceB)
{
    C2Host * h = c2_get(req, deriv, forceB);
    if(!h->ok)
    {
        set_error("class outside the cooperative kernel's range");
        return SIMINT_B200_ERR_CLASS;
    }
    upload_cart_info();
    int dev = 0;
    cudaGetDevice(&dev);
    C2Params p = h->p;
    {
        std::lock_guard<std::mutex> lk(g_c2_mutex);
        auto it = h->dev_items.find(dev);
        if(it == h->dev_items.end())
        {
            int4 * d = nullptr;
            if(cudaMalloc(&d, std::max<size_t>(1, h->items.size()) * sizeof(int4)) != cudaSuccess)
            {
                cudaGetLastError();
                set_error("out of device memory for cooperative-kernel tables");
                return SIMINT_B200_ERR_CUDA;
            }
            cudaMemcpy(d, h->items.data(), h->items.size() * sizeof(int4), cudaMemcpyHostToDevice);
            it = h->dev_items.emplace(dev, d).first;
        }
        p.items = it->second;
    }
    p.ordering = ordering();
    a.swapB = a.swapK = a.pq = 0;
    a.oidx = nullptr;
    const size_t smem = (size_t)p.smem_doubles * sizeof(double) + 256;
    static bool attr[3][2] = {{false, false}, {false, false}, {false, false}};
    const int mixed = 0;   // the FP32 variant of this kernel is not built yet
    (void)prec;
    if(!attr[mode][mixed])
    {
        if(mode == 0) cudaFuncSetAttribute(k_coop2<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024 + 256);
        if(mode == 1) cudaFuncSetAttribute(k_coop2<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024 + 256);
        if(mode == 2) cudaFuncSetAttribute(k_coop2<2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024 + 256);
        attr[mode][mixed] = true;
    }
    const int per_sm = std::max(1, std::min(4, (int)((220 * 1024) / smem)));
    long long grid = std::min<long long>(a.ntask, 148LL * per_sm);
    grid = std::max<long long>(grid, 1);
    Workspace & w = workspace();
    const size_t scratch = (size_t)grid * p.res_size * sizeof(double);
    if(!w.dscratch.reserve(scratch))
    {
        set_error("out of device memory for cooperative-kernel scratch");
        return SIMINT_B200_ERR_CUDA;
    }
    if(mode == 0)
        k_coop2<0, false><<<(unsigned)grid, C2_THREADS, smem, stream>>>(a, p, (double *)w.dscratch.ptr);
    else if(mode == 1)
        k_coop2<1, false><<<(unsigned)grid, C2_THREADS, smem, stream>>>(a, p, (double *)w.dscratch.ptr);
    else
        k_coop2<2, false><<<(unsigned)grid, C2_THREADS, smem, stream>>>(a, p, (double *)w.dscratch.ptr);
    count_launch(1);
    return 0;
}

} // namespace sb200
