// CTA-cooperative ERI kernel, table-driven: large AM classes, deriv 0/1.
//
// One CTA computes one shell quartet at a time.  Per class the host builds
// (once) a table of work items: one item per Cartesian pair (e-cart, f-cart)
// of every needed (e|f) block of the dense Obara-Saika VRR, holding the
// shared-memory offsets of its sources, the recursion direction and the
// integer factors of the reference's 8-term step (Makowski.hpp:87-242,
// centre order OSTEI_VRR_Algorithm_Base.cpp:449-469).  Blocks are grouped
// into anti-diagonal wavefronts s = e+f (a block depends only on s-1 and
// s-2) and each block keeps only the auxiliary orders m it really feeds.
// An item is one auxiliary order m of one element, so the (independent)
// orders of an element spread over threads; items keep the natural order so
// neighbouring threads touch neighbouring shared-memory words.
//
// Surviving primitive quartets (the reference's screening tests) are
// compacted in order; their set-up and Boys values are computed 16 at a time
// by 16 threads into shared memory, then processed B at a time: a thread
// owns an item and runs it for all B primitive quartets, so one
// __syncthreads per wavefront serves B primitive quartets.
// Per primitive quartet the step coefficients are stored as six
// (direction, side) combos of [X, Y, Z, 1/2s] so an item reads its four
// coefficients with two 16-byte loads.  Top quartets are summed into
// per-tag accumulators by the owning thread in primitive order (deriv
// weights of OSTEIDeriv1_Writer.cpp:53-94).  After the primitive loop the
// HRR (OSTEI_HRR_Algorithm_Base.cpp:160-283) runs level by level in shared
// memory: the first layer reads the accumulators, the last layer writes its
// destination directly; deriv=1 components are formed by translational
// invariance (OSTEIDeriv1_Writer.cpp:334-537).
//
// Variants: 256, 128 or 64 threads per CTA, B = 1, 2, 4 or 8 (variant codes
// 20+B, 40+B and 60+B).

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

#include "coop2.cuh"

// Coefficient combo of one prepared primitive quartet: X, Y, Z, 1/2s.
__device__ __forceinline__ void c2_combo(const double * cf, int combo, double & X, double & Y, double & Z, double & O)
{
    const double2 XY = *(const double2 *)(cf + 4 * combo);
    const double2 ZO = *(const double2 *)(cf + 4 * combo + 2);
    X = XY.x; Y = XY.y; Z = ZO.x; O = ZO.y;
}

__device__ __forceinline__ void c2_combo(const float * cf, int combo, float & X, float & Y, float & Z, float & O)
{
    const float4 q = *(const float4 *)(cf + 4 * combo);
    X = q.x; Y = q.y; Z = q.z; O = q.w;
}

// One VRR unit (one element, one auxiliary order) for NB primitive quartets.
template<typename T, int NB>
__device__ __forceinline__ void c2_unit(const int4 q, const T * __restrict__ w1, const T * __restrict__ w2,
                                        int W, const T * const * cft, T * v)
{
    const int o1 = (int)((unsigned)q.x >> 16);
    const int o2 = q.y & 0xffff, o3 = (int)((unsigned)q.y >> 16);
    const int combo = (q.z >> 16) & 7;
    const bool has2 = (q.z >> 24) & 1, has3 = (q.z >> 25) & 1;
    T dA, dB;
    c2_small(q.w & 15, dA);
    c2_small((q.w >> 4) & 15, dB);
    #pragma unroll
    for(int bb = 0; bb < NB; bb++)
    {
        T X, Y, Z, O;
        c2_combo(cft[bb], combo, X, Y, Z, O);
        const T * s1 = w1 + bb * W + o1;
        const T * s2 = w2 + bb * W + o2;
        const T * s3 = w2 + bb * W + o3;
        T r = X * s1[0];
        r = fma(Y, s1[1], r);
        if(has2)
            r = fma(dA * O, fma(Z, s2[1], s2[0]), r);
        if(has3)
            r = fma(dB * cft[bb][K_O2PQ], s3[1], r);
        v[bb] = r;
    }
}

// Store a unit's NB results and add its tops to the FP64 accumulators in
// primitive order.
template<typename T, int NB, int DERIV>
__device__ __forceinline__ void c2_unit_store(const C2Params & p, const int4 q, T * __restrict__ cur, int W,
                                              const double * const * cfd, const T * v, double * __restrict__ acc)
{
    const int dsto = q.x & 0xffff;
    #pragma unroll
    for(int bb = 0; bb < NB; bb++)
        cur[bb * W + dsto] = v[bb];
    const int acc0 = q.z & 0xffff;
    if(acc0 != 0xffff)
    {
        double a = acc[acc0];
        #pragma unroll
        for(int bb = 0; bb < NB; bb++)
            a += (double)v[bb];
        acc[acc0] = a;
    }
    if(DERIV)
    {
        const int tmask = ((q.z >> 26) & 15) << 1;
        if(tmask)
        {
            const int gE = (q.w >> 8) & 1023, gF = (q.w >> 18) & 1023;
            for(int tg = 1; tg < p.ntag; tg++)
                if((tmask >> tg) & 1)
                {
                    const int re = gE - c2_lev_off(p.elo[tg]);
                    const int rf = gF - c2_lev_off(p.flo[tg]);
                    double & a = acc[p.acc_off[tg] + re * p.acc_nf[tg] + rf];
                    #pragma unroll
                    for(int bb = 0; bb < NB; bb++)
                        a += (double)v[bb] * cfd[bb][K_W1 + tg - 1];
                }
        }
    }
}

// The wavefronts s >= 1 of NB primitive quartets (prepared slots
// slot[0..NB)) in type T.  A thread takes units it = tid, tid + NT, ... of
// each wavefront, two at a time, and runs each for all NB primitive
// quartets as independent chains; the tops go to the FP64 accumulators in
// slot order.
template<typename T, int NT, int DERIV, int NB>
__device__ __forceinline__ void c2_waves(const C2Params & p, T * __restrict__ wave, int cap, int W,
                                         const double * __restrict__ prep, int PS, int off32,
                                         const int * __restrict__ slot, double * __restrict__ acc)
{
    const int tid = threadIdx.x;
    const double * cfd[NB];
    const T * cft[NB];
    #pragma unroll
    for(int bb = 0; bb < NB; bb++)
    {
        cfd[bb] = prep + slot[bb] * PS;
        cft[bb] = (const T *)(cfd[bb] + off32);
    }
    // the units of the next iteration are loaded one iteration (or one
    // barrier) ahead: the tables of large classes live in L2, not L1
    int4 q0n = make_int4(0, 0, 0, 0), q1n = q0n;
    {
        const int it0 = p.wstart[1] + tid, end1 = p.wstart[2];
        if(it0 < end1)
        {
            q0n = __ldg(&p.items[it0]);
            q1n = it0 + NT < end1 ? __ldg(&p.items[it0 + NT]) : q0n;
        }
    }
    for(int sf = 1; sf <= p.smax; sf++)
    {
        T * cur = wave + (sf % 3) * cap * W;
        const T * w1 = wave + ((sf + 2) % 3) * cap * W;
        const T * w2 = wave + ((sf + 1) % 3) * cap * W;
        const int end = p.wstart[sf + 1];
        for(int it = p.wstart[sf] + tid; it < end; it += 2 * NT)
        {
            const bool two = it + NT < end;
            const int4 q0 = q0n;
            const int4 q1 = q1n;
            {
                // prefetch: the next iteration of this wavefront, or the
                // first of the next wavefront
                int nx = it + 2 * NT, ne = end;
                if(nx >= end && sf < p.smax)
                {
                    nx = p.wstart[sf + 1] + tid;
                    ne = p.wstart[sf + 2];
                }
                if(nx < ne)
                {
                    q0n = __ldg(&p.items[nx]);
                    q1n = nx + NT < ne ? __ldg(&p.items[nx + NT]) : q0n;
                }
            }
            T v0[NB], v1[NB];
            c2_unit<T, NB>(q0, w1, w2, W, cft, v0);
            c2_unit<T, NB>(q1, w1, w2, W, cft, v1);
            c2_unit_store<T, NB, DERIV>(p, q0, cur, W, cfd, v0, acc);
            if(two)
                c2_unit_store<T, NB, DERIV>(p, q1, cur, W, cfd, v1, acc);
        }
        if(p.wstart[sf] + tid >= end && sf < p.smax)
        {
            // no unit of this wavefront: fetch the first of the next one here
            const int nx = p.wstart[sf + 1] + tid, ne = p.wstart[sf + 2];
            if(nx < ne)
            {
                q0n = __ldg(&p.items[nx]);
                q1n = nx + NT < ne ? __ldg(&p.items[nx + NT]) : q0n;
            }
        }
        __syncthreads();
    }
}

// The VRR of nb primitive quartets (prepared slots slot[0..nb)) in type T:
// block (0,0) from the Boys values, the (ss|ss) tops, then the wavefronts.
// wave holds 3 wavefronts x cap batch entries x W values of T.
template<typename T, int NT, int DERIV, int MAXB>
__device__ __forceinline__ void c2_batch(const C2Params & p, T * __restrict__ wave, int cap, int W,
                                         const double * __restrict__ prep, int PS, int off32,
                                         const int * __restrict__ slot, int nb, double * __restrict__ acc)
{
    const int tid = threadIdx.x;
    const int L = p.L;
    for(int k2 = tid; k2 < nb * (L + 1); k2 += NT)
    {
        const int bb = k2 / (L + 1), n = k2 - bb * (L + 1);
        wave[bb * W + n] = (T)prep[slot[bb] * PS + C2_NCOEF + n];
    }
    // (ss|ss) top (only when a tag's range starts at s on both sides), in order
    if(tid == 0)
        for(int bb = 0; bb < nb; bb++)
        {
            const double * cf = prep + slot[bb] * PS;
            for(int tg = 0; tg < (DERIV ? p.ntag : 1); tg++)
                if(p.elo[tg] == 0 && p.flo[tg] == 0 && p.ehi[tg] >= 0)
                    acc[p.acc_off[tg]] += (tg == 0 ? 1.0 : cf[K_W1 + tg - 1]) * cf[C2_NCOEF];
        }
    __syncthreads();
    switch(nb)
    {
        case 1: c2_waves<T, NT, DERIV, 1>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
        case 2: if constexpr(MAXB >= 2) c2_waves<T, NT, DERIV, 2>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
        case 3: if constexpr(MAXB >= 3) c2_waves<T, NT, DERIV, 3>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
        case 4: if constexpr(MAXB >= 4) c2_waves<T, NT, DERIV, 4>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
        case 5: if constexpr(MAXB >= 5) c2_waves<T, NT, DERIV, 5>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
        case 6: if constexpr(MAXB >= 6) c2_waves<T, NT, DERIV, 6>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
        case 7: if constexpr(MAXB >= 7) c2_waves<T, NT, DERIV, 7>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
        default: if constexpr(MAXB >= 8) c2_waves<T, NT, DERIV, 8>(p, wave, cap, W, prep, PS, off32, slot, acc); break;
    }
}

template<int MODE, int NT, int DERIV, bool MIXED>
__global__ void __launch_bounds__(NT, NT == 64 ? 8 : (NT == 128 ? 4 : 2)) k_coop2(const KernArgs a, const C2Params p,
                                                                 double * __restrict__ gres)
{
    extern __shared__ __align__(16) double sm[];
    __shared__ CartInfo ci[CI_NCART];
    __shared__ int s_cnt;
    __shared__ int wcount[NT / 32];
    __shared__ int obra[C2_MAXN], oket[C2_MAXN];
    __shared__ int s_slot[C2_SETUP];
    __shared__ int s_nhigh;
    const int tid = threadIdx.x;
    for(int k = tid; k < CI_NCART; k += NT)
        ci[k] = c_cartinfo[k];
    __syncthreads();
    const int * am = p.am;
    const int n0 = c2_nc(am[0]), n1 = c2_nc(am[1]), n2 = c2_nc(am[2]), n3 = c2_nc(am[3]);
    // output offsets of the (a b) rows and (c d) columns of the requested class
    for(int k = tid; k < n0 * n1; k += NT)
        obra[k] = (c2_index(ci, c2_lev_off(am[0]) + k / n1, p.ordering) * n1
                   + c2_index(ci, c2_lev_off(am[1]) + k % n1, p.ordering)) * (n2 * n3);
    for(int k = tid; k < n2 * n3; k += NT)
        oket[k] = c2_index(ci, c2_lev_off(am[2]) + k / n3, p.ordering) * n3
                + c2_index(ci, c2_lev_off(am[3]) + k % n3, p.ordering);
    const int B = p.B, L = p.L, W = p.wsize, PS = p.prep_stride;
    double * wave = sm;
    double * acc = sm + p.off_acc;
    double * prep = sm + p.off_prep;
    int * surv = (int *)(sm + p.off_surv);
    double * res = gres + (size_t)blockIdx.x * p.res_size;
    __syncthreads();

    __shared__ long long s_qslot;
    long long t = 0;
    for(long long slot = blockIdx.x; cta_next_task(a, slot, t, &s_qslot); slot += gridDim.x)
    {
        int iP, iQ;
        long long off;
        task_of<MODE>(a, t, iP, iQ, off);
        QuartetCtx c;
        make_ctx(a, iP, iQ, c);
        if(MIXED)
        {
            c.gL = L;
            c.gamp = hrr_amp(c, min(am[0], am[1]), min(am[2], am[3]));
            // the gate bounds the error of one integral: each of the shell
            // quartet's primitive quartets may take gate / (their number)
            c.gate = a.gate / (double)max(1, (c.bi1 - c.bi0) * (c.kj1 - c.kj0));
        }
        for(int k = tid; k < p.acc_size; k += NT)
            acc[k] = 0.0;
        const int ni = c.bi1 - c.bi0, nj = c.kj1 - c.kj0;
        const int ncand = ni * nj;
        // k / nj as a multiply-high, exact while k * nj < 2^32; a division
        // otherwise (contractions of thousands of primitive pairs)
        const unsigned long long njinv = nj > 0 ? (1ull << 32) / (unsigned)nj + 1ull : 0ull;
        const bool fastdiv = (long long)ncand * nj < (1LL << 32);
        for(int k0 = 0; k0 < ncand; k0 += NT)
        {
            // ordered compaction of the surviving primitive quartets k0..k0+NT
            if(tid == 0)
                s_cnt = 0;
            const int k = k0 + tid;
            bool ok = false;
            if(k < ncand)
            {
                const int kq = fastdiv ? (int)(((unsigned long long)k * njinv) >> 32) : k / nj;
                const int i = c.bi0 + kq, j = c.kj0 + (k - kq * nj);
                const BraPrim bp = load_bra_prim(c, i);
                ok = !(c.check && (bp.skip || !prim_survives(c, bp, j)));
            }
            const unsigned ball = __ballot_sync(0xffffffffu, ok);
            const int lane = tid & 31, warp = tid >> 5;
            if(lane == 0)
                wcount[warp] = __popc(ball);
            __syncthreads();
            int base = 0;
            for(int w = 0; w < warp; w++)
                base += wcount[w];
            if(ok)
                surv[base + __popc(ball & ((1u << lane) - 1))] = k;
            if(tid == NT - 1)
            {
                int tot = 0;
                for(int w = 0; w < NT / 32; w++)
                    tot += wcount[w];
                s_cnt = tot;
            }
            __syncthreads();
            const int nsurv = s_cnt;
            for(int g0 = 0; g0 < nsurv; g0 += C2_SETUP)
            {
                const int ng = min(C2_SETUP, nsurv - g0);
                // set-up and Boys of up to C2_SETUP primitive quartets in parallel
                bool low = false;
                if(tid < ng)
                {
                    const int kk = surv[g0 + tid];
                    const int kq = fastdiv ? (int)(((unsigned long long)kk * njinv) >> 32) : kk / nj;
                    const int i = c.bi0 + kq, j = c.kj0 + (kk - kq * nj);
                    const BraPrim bp = load_bra_prim(c, i);
                    PrimSetup s;
                    prim_setup(c, bp, j, s);
                    double * cf = prep + tid * PS;
                    const double XP[3] = {p.brastep_j ? s.PAx : s.PBx, p.brastep_j ? s.PAy : s.PBy,
                                          p.brastep_j ? s.PAz : s.PBz};
                    const double XQ[3] = {p.ketstep_l ? s.QCx : s.QDx, p.ketstep_l ? s.QCy : s.QDy,
                                          p.ketstep_l ? s.QCz : s.QDz};
                    const double YP[3] = {s.aopPQx, s.aopPQy, s.aopPQz};
                    const double YQ[3] = {s.aoqPQx, s.aoqPQy, s.aoqPQz};
                    #pragma unroll
                    for(int x = 0; x < 3; x++)
                    {
                        double * b4 = cf + 4 * x;
                        b4[0] = XP[x]; b4[1] = YP[x]; b4[2] = s.a_over_p; b4[3] = s.oo2p;
                        double * k4 = cf + 12 + 4 * x;
                        k4[0] = XQ[x]; k4[1] = YQ[x]; k4[2] = s.a_over_q; k4[3] = s.oo2q;
                    }
                    cf[K_O2PQ] = s.oo2pq;
                    cf[K_W1 + 0] = s.c2a; cf[K_W1 + 1] = s.c2b; cf[K_W1 + 2] = s.c2c; cf[K_W1 + 3] = s.c2d;
                    c2_boys(c.boys, s.T, L, s.prefac, cf + C2_NCOEF);
                    if(MIXED)
                    {
                        low = s.lowprec;
                        float * f32 = (float *)(cf + p.off32);
                        #pragma unroll
                        for(int k2 = 0; k2 <= K_O2PQ; k2++)
                            f32[k2] = (float)cf[k2];
                    }
                }
                if(MIXED)
                {
                    // FP64 primitive quartets first, then the FP32 ones, each in order
                    if(tid < 32)
                    {
                        const unsigned lowm = __ballot_sync(0xffffffffu, low);
                        const unsigned valid = ng >= 32 ? 0xffffffffu : ((1u << ng) - 1u);
                        const unsigned lt = (1u << (tid & 31)) - 1u;
                        const int nhigh = __popc(valid & ~lowm);
                        if(tid < ng)
                            s_slot[low ? nhigh + __popc(lowm & valid & lt) : __popc(valid & ~lowm & lt)] = tid;
                        if(tid == 0)
                            s_nhigh = nhigh;
                    }
                }
                else if(tid < ng)
                    s_slot[tid] = tid;
                __syncthreads();
                const int nhigh = MIXED ? s_nhigh : ng;
                if(MIXED && tid == 0 && ng > nhigh && a.fp32_count)
                    atomicAdd(a.fp32_count, (unsigned long long)(ng - nhigh));
                // batches of up to 8 in FP64 (codes 2x, 4x, 6x: B = x); the
                // 8-way batch dispatch also made the 2-wide batches of the
                // largest classes 5-8 % faster than a 4-way one (measured)
                for(int b0 = 0; b0 < nhigh; b0 += B)
                    c2_batch<double, NT, DERIV, 8>(p, wave, B, W, prep, PS, 0, s_slot + b0, min(B, nhigh - b0), acc);
                if constexpr(MIXED)
                {
                    // FP32 batches of 2B (the same bytes), at most 8
                    const int FB = min(2 * B, 8);
                    for(int b0 = nhigh; b0 < ng; b0 += FB)
                        c2_batch<float, NT, DERIV, 8>(p, (float *)wave, 2 * B, W, prep, PS, p.off32, s_slot + b0,
                                                      min(FB, ng - b0), acc);
                }
            }
            __syncthreads();      // surv, s_cnt and wcount are reused by the next chunk
        }
        // ---------------- HRR ----------------
        double * LA = sm + p.off_hrr_b;
        double * LB = LA + p.hrr_layer;
        double * mid = sm + p.off_hrr_mid;          // (ab | f) for all columns
        double * o = a.out + off;
        for(int ti = 0; ti < p.ntarget; ti++)
        {
            const int * tt = p.tgt[ti];
            const int tg = p.tgt_tag[ti];
            const int klo = p.ketstep_l ? tt[2] : tt[3];
            const int ncol = c2_lev_off(tt[2] + tt[3] + 1) - c2_lev_off(klo);
            const int nbra = c2_nc(tt[0]) * c2_nc(tt[1]);
            const int nket = c2_nc(tt[2]) * c2_nc(tt[3]);
            const int accb = p.acc_off[tg], accnf = p.acc_nf[tg];
            const int e0 = c2_lev_off(p.elo[tg]), f0 = c2_lev_off(p.flo[tg]), fk = c2_lev_off(klo);
            c2_hrr_side<NT>(p.brastep_j, p.hrr_nl[ti][0], ncol, p.hrr_rows + p.hrr_base[ti][0],
                            p.hrr_loff[ti][0], c.AB[0], c.AB[1], c.AB[2],
                            [&](int g, int col) { return acc[accb + (g - e0) * accnf + (fk + col - f0)]; },
                            [&](int r, int col, double v) { mid[r * ncol + col] = v; }, LA, LB);
            const int kl = c2_lev_off(klo);
            double * resd = res + p.res_off[ti];
            if(DERIV == 0)
                c2_hrr_side<NT>(p.ketstep_l, p.hrr_nl[ti][1], nbra, p.hrr_rows + p.hrr_base[ti][1],
                                p.hrr_loff[ti][1], c.CD[0], c.CD[1], c.CD[2],
                                [&](int g, int row) { return mid[row * ncol + (g - kl)]; },
                                [&](int r, int row, double v) { o[obra[row] + oket[r]] = v; }, LA, LB);
            else
                c2_hrr_side<NT>(p.ketstep_l, p.hrr_nl[ti][1], nbra, p.hrr_rows + p.hrr_base[ti][1],
                                p.hrr_loff[ti][1], c.CD[0], c.CD[1], c.CD[2],
                                [&](int g, int row) { return mid[row * ncol + (g - kl)]; },
                                [&](int r, int row, double v) { resd[row * nket + r] = v; }, LA, LB);
        }
        if(DERIV == 1)
        {
            __syncthreads();
            for(int idx = tid; idx < n0 * n1 * n2 * n3; idx += NT)
            {
                const int pd = idx % n3, pc = (idx / n3) % n2, pb = (idx / (n3 * n2)) % n1, pa = idx / (n3 * n2 * n1);
                const int gg[4] = {c2_lev_off(am[0]) + pa, c2_lev_off(am[1]) + pb, c2_lev_off(am[2]) + pc,
                                   c2_lev_off(am[3]) + pd};
                const int oi = obra[pa * n1 + pb] + oket[pc * n3 + pd];
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

static bool c2_is_variant(int v)
{
    return v == 21 || v == 22 || v == 24 || v == 28 || v == 41 || v == 42 || v == 44 || v == 48 || v == 61 || v == 62
        || v == 64 || v == 68;
}
static int c2_threads(int v) { return v >= 60 ? 64 : (v >= 40 ? 128 : 256); }

struct C2ItemHost
{
    int dst, s1, s2, s3, combo, mlen, acc0, mask, gE, gF, nA, nB;
};

struct C2Host
{
    bool ok = false;
    int nthreads = 256;
    C2Params p;
    std::vector<C2Item> items;
    std::vector<int2> hrr;                 // HRR row tables
    std::map<int, char *> dev_tables;      // per device: items then HRR rows
};

// HRR row tables of every target and side (see c2_hrr_side).
static bool c2_build_hrr(C2Params & p, std::vector<int2> & rows)
{
    const std::vector<CartInfo> ct = cart_table_host();
    rows.clear();
    for(int t = 0; t < p.ntarget; t++)
        for(int side = 0; side < 2; side++)
        {
            const int * tt = p.tgt[t];
            const int right = side == 0 ? p.brastep_j : p.ketstep_l;
            const int ta = side == 0 ? tt[0] : tt[2], tb = side == 0 ? tt[1] : tt[3];
            const int lt = ta + tb, lo = right ? ta : tb, slm = right ? tb : ta, nbb = nc2(tb);
            if(slm > 5)
                return false;
            p.hrr_base[t][side] = (int)rows.size();
            p.hrr_nl[t][side] = slm;
            if(slm == 0)
            {
                const int nr = nc2(ta) * nbb;
                for(int r = 0; r < nr; r++)
                    rows.push_back(make_int2(lo_h(lt) + r, 0));
                p.hrr_loff[t][side][0] = nr;
                continue;
            }
            p.hrr_loff[t][side][0] = 0;
            int cnt = 0;
            for(int sl = 1; sl <= slm; sl++)
            {
                const int ngt = lo_h(lt - sl + 1) - lo_h(lo);
                const int nsl = nc2(sl), nslm = nc2(sl - 1);
                for(int r = 0; r < ngt * nsl; r++)
                {
                    const int ps = r % nsl, itq = r / nsl;
                    const int it = lo_h(lo) + itq, is = lo_h(sl) + ps;
                    const int x = ct[is].dir;
                    const int ism = ct[is].m1[x];
                    const int itp = ct[it].p1[x];
                    const int pm = ct[ism].pos;
                    int A, B;
                    if(sl == 1)
                    {
                        A = it;
                        B = itp;
                    }
                    else
                    {
                        A = (it - lo_h(lo)) * nslm + pm;
                        B = (itp - lo_h(lo)) * nslm + pm;
                    }
                    const int orow = right ? itq * nbb + ps : ps * nbb + itq;
                    if(A < 0 || A >= 65536 || B < 0 || B >= 65536)
                        return false;
                    rows.push_back(make_int2((int)((unsigned)A | ((unsigned)B << 16)), x | (orow << 2)));
                    cnt++;
                }
                p.hrr_loff[t][side][sl] = cnt;
            }
        }
    return true;
}

// Plan of one class for one variant (v = 0: the default, 256 threads, B = 4
// halved until shared memory fits).
static bool c2_build(const int am[4], int deriv, int v, C2Host & h)
{
    C2Params & p = h.p;
    memset(&p, 0, sizeof(p));
    memcpy(p.am, am, sizeof(p.am));
    p.deriv = deriv;
    p.missing = -1;
    h.nthreads = v ? c2_threads(v) : 256;
    const int forceB = v ? v % 20 : 0;
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
        p.wstart[s] = (int)h.items.size();
        std::vector<C2ItemHost> wv;
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
                            C2ItemHost itm;
                            int x, nA, nB;
                            itm.dst = slot(e, f, gE, gF);
                            if(ket)
                            {
                                x = c2_stepdir(i_f, jf, kf);
                                int f1[3] = {F3[0], F3[1], F3[2]}; f1[x]--;
                                const int gF1 = flat(f1[0], f1[1], f1[2]);
                                itm.s1 = slot(e, f - 1, gE, gF1);
                                nA = F3[x] - 1;
                                if(F3[x] >= 2)
                                {
                                    int f2[3] = {F3[0], F3[1], F3[2]}; f2[x] -= 2;
                                    itm.s2 = slot(e, f - 2, gE, flat(f2[0], f2[1], f2[2]));
                                }
                                else
                                    itm.s2 = -1;
                                nB = E3[x];
                                if(E3[x] >= 1)
                                {
                                    int e1[3] = {E3[0], E3[1], E3[2]}; e1[x]--;
                                    itm.s3 = slot(e - 1, f - 1, flat(e1[0], e1[1], e1[2]), gF1);
                                }
                                else
                                    itm.s3 = -1;
                            }
                            else
                            {
                                x = c2_stepdir(ie, je, ke);
                                int e1[3] = {E3[0], E3[1], E3[2]}; e1[x]--;
                                const int gE1 = flat(e1[0], e1[1], e1[2]);
                                itm.s1 = slot(e - 1, f, gE1, gF);
                                nA = E3[x] - 1;
                                if(E3[x] >= 2)
                                {
                                    int e2[3] = {E3[0], E3[1], E3[2]}; e2[x] -= 2;
                                    itm.s2 = slot(e - 2, f, flat(e2[0], e2[1], e2[2]), gF);
                                }
                                else
                                    itm.s2 = -1;
                                nB = F3[x];
                                if(F3[x] >= 1)
                                {
                                    int f1[3] = {F3[0], F3[1], F3[2]}; f1[x]--;
                                    itm.s3 = slot(e - 1, f - 1, gE1, flat(f1[0], f1[1], f1[2]));
                                }
                                else
                                    itm.s3 = -1;
                            }
                            int mask = 0, acc0 = -1;
                            for(int tg = 0; tg < p.ntag; tg++)
                                if(e >= p.elo[tg] && e <= p.ehi[tg] && f >= p.flo[tg] && f <= p.fhi[tg])
                                {
                                    if(tg == 0)
                                        acc0 = p.acc_off[0] + (gE - lo_h(p.elo[0])) * p.acc_nf[0]
                                             + (gF - lo_h(p.flo[0]));
                                    else
                                        mask |= 1 << tg;
                                }
                            itm.combo = (ket ? 3 : 0) + x;
                            itm.mlen = mneed[e][f] + 1;
                            itm.acc0 = acc0;
                            itm.mask = mask;
                            itm.gE = gE;
                            itm.gF = gF;
                            itm.nA = std::max(nA, 0);
                            itm.nB = nB;
                            // one unit per auxiliary order m: the orders of an element are
                            // independent, so they spread over threads instead of
                            // running as one serial chain
                            for(int m = 0; m < itm.mlen; m++)
                            {
                                C2ItemHost u = itm;
                                u.dst += m;
                                u.s1 += m;
                                if(u.s2 >= 0) u.s2 += m;
                                if(u.s3 >= 0) u.s3 += m;
                                u.mlen = 1;
                                if(m > 0)
                                {
                                    u.acc0 = -1;
                                    u.mask = 0;
                                }
                                wv.push_back(u);
                            }
                        }
        }
        // natural order (block by block, element by element, m innermost):
        // neighbouring threads touch neighbouring shared-memory words
        for(const C2ItemHost & u : wv)
        {
            if(u.dst >= 65536 || u.s1 >= 65536 || u.s2 >= 65536 || u.s3 >= 65536 || u.acc0 >= 65535
               || u.nA > 15 || u.nB > 15 || u.gE >= 1024 || u.gF >= 1024 || u.mlen != 1)
                return false;            // outside the packed item format
            C2Item q;
            q.x = (int)((unsigned)u.dst | ((unsigned)u.s1 << 16));
            q.y = (int)((unsigned)(u.s2 < 0 ? 0 : u.s2) | ((unsigned)(u.s3 < 0 ? 0 : u.s3) << 16));
            q.z = (u.acc0 < 0 ? 0xffff : u.acc0) | (u.combo << 16) | ((u.s2 >= 0) << 24)
                | ((u.s3 >= 0) << 25) | (((u.mask >> 1) & 15) << 26);
            q.w = u.nA | (u.nB << 4) | (u.gE << 8) | (u.gF << 18);
            h.items.push_back(q);
        }
    }
    p.wstart[E + F + 1] = (int)h.items.size();
    for(int s = p.smax + 1; s <= E + F + 1; s++)
        p.wstart[s] = p.wstart[E + F + 1];
    // HRR buffers: intermediate layers (not the first, which reads the
    // accumulators, nor the last, which writes its destination) ping-pong in
    // two buffers; the bra side's result (ab|f) for all columns sits in mid
    int hl = 0, midmax = 0, maxslm = 0;
    for(int t = 0; t < p.ntarget; t++)
    {
        const int * tt = p.tgt[t];
        const int klo = p.ketstep_l ? tt[2] : tt[3];
        const int ncol = lo_h(tt[2] + tt[3] + 1) - lo_h(klo);
        const int nbra = nc2(tt[0]) * nc2(tt[1]);
        auto side = [&](int right, int ta, int tb, int ncl) {
            const int lt = ta + tb, lo = right ? ta : tb, slm = right ? tb : ta;
            int mx = 0;
            for(int sl = 1; sl < slm; sl++)
                mx = std::max(mx, (lo_h(lt - sl + 1) - lo_h(lo)) * nc2(sl) * ncl);
            return mx;
        };
        hl = std::max(hl, side(p.brastep_j, tt[0], tt[1], ncol));
        hl = std::max(hl, side(p.ketstep_l, tt[2], tt[3], nbra));
        midmax = std::max(midmax, nbra * ncol);
        maxslm = std::max(maxslm, std::max(p.brastep_j ? tt[1] : tt[0], p.ketstep_l ? tt[3] : tt[2]));
    }
    // one intermediate buffer suffices up to two transfer steps per side
    const int nbuf = maxslm >= 3 ? 2 : (maxslm == 2 ? 1 : 0);
    p.hrr_layer = (hl + 1) & ~1;
    p.hrr_need = nbuf * p.hrr_layer + midmax;
    // prepared primitive quartet: FP64 coefficients and Boys values, then an
    // FP32 copy of the coefficients (25 floats) for the mixed-precision VRR
    p.off32 = (C2_NCOEF + p.L + 1 + 1) & ~1;
    p.prep_stride = p.off32 + 14;
    // shared memory: [waves | HRR (reuses waves) | acc | prep | surv]
    const int NT = h.nthreads;
    p.B = forceB > 0 ? forceB : 4;
    for(;;)
    {
        const int waves = 3 * p.B * p.wsize;
        const int hrr = nbuf * p.hrr_layer + midmax;
        p.off_hrr_b = 0;
        p.off_hrr_mid = nbuf * p.hrr_layer;
        p.off_acc = (std::max(waves, hrr) + 1) & ~1;
        p.off_prep = (p.off_acc + p.acc_size + 1) & ~1;
        p.off_surv = p.off_prep + C2_SETUP * p.prep_stride;
        p.smem_doubles = p.off_surv + NT / 2;
        if(p.smem_doubles * 8 <= 200 * 1024 || p.B == 1 || forceB > 0)
            break;
        p.B /= 2;
    }
    p.ordering = 0;
    int ro = 0;
    for(int t = 0; t < p.ntarget; t++)
    {
        p.res_off[t] = ro;
        if(deriv)
            ro += nc2(p.tgt[t][0]) * nc2(p.tgt[t][1]) * nc2(p.tgt[t][2]) * nc2(p.tgt[t][3]);
    }
    p.res_size = std::max(ro, 1);
    if(!c2_build_hrr(p, h.hrr))
        return false;
    return p.smem_doubles * 8 <= 200 * 1024 && nc2(am[0]) * nc2(am[1]) <= C2_MAXN
        && nc2(am[2]) * nc2(am[3]) <= C2_MAXN;
}

static std::mutex g_c2_mutex;
static std::map<std::array<int, 6>, C2Host> g_c2;

static C2Host * c2_get(const int am[4], int deriv, int v)
{
    std::lock_guard<std::mutex> lk(g_c2_mutex);
    std::array<int, 6> key = {am[0], am[1], am[2], am[3], deriv, v};
    auto it = g_c2.find(key);
    if(it == g_c2.end())
    {
        C2Host h;
        h.ok = (v == 0 || c2_is_variant(v)) && c2_build(am, deriv, v, h);
        it = g_c2.emplace(key, std::move(h)).first;
    }
    return &it->second;
}

// Device copies of the unit and HRR tables of plan h on the current device
// (uploaded once per device); their addresses go into p.
static bool c2_dev_tables(C2Host * h, C2Params & p)
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_c2_mutex);
    auto it = h->dev_tables.find(dev);
    if(it == h->dev_tables.end())
    {
        const size_t bi = h->items.size() * sizeof(C2Item), bh = h->hrr.size() * sizeof(int2);
        char * d = nullptr;
        if(cudaMalloc(&d, std::max<size_t>(16, bi + bh)) != cudaSuccess)
        {
            cudaGetLastError();
            set_error("out of device memory for cooperative-kernel tables");
            return false;
        }
        cudaMemcpy(d, h->items.data(), bi, cudaMemcpyHostToDevice);
        cudaMemcpy(d + bi, h->hrr.data(), bh, cudaMemcpyHostToDevice);
        it = h->dev_tables.emplace(dev, d).first;
    }
    p.items = (const C2Item *)it->second;
    p.hrr_rows = (const int2 *)(it->second + h->items.size() * sizeof(C2Item));
    return true;
}

bool coop2_hrr_params(const int am[4], C2Params & out)
{
    C2Host * h = c2_get(am, 0, 0);
    if(!h->ok)
        return false;
    upload_cart_info();
    out = h->p;
    return c2_dev_tables(h, out);
}

bool coop2_supported(const int am[4], int deriv, int v)
{
    return c2_get(am, deriv, v)->ok;
}

bool coop2_is_variant(int v) { return c2_is_variant(v); }

template<int MODE, int NT, int DERIV, bool MIXED>
static int c2_launch(KernArgs & a, const C2Params & p, cudaStream_t stream)
{
    static std::mutex m;
    static std::map<std::pair<int, int>, int> per_sm_cache;     // (device, smem) -> CTAs per SM
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t smem = (size_t)p.smem_doubles * sizeof(double);
    int per_sm = 0, nsm = 148;
    {
        std::lock_guard<std::mutex> lk(m);
        auto it = per_sm_cache.find({dev, (int)smem});
        if(it == per_sm_cache.end())
        {
            cudaFuncSetAttribute(k_coop2<MODE, NT, DERIV, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
            if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_coop2<MODE, NT, DERIV, MIXED>, NT, smem) != cudaSuccess)
            {
                cudaGetLastError();
                per_sm = 1;
            }
            it = per_sm_cache.emplace(std::make_pair(dev, (int)smem), std::max(per_sm, 1)).first;
        }
        per_sm = it->second;
    }
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    long long grid = std::min<long long>(a.ntask, (long long)nsm * per_sm);
    grid = std::max<long long>(grid, 1);
    Workspace & w = workspace();
    const size_t scratch = (size_t)grid * p.res_size * sizeof(double);
    if(!w.dscratch.reserve(scratch))
    {
        set_error("out of device memory for cooperative-kernel scratch");
        return SIMINT_B200_ERR_CUDA;
    }
    k_coop2<MODE, NT, DERIV, MIXED><<<(unsigned)grid, NT, smem, stream>>>(a, p, (double *)w.dscratch.ptr);
    count_launch(1);
    return 0;
}

int launch_coop2(KernArgs & a, const int req[4], int deriv, int mode, int prec, cudaStream_t stream,
                 int v)
{
    C2Host * h = c2_get(req, deriv, v);
    if(!h->ok)
    {
        set_error("class outside the cooperative kernel's range");
        return SIMINT_B200_ERR_CLASS;
    }
    upload_cart_info();
    C2Params p = h->p;
    if(!c2_dev_tables(h, p))
        return SIMINT_B200_ERR_CUDA;
    p.ordering = ordering();
    a.swapB = a.swapK = a.pq = 0;
    a.oidx = nullptr;
    // the FP32 VRR applies to deriv 0 in mixed mode with a positive gate
    const bool mixed = prec == SIMINT_B200_PREC_MIXED && a.gate > 0.0 && deriv == 0;
    if(h->nthreads == 64)
    {
        if(deriv)
            return mode == 0 ? c2_launch<0, 64, 1, false>(a, p, stream)
                 : mode == 1 ? c2_launch<1, 64, 1, false>(a, p, stream) : c2_launch<2, 64, 1, false>(a, p, stream);
        if(mixed)
            return mode == 0 ? c2_launch<0, 64, 0, true>(a, p, stream)
                 : mode == 1 ? c2_launch<1, 64, 0, true>(a, p, stream) : c2_launch<2, 64, 0, true>(a, p, stream);
        return mode == 0 ? c2_launch<0, 64, 0, false>(a, p, stream)
             : mode == 1 ? c2_launch<1, 64, 0, false>(a, p, stream) : c2_launch<2, 64, 0, false>(a, p, stream);
    }
    if(h->nthreads == 128)
    {
        if(deriv)
            return mode == 0 ? c2_launch<0, 128, 1, false>(a, p, stream)
                 : mode == 1 ? c2_launch<1, 128, 1, false>(a, p, stream) : c2_launch<2, 128, 1, false>(a, p, stream);
        if(mixed)
            return mode == 0 ? c2_launch<0, 128, 0, true>(a, p, stream)
                 : mode == 1 ? c2_launch<1, 128, 0, true>(a, p, stream) : c2_launch<2, 128, 0, true>(a, p, stream);
        return mode == 0 ? c2_launch<0, 128, 0, false>(a, p, stream)
             : mode == 1 ? c2_launch<1, 128, 0, false>(a, p, stream) : c2_launch<2, 128, 0, false>(a, p, stream);
    }
    if(deriv)
        return mode == 0 ? c2_launch<0, 256, 1, false>(a, p, stream)
             : mode == 1 ? c2_launch<1, 256, 1, false>(a, p, stream) : c2_launch<2, 256, 1, false>(a, p, stream);
    if(mixed)
        return mode == 0 ? c2_launch<0, 256, 0, true>(a, p, stream)
             : mode == 1 ? c2_launch<1, 256, 0, true>(a, p, stream) : c2_launch<2, 256, 0, true>(a, p, stream);
    return mode == 0 ? c2_launch<0, 256, 0, false>(a, p, stream)
         : mode == 1 ? c2_launch<1, 256, 0, false>(a, p, stream) : c2_launch<2, 256, 0, false>(a, p, stream);
}

} // namespace sb200
