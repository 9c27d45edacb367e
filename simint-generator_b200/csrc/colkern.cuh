// Column kernel: one CTA per shell quartet, one thread per (bra Cartesian
// function, primitive quartet of a batch), the ket recursion of a thread's
// bra function held in registers.
//
// Why: the table-driven cooperative kernel (coop2.cu) keeps every VRR
// intermediate in shared memory, so each 4-FMA step costs five or more
// shared-memory accesses and the kernel is bound by shared-memory bandwidth
// and latency.  Here a thread owns the column (g_e, 0 | f)^(m) of one bra
// function g_e over all ket functions f; three of the four source terms of a
// ket step are the thread's own registers and only the (e-1_y, f-1_y)^(m+1)
// term is read from another thread, so a step is ~5 FP64 operations and at
// most one shared-memory load and one store.
//
// Per shell quartet: the surviving primitive quartets (the reference's
// primitive screening, in order; in mixed mode split into an FP64 and an FP32
// list by the error gate) are processed in blocks of FS (up to 32, chosen per
// class to fit shared memory):
//   1. set-up and Boys, one thread per primitive quartet (col_setup),
//   2. the bra-only recursion (g_e, 0|0)^(m) of the whole block, level by
//      level, into a level-major block in shared memory (col_f0_block),
//   3. per batch of NP primitive quartets of the block, the ket stages
//      f = 1..c+d (generated per class: CT::stages), the top quartets summed
//      into per-thread FP64 registers;
// then the per-thread sums are added over the batch slots in a fixed order
// into the cooperative kernel's accumulator layout, and its HRR
// (c2_hrr_side, OSTEI_HRR_Algorithm_Base.cpp:160-283) runs in shared memory
// and writes through the output index table (ordering and role swaps).
// Shell quartets come from the launch's work queue (cta_next_task).
//
// Class constants, shared-memory sizes and the stage code come from a
// generated traits struct CT (simint_b200/gen/colgen.py).
#pragma once

#include <vector>

#include "coop2.cuh"

__device__ __forceinline__ double cfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ float cfma(float a, float b, float c) { return fmaf(a, b, c); }

// coefficient record of a set-up primitive quartet (doubles, rows of FS)
enum { CC_XP = 0, CC_YP = 3, CC_XQ = 6, CC_YQ = 9, CC_ZP = 12, CC_ZQ = 13, CC_O2P = 14, CC_O2Q = 15,
       CC_O2PQ = 16, CC_F = 17 };

__host__ __device__ constexpr int col_lo(int l) { return l <= 0 ? 0 : (l * (l + 1) * (l + 2)) / 6; }
__host__ __device__ constexpr int col_nt(int nrole, int np) { return ((nrole * np + 31) / 32) * 32; }

// Cartesian exponents of flat index g (levels in order, Psi4 order inside a
// level) and its level.
__device__ __forceinline__ void col_cart(int g, int & i, int & j, int & k, int & l)
{
    l = 0;
    while(col_lo(l + 1) <= g)
        l++;
    int p = g - col_lo(l);
    for(i = l; i >= 0; i--)
    {
        const int n = l - i + 1;             // functions with this x exponent
        if(p < n)
            break;
        p -= n;
    }
    k = p;
    j = l - i - k;
}

__device__ __forceinline__ int col_flat(int i, int j, int k)
{
    const int l = i + j + k;
    return col_lo(l) + ((l - i) * (l - i + 1)) / 2 + k;
}

// First row of level e in the level-major bra block: levels 0..e-1 hold
// orders 0..L-e' of their nc(e') functions.
__host__ __device__ constexpr int col_lb(int L, int e)
{
    int r = 0;
    for(int x = 0; x < e; x++)
        r += ((x + 1) * (x + 2)) / 2 * (L - x + 1);
    return r;
}

__device__ __forceinline__ int col_stepdir(int i, int j, int k)
{
    const int e[3] = {i, j, k};
    int mn = 1000;
    for(int x = 0; x < 3; x++)
        if(e[x] > 0 && e[x] < mn) mn = e[x];
    for(int x = 2; x >= 0; x--)
        if(e[x] == mn) return x;
    return 0;
}

// Row pitch of the bra block for FS slots: FS + 8 doubles from 16 slots up,
// so that the 8-slot segments of the four roles a warp reads fall on both
// halves of the shared-memory banks (a multiple of 16 would put them all on
// one half).
__host__ __device__ constexpr int col_pitch(int FS) { return FS >= 16 ? FS + 8 : FS; }

// Barrier of one group of NTH threads of a CTA: group g waits on named
// barrier 1 + g, so the H groups of a CTA run their shell quartets
// independently (a CTA barrier when the CTA is one group).
template<int H, int NTH>
struct ColSync
{
    int id;
    __device__ __forceinline__ void operator()() const
    {
        if constexpr(H == 1)
            __syncthreads();
        else
            asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(NTH) : "memory");
    }
};

// Set-up and Boys values of survivors list[s0 .. s0 + ns) (ns <= FS threads
// in parallel; slots past n get zeros, which run through the recursion as
// zeros) into coef[k * FS + slot].
template<class CT, typename SYNC>
__device__ __forceinline__ void col_setup(const QuartetCtx & c, const int * __restrict__ list, int s0, int n,
                                          int nj, unsigned long long njinv, bool fastdiv,
                                          double * __restrict__ coef, int FS, int ns, int tid, SYNC sync)
{
    if(tid < ns)
    {
        const int g = s0 + tid;
        double v[CC_F + CT::L + 1];
        #pragma unroll
        for(int k = 0; k < CC_F + CT::L + 1; k++)
            v[k] = 0.0;
        if(g < n)
        {
            const int kk = list[g];
            const int kq = fastdiv ? (int)(((unsigned long long)kk * njinv) >> 32) : kk / nj;
            const int i = c.bi0 + kq, j = c.kj0 + (kk - kq * nj);
            const BraPrim bp = load_bra_prim(c, i);
            PrimSetup s;
            prim_setup(c, bp, j, s);
            v[CC_XP + 0] = s.PAx; v[CC_XP + 1] = s.PAy; v[CC_XP + 2] = s.PAz;
            v[CC_YP + 0] = s.aopPQx; v[CC_YP + 1] = s.aopPQy; v[CC_YP + 2] = s.aopPQz;
            v[CC_XQ + 0] = s.QCx; v[CC_XQ + 1] = s.QCy; v[CC_XQ + 2] = s.QCz;
            v[CC_YQ + 0] = s.aoqPQx; v[CC_YQ + 1] = s.aoqPQy; v[CC_YQ + 2] = s.aoqPQz;
            v[CC_ZP] = s.a_over_p; v[CC_ZQ] = s.a_over_q;
            v[CC_O2P] = s.oo2p; v[CC_O2Q] = s.oo2q; v[CC_O2PQ] = s.oo2pq;
            c2_boys(c.boys, s.T, CT::L, s.prefac, v + CC_F);
        }
        #pragma unroll
        for(int k = 0; k < CC_F + CT::L + 1; k++)
            coef[k * FS + tid] = v[k];
    }
    sync();
}

// Bra-only recursion of the first ns slots of a block into the
// level-major block F0: (g, 0|0)^(m) of bra function g = lo(e) + p at
// F0[(lb(e) + m * nc(e) + p) * FR + slot], orders 0..L - e (level 0: F_m
// times the pair prefactors).  Work items (function, slot) of a level spread
// over the CTA; one barrier per level.
template<typename T, class CT, int NT, typename SYNC>
__device__ __forceinline__ void col_f0_block(T * __restrict__ F0, const double * __restrict__ coef, int FS,
                                             int FR, int ns, int tid, SYNC sync)
{
    for(int it = tid; it < (CT::L + 1) * ns; it += NT)
    {
        const int m = it / ns, slot = it - m * ns;
        F0[m * FR + slot] = (T)coef[(CC_F + m) * FS + slot];
    }
    sync();
    int lb2 = 0, lb1 = 0, lbe = CT::L + 1;           // first rows of levels e-2, e-1, e
    #pragma unroll 1
    for(int e = 1; e <= CT::E; e++)
    {
        const int nce = ((e + 1) * (e + 2)) / 2, nc1 = (e * (e + 1)) / 2, nc2 = ((e - 1) * e) / 2;
        const int nitem = nce * ns;
        for(int it = tid; it < nitem; it += NT)
        {
            const int pe = it / ns, slot = it - pe * ns;
            int i, j, k, l;
            col_cart(col_lo(e) + pe, i, j, k, l);
            const int x = col_stepdir(i, j, k);
            int q[3] = {i, j, k};
            const int n = q[x] - 1;
            q[x] -= 1;
            const int p1 = col_flat(q[0], q[1], q[2]) - col_lo(e - 1);
            q[x] -= 1;
            const int p2 = n > 0 ? col_flat(q[0], q[1], q[2]) - col_lo(e - 2) : 0;
            const T XP = (T)coef[(CC_XP + x) * FS + slot];
            const T YP = (T)coef[(CC_YP + x) * FS + slot];
            const T Zp = (T)coef[CC_ZP * FS + slot];
            const T k2 = (T)((double)n * coef[CC_O2P * FS + slot]);
            const T * s1 = F0 + (lb1 + p1) * FR + slot;
            const T * s2 = F0 + (n > 0 ? (lb2 + p2) * FR + slot : 0);
            T * dst = F0 + (lbe + pe) * FR + slot;
            const int st1 = nc1 * FR, st2 = nc2 * FR, st = nce * FR;
            for(int m = 0; m <= CT::L - e; m++)
            {
                T r = XP * s1[m * st1];
                r = cfma(YP, s1[(m + 1) * st1], r);
                if(n > 0)
                    r = cfma(k2, cfma(Zp, s2[(m + 1) * st2], s2[m * st2]), r);
                dst[m * st] = r;
            }
        }
        sync();
        lb2 = lb1;
        lb1 = lbe;
        lbe += nce * (CT::L - e + 1);
    }
}

// Per-thread constants of the column kernel: the thread's role (bra
// function g_e) and slot, its positions in the batch areas (own, loff) and
// in the bra block (ownF + m * ostr: order m of its own column; loffF[y] +
// m * mstrF[y]: order m of g_e - 1_y).
struct ColThread
{
    int role, slot, own, ownF, ostr;
    bool valid;
    int ny[3], loff[3], loffF[3], mstrF[3];
};

template<class CT, int NP>
__device__ __forceinline__ void col_thread(ColThread & t, int FR, int tid)
{
    t.role = tid / NP;
    t.slot = tid - t.role * NP;
    t.valid = t.role < CT::NROLE;
    int ri = 0, rj = 0, rk = 0, re = 0;
    if(t.valid)
        col_cart(t.role, ri, rj, rk, re);
    t.ny[0] = ri; t.ny[1] = rj; t.ny[2] = rk;
    t.own = t.role * NP + t.slot;
    const int pe = t.valid ? t.role - col_lo(re) : 0;
    const int lbr = col_lb(CT::L, re), lbr1 = re > 0 ? col_lb(CT::L, re - 1) : 0;
    t.ownF = t.valid ? (lbr + pe) * FR + t.slot : t.slot;
    t.ostr = ((re + 1) * (re + 2)) / 2 * FR;
    #pragma unroll
    for(int y = 0; y < 3; y++)
    {
        int q[3] = {ri, rj, rk};
        q[y] -= 1;
        const bool has = t.valid && t.ny[y] > 0;
        const int g1 = has ? col_flat(q[0], q[1], q[2]) : 0;
        // absent g_e - 1_y: the thread's own position (its coefficient n_y
        // is 0 and the value read is a finite one)
        t.loff[y] = (has ? g1 : (t.valid ? t.role : 0)) * NP + t.slot;
        t.loffF[y] = has ? (lbr1 + g1 - col_lo(re - 1)) * FR + t.slot : t.ownF;
        t.mstrF[y] = has ? (re * (re + 1)) / 2 * FR : t.ostr;
    }
}

// The ket stages of batch [b0, b0 + NP) of a block (coef: the block's
// records, row stride FS) in type T.
template<typename T, class CT, int NP, typename SYNC>
__device__ __forceinline__ void col_batch(const T * __restrict__ F0, T * __restrict__ SA, T * __restrict__ SB,
                                          const double * __restrict__ coef, int FS, int b0,
                                          const ColThread & t, double (&acc)[CT::NTOP], SYNC sync)
{
    const int cs = b0 + t.slot;
    T XQ[3], YQ[3], cB[3], kq[CT::KQN], Zq = 0;
    #pragma unroll
    for(int y = 0; y < 3; y++)
    {
        XQ[y] = t.valid ? (T)coef[(CC_XQ + y) * FS + cs] : (T)0;
        YQ[y] = t.valid ? (T)coef[(CC_YQ + y) * FS + cs] : (T)0;
        cB[y] = t.valid ? (T)((double)t.ny[y] * coef[CC_O2PQ * FS + cs]) : (T)0;
    }
    if(t.valid)
        Zq = (T)coef[CC_ZQ * FS + cs];
    #pragma unroll
    for(int k = 0; k < CT::KQN; k++)
        kq[k] = t.valid ? (T)((double)(k + 1) * coef[CC_O2Q * FS + cs]) : (T)0;
    CT::template stages<T, NP>(F0 + b0, SA, SB, t.own, t.ownF, t.ostr, t.loff, t.loffF, t.mstrF, XQ, YQ, Zq, kq,
                               cB, t.valid, acc, sync);
}

// One block of survivors list[s0 ..) in type T: set-up, bra block, batches.
template<typename T, class CT, int NP, int NT, typename SYNC>
__device__ __forceinline__ void col_block(const QuartetCtx & c, const int * __restrict__ list, int s0, int n,
                                          int nj, unsigned long long njinv, bool fastdiv, double * __restrict__ coef,
                                          double * __restrict__ V, int FS, const ColThread & t,
                                          double (&acc)[CT::NTOP], int tid, SYNC sync)
{
    const int FR = col_pitch(FS);
    T * F0 = (T *)V;
    T * SA = F0 + CT::F0B * FR;
    T * SB = SA + CT::SAN * NP;
    // a short last block (or a short contraction) sets up and runs the
    // bra recursion for its batches only
    const int nb = min(FS, n - s0);
    const int ns = ((nb + NP - 1) / NP) * NP;
    col_setup<CT>(c, list, s0, n, nj, njinv, fastdiv, coef, FS, ns, tid, sync);
    col_f0_block<T, CT, NT>(F0, coef, FS, FR, ns, tid, sync);
    for(int b0 = 0; b0 < nb; b0 += NP)
        col_batch<T, CT, NP>(F0, SA, SB, coef, FS, b0, t, acc, sync);
}

// Task loop of one group: static stride over the group slots of the grid,
// or pulls from the launch's work queue (thread 0 of the group pulls).
template<typename SYNC>
__device__ __forceinline__ bool col_next_task(const KernArgs & a, long long & slot, long long & t,
                                              long long * s_slot, int tid, SYNC sync)
{
    if(a.wq)
    {
        if(tid == 0)
            *s_slot = queue_pull(a.wq);
        sync();
        slot = *s_slot;
        sync();
        if(slot < 0)
            return false;
    }
    else if(slot >= a.ntask)
        return false;
    t = a.tperm ? (long long)__ldg(a.tperm + slot) : slot;
    return true;
}

// H groups of NT threads per CTA (H = 1 or 2), each with its own part of
// shared memory (phd doubles) running its own shell quartets: while one
// group waits at a barrier the other computes.
template<class CT, int MODE, bool MIXED, int NP, int H>
__global__ void __launch_bounds__(H * col_nt(CT::NROLE, NP), 1)
k_col(const KernArgs a, const C2Params p, const int vdoubles, const int FS, const int phd)
{
    constexpr int NT = col_nt(CT::NROLE, NP);       // threads of a group
    extern __shared__ __align__(16) double sm[];
    __shared__ int wcount_g[H][2][NT / 32];
    __shared__ int s_cnt_g[H][2];
    __shared__ long long s_qslot_g[H];
    const int grp = H == 1 ? 0 : (int)threadIdx.x / NT;
    const int tid = (int)threadIdx.x - grp * NT;
    const ColSync<H, NT> sync{1 + grp};
    int (*wcount)[NT / 32] = wcount_g[grp];
    int * s_cnt = s_cnt_g[grp];
    double * V = sm + (size_t)grp * phd;
    double * coef = V + vdoubles;
    double * acc2 = coef + (CC_F + CT::L + 1) * FS;
    int * surv = (int *)(acc2 + ((p.acc_size + 1) & ~1));   // [0, NT): FP64 list, [NT, 2 NT): FP32 list
    ColThread th;
    col_thread<CT, NP>(th, col_pitch(FS), tid);
    const int role = th.role, slot = th.slot;
    const bool valid = th.valid;
    const int lane = tid & 31, warp = tid >> 5;
    long long t = 0;
    for(long long qslot = (long long)blockIdx.x * H + grp; col_next_task(a, qslot, t, &s_qslot_g[grp], tid, sync);
        qslot += (long long)gridDim.x * H)
    {
        int iP, iQ;
        long long off;
        task_of<MODE>(a, t, iP, iQ, off);
        QuartetCtx c;
        make_ctx(a, iP, iQ, c);
        const int ni = c.bi1 - c.bi0, nj = c.kj1 - c.kj0;
        if(MIXED)
        {
            c.gL = CT::L;
            c.gamp = hrr_amp(c, CT::A1, CT::A3);
            // the gate bounds the error of one integral: each of the shell
            // quartet's primitive quartets may take gate / (their number)
            c.gate = a.gate / (double)max(1, ni * nj);
        }
        double acc[CT::NTOP];
        #pragma unroll
        for(int k = 0; k < CT::NTOP; k++)
            acc[k] = 0.0;
        const int ncand = ni * nj;
        const unsigned long long njinv = nj > 0 ? (1ull << 32) / (unsigned)nj + 1ull : 0ull;
        const bool fastdiv = (long long)ncand * nj < (1LL << 32);
        for(int k0 = 0; k0 < ncand; k0 += NT)
        {
            // ordered compaction of the surviving candidates k0 .. k0 + NT
            // (FP64 list; in mixed mode the gated ones go to the FP32 list)
            const int k = k0 + tid;
            bool ok = false, low = false;
            if(k < ncand)
            {
                const int kq = fastdiv ? (int)(((unsigned long long)k * njinv) >> 32) : k / nj;
                const int i = c.bi0 + kq, j = c.kj0 + (k - kq * nj);
                const BraPrim bp = load_bra_prim(c, i);
                ok = !(c.check && (bp.skip || !prim_survives(c, bp, j)));
                if(MIXED && ok)
                {
                    PrimSetup s;
                    prim_setup(c, bp, j, s);
                    low = s.lowprec;
                }
            }
            const bool hi = ok && !low, lo = ok && low;
            const unsigned bh = __ballot_sync(0xffffffffu, hi);
            const unsigned bl = __ballot_sync(0xffffffffu, lo);
            if(lane == 0)
            {
                wcount[0][warp] = __popc(bh);
                wcount[1][warp] = __popc(bl);
            }
            sync();
            int b0 = 0, b1 = 0;
            for(int w = 0; w < warp; w++)
            {
                b0 += wcount[0][w];
                b1 += wcount[1][w];
            }
            const unsigned below = (1u << lane) - 1u;
            if(hi)
                surv[b0 + __popc(bh & below)] = k;
            if(lo)
                surv[NT + b1 + __popc(bl & below)] = k;
            if(tid == NT - 1)
            {
                int t0 = 0, t1 = 0;
                for(int w = 0; w < NT / 32; w++)
                {
                    t0 += wcount[0][w];
                    t1 += wcount[1][w];
                }
                s_cnt[0] = t0;
                s_cnt[1] = t1;
            }
            sync();
            const int nhi = s_cnt[0], nlo = s_cnt[1];
            if(MIXED && tid == 0 && nlo > 0 && a.fp32_count)
                atomicAdd(a.fp32_count, (unsigned long long)nlo);
            for(int s0 = 0; s0 < nhi; s0 += FS)
                col_block<double, CT, NP, NT>(c, surv, s0, nhi, nj, njinv, fastdiv, coef, V, FS, th, acc, tid, sync);
            if constexpr(MIXED)
            {
                for(int s0 = 0; s0 < nlo; s0 += FS)
                    col_block<float, CT, NP, NT>(c, surv + NT, s0, nlo, nj, njinv, fastdiv, coef, V, FS, th, acc, tid,
                                                 sync);
            }
            sync();      // surv, s_cnt and wcount are reused
        }
        // sums over the batch slots, in slot order, into the accumulator
        // layout of the HRR: acc2[(g_e - lo(a)) * NTOP + t]
        constexpr int TOP0 = col_lo(CT::A0);
        constexpr int NTR = CT::NROLE - TOP0;          // bra functions of levels a .. a+b
        if(valid && role >= TOP0)
        {
            #pragma unroll
            for(int k = 0; k < CT::NTOP; k++)
                V[(k * NTR + (role - TOP0)) * NP + slot] = acc[k];
        }
        sync();
        for(int idx = tid; idx < NTR * CT::NTOP; idx += NT)
        {
            const int k = idx / NTR, rr = idx - k * NTR;
            double sum = 0.0;
            #pragma unroll
            for(int s2 = 0; s2 < NP; s2++)
                sum += V[(k * NTR + rr) * NP + s2];
            acc2[p.acc_off[0] + rr * p.acc_nf[0] + k] = sum;
        }
        sync();
        // ---------------- HRR ----------------
        double * LA = V + p.off_hrr_b;
        double * LB = LA + p.hrr_layer;
        double * mid = V + p.off_hrr_mid;
        double * o = a.out + off;
        const unsigned short * __restrict__ oidx = a.oidx;
        const int * tt = p.tgt[0];
        const int klo = tt[2];
        const int ncol = c2_lev_off(tt[2] + tt[3] + 1) - c2_lev_off(klo);
        const int nbra = c2_nc(tt[0]) * c2_nc(tt[1]);
        const int nket = c2_nc(tt[2]) * c2_nc(tt[3]);
        const int accb = p.acc_off[0], accnf = p.acc_nf[0];
        const int e0 = c2_lev_off(p.elo[0]), f0 = c2_lev_off(p.flo[0]), fk = c2_lev_off(klo);
        c2_hrr_side_t<NT>(tid, sync, p.brastep_j, p.hrr_nl[0][0], ncol, p.hrr_rows + p.hrr_base[0][0], p.hrr_loff[0][0],
                        c.AB[0], c.AB[1], c.AB[2],
                        [&](int g, int col) { return acc2[accb + (g - e0) * accnf + (fk + col - f0)]; },
                        [&](int r, int col, double v) { mid[r * ncol + col] = v; }, LA, LB);
        const int kl = c2_lev_off(klo);
        c2_hrr_side_t<NT>(tid, sync, p.ketstep_l, p.hrr_nl[0][1], nbra, p.hrr_rows + p.hrr_base[0][1], p.hrr_loff[0][1],
                        c.CD[0], c.CD[1], c.CD[2],
                        [&](int g, int row) { return mid[row * ncol + (g - kl)]; },
                        [&](int r, int row, double v) { o[oidx[row * nket + r]] = v; }, LA, LB);
        sync();
    }
}

// ---------------------------------------------------------------------
// registry of the generated classes
// ---------------------------------------------------------------------

typedef void (*ColFn)(const KernArgs, const C2Params, const int, const int, const int);

// variants 81, 82, 83: (primitive quartets per batch, groups per CTA)
#define COL_NNP 3
static constexpr int COL_NPS[COL_NNP] = {4, 8, 4};
static constexpr int COL_HS[COL_NNP] = {1, 1, 2};

struct ColKernels
{
    int am[4];
    int L, nrole, ntop;
    int f0b;                             // doubles of the bra block per slot
    int sab;                             // doubles of the stage areas SA + SB per batch slot
    int red_per_np;                      // doubles of the slot-sum scratch per batch slot
    int ncoef;                           // doubles of a coefficient record
    int nt[COL_NNP];                     // threads per group for each variant (H groups per CTA)
    ColFn fn[COL_NNP][3][2];             // [np][mode][fp64, mixed]
};

struct ColTable
{
    std::vector<ColKernels> list;
    void add(const ColKernels & k) { list.push_back(k); }
};

template<class CT, int NPI>
static void col_fill_np(ColKernels & k)
{
    constexpr int NP = COL_NPS[NPI];
    constexpr int H = COL_HS[NPI];
    k.nt[NPI] = col_nt(CT::NROLE, NP);
    for(int md = 0; md < 3; md++)
        k.fn[NPI][md][0] = k.fn[NPI][md][1] = nullptr;
    if constexpr(H * col_nt(CT::NROLE, NP) <= 1024)
    {
        k.fn[NPI][0][0] = k_col<CT, 0, false, NP, H>;
        k.fn[NPI][0][1] = k_col<CT, 0, true, NP, H>;
        k.fn[NPI][1][0] = k_col<CT, 1, false, NP, H>;
        k.fn[NPI][1][1] = k_col<CT, 1, true, NP, H>;
        k.fn[NPI][2][0] = k_col<CT, 2, false, NP, H>;
        k.fn[NPI][2][1] = k_col<CT, 2, true, NP, H>;
    }
}

template<class CT>
static void col_fill(ColKernels & k)
{
    k.L = CT::L;
    k.nrole = CT::NROLE;
    k.ntop = CT::NTOP;
    k.f0b = CT::F0B;
    k.sab = CT::SAN + CT::SBN;
    k.red_per_np = CT::NTOP * (CT::NROLE - col_lo(CT::A0));
    k.ncoef = CC_F + CT::L + 1;
    col_fill_np<CT, 0>(k);
    col_fill_np<CT, 1>(k);
    col_fill_np<CT, 2>(k);
}

void simint_b200_register_col(ColTable & t);
