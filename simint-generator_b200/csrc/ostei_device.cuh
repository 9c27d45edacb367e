// Device-side building blocks shared by every generated ERI kernel.
//
// Primitive-pair records: the host packs the SoA arrays of a
// simint_multi_shellpair (skel/simint/shell/shell.h:47-85) into 128-byte
// records, one per padded primitive slot, so a thread fetches everything
// about one primitive pair with full-sector loads:
//   [0] alpha=a+b  [1] prefac  [2..4] P  [5..7] P-A  [8..10] P-B
//   [11] 2a  [12] 2b  [13] screen  [14] max screen of the aligned 8-slot
//   group the slot belongs to  [15] sqrt(screen)
// Field 14 reproduces the reference's 8-wide ket-vector screening test
// (generator/ostei/OSTEI_Writer.cpp:570-586): a ket primitive is skipped
// when the largest P.screen[i]*Q.screen[j'] over its aligned vector of 8
// padded slots is below tol^2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define SB_REC 16

struct PairSetDev
{
    const double * prim;      // records [npad][SB_REC]
    const int * pstart;       // first slot of each shell pair
    const int * nprim;        // primitive pairs per shell pair
    const double * AB;        // A-B per shell pair, [npair][3]
    double screen_max;
    int npair;
};

// Device work queue of one launch.  Tasks 0 .. published-1 may be taken; a
// CTA takes the next index with one atomic add.  When it runs past the
// published count it waits for more -- at most spin_limit polls of about a
// microsecond each -- or leaves once the queue is closed.  A wait that runs
// out sets bit 0 of status (SIMINT_B200_ERR_TIMEOUT on the host) and the CTA
// returns, so a producer that never finishes cannot hang the device.
struct WorkQueue
{
    unsigned long long next;
    unsigned long long published;
    unsigned int closed;
    unsigned int status;
    unsigned long long spin_limit;
};

struct KernArgs
{
    PairSetDev P, Q;          // requested bra and ket pair sets
    const int * kord;         // rectangle mode: ket visiting order
    const int2 * tasks;       // list mode: (bra pair, ket pair)
    const long long * outoff; // list mode: output offset of each task (doubles)
    long long ntask;
    int nQ;                   // rectangle mode: number of ket pairs (output stride)
    int nQc;                  // rectangle mode: ket pairs of this launch (kord entries)
    int swapB, swapK, pq;     // role swaps (see emit.unique_class)
    int check;                // screening on
    double tol2;              // squared tolerance
    double gate;              // mixed precision: FP32 VRR when bound < gate
    const unsigned short * oidx;
    double * out;
    int nout;                 // doubles per shell quartet
    int * status;             // device status word (error flags)
    const double * boys;      // Boys tables (see SB_BOYS_LONGFAC_OFF)
    // MODE 2 (screened sweep): bra pairs border[b], b < nb, each with the
    // ket pairs korder[0 .. prefix[b+1]-prefix[b]); tasks task0.. of it
    const long long * prefix;
    const int * border;
    const int * korder;
    int nb;
    long long task0;
    // CTA-per-quartet kernels: tasks handed out by a device work queue
    // (nullptr: static grid-stride order), queue slot q running task
    // tperm[q] (nullptr: q) -- the host orders a class's tasks by primitive
    // count, heaviest first
    WorkQueue * wq;
    const int * tperm;
    // mixed precision: primitive quartets the CTA-per-quartet kernels ran
    // in FP32 are added here (nullptr: not counted)
    unsigned long long * fp32_count;
    // (ss|ss) with a clipped ket list: ket slots [kvec0, kvec1) are the
    // partial last vector below the clip, whose vector test covers only
    // them (empty range: no such vector)
    int kvec0, kvec1;
    // MODE 2 (ss|ss): per bra pair, the end of its row's ket primitives
    // (the clip of that row's ket list); nullptr: none
    const int * kvend;
};

// The next queue slot of the calling thread's CTA (thread 0 calls it), or -1
// when the queue is drained or a wait ran out.
__device__ __forceinline__ long long queue_pull(WorkQueue * q)
{
    const unsigned long long t = atomicAdd(&q->next, 1ull);
    volatile WorkQueue * v = q;
    for(unsigned long long it = 0;; it++)
    {
        if(t < v->published)
            return (long long)t;
        if(v->closed)
        {
            __threadfence();
            return t < v->published ? (long long)t : -1;
        }
        if(it >= v->spin_limit)
        {
            atomicOr(&q->status, 1u);
            return -1;
        }
        __nanosleep(1000);
    }
}

// Task loop of a CTA-per-quartet kernel: static grid stride, or queue pulls.
// Returns false when the CTA has no further task; t is the task index.
__device__ __forceinline__ bool cta_next_task(const KernArgs & a, long long & slot, long long & t,
                                              long long * s_slot)
{
    if(a.wq)
    {
        if(threadIdx.x == 0)
            *s_slot = queue_pull(a.wq);
        __syncthreads();
        slot = *s_slot;
        __syncthreads();
        if(slot < 0)
            return false;
    }
    else if(slot >= a.ntask)
        return false;
    t = a.tperm ? (long long)__ldg(a.tperm + slot) : slot;
    return true;
}

struct QuartetCtx
{
    const double * __restrict__ bprim;
    const double * __restrict__ kprim;
    int bi0, bi1, kj0, kj1;
    double AB[3], CD[3];
    int swapB, swapK, pq, check;
    double tol2;
    double bscreen_max;       // screen_max of the pair set in the bra role
    double kscreen_max;       // screen_max of the pair set in the ket role
    double gate;
    int gL;                   // mixed precision: recursion depth L of the class
    double gamp;              // mixed precision: HRR growth (1+|AB|)^nb (1+|CD|)^nd
    const unsigned short * oidx;
    const double * boys;
    int kvec0, kvec1;         // see KernArgs
    unsigned long long * fp32_count;   // see KernArgs
};

struct BraPrim
{
    double alpha, prefac, x, y, z;
    double PAx, PAy, PAz, PBx, PBy, PBz;
    double a2, b2;
    double screen, vecmax, sq;
    bool skip;
};

struct PrimSetup
{
    double T, prefac;
    double PAx, PAy, PAz, PBx, PBy, PBz;
    double QCx, QCy, QCz, QDx, QDy, QDz;
    double aopPQx, aopPQy, aopPQz, aoqPQx, aoqPQy, aoqPQz;
    double a_over_p, a_over_q;
    double oo2p, oo2q, oo2pq;
    double c2a, c2b, c2c, c2d;    // deriv=1 contraction weights
    bool lowprec;
    // FP32 copies for the mixed-precision VRR
    float PAx_f, PAy_f, PAz_f, PBx_f, PBy_f, PBz_f;
    float QCx_f, QCy_f, QCz_f, QDx_f, QDy_f, QDz_f;
    float aopPQx_f, aopPQy_f, aopPQz_f, aoqPQx_f, aoqPQy_f, aoqPQz_f;
    float a_over_p_f, a_over_q_f, oo2p_f, oo2q_f, oo2pq_f;

    __device__ __forceinline__ void make_f32()
    {
        PAx_f = (float)PAx; PAy_f = (float)PAy; PAz_f = (float)PAz;
        PBx_f = (float)PBx; PBy_f = (float)PBy; PBz_f = (float)PBz;
        QCx_f = (float)QCx; QCy_f = (float)QCy; QCz_f = (float)QCz;
        QDx_f = (float)QDx; QDy_f = (float)QDy; QDz_f = (float)QDz;
        aopPQx_f = (float)aopPQx; aopPQy_f = (float)aopPQy; aopPQz_f = (float)aopPQz;
        aoqPQx_f = (float)aoqPQx; aoqPQy_f = (float)aoqPQy; aoqPQz_f = (float)aoqPQz;
        a_over_p_f = (float)a_over_p; a_over_q_f = (float)a_over_q;
        oo2p_f = (float)oo2p; oo2q_f = (float)oo2q; oo2pq_f = (float)oo2pq;
    }
};

// Boys tables: a device buffer holding the grid F_n(0.1 i) [366][32]
// followed by the 32 asymptotic factors (uploaded once per device).
#define SB_BOYS_LONGFAC_OFF (366 * 32)

__device__ __forceinline__ double boys_taylor(const double * __restrict__ g, double dx)
{
    // F_n(x) = sum_k F_{n+k}(x_i) (x_i - x)^k / k!, k = 0..7 (boys_taylor.h:14-39)
    return __ldg(g + 0) + dx * (__ldg(g + 1) + dx * ((1.0 / 2.0) * __ldg(g + 2)
         + dx * ((1.0 / 6.0) * __ldg(g + 3) + dx * ((1.0 / 24.0) * __ldg(g + 4)
         + dx * ((1.0 / 120.0) * __ldg(g + 5) + dx * ((1.0 / 720.0) * __ldg(g + 6)
         + dx * ((1.0 / 5040.0) * __ldg(g + 7))))))));
}

// F_0..F_L(x).  L < 4: every order from the grid (or the asymptotic form for
// x >= 36.5); L >= 4: F_L only, then downward recursion
// F_n = (2x F_{n+1} + e^{-x}) / (2n+1)  (boys.h:14-92).
template<int L>
__device__ __forceinline__ void boys_split(const double * __restrict__ tab, double x, double * F)
{
    if(L < 4)
    {
        if(x >= 0.0 && x < 36.5)
        {
            const int idx = (int)(10.0 * (x + 0.05));
            const double dx = (double)idx * 0.1 - x;
            const double * g = tab + idx * 32;
            #pragma unroll
            for(int n = 0; n <= L; n++)
                F[n] = boys_taylor(g + n, dx);
        }
        else
        {
            const double x1 = 1.0 / x;
            double x2 = sqrt(x1);
            #pragma unroll
            for(int n = 0; n <= L; n++)
            {
                F[n] = __ldg(tab + SB_BOYS_LONGFAC_OFF + n) * x2;
                x2 *= x1;
            }
        }
    }
    else
    {
        if(x >= 0.0 && x < 36.5)
        {
            const int idx = (int)(10.0 * (x + 0.05));
            const double dx = (double)idx * 0.1 - x;
            F[L] = boys_taylor(tab + idx * 32 + L, dx);
        }
        else
            F[L] = __ldg(tab + SB_BOYS_LONGFAC_OFF + L) * pow(x, -((double)L + 0.5));
        const double x2 = 2.0 * x;
        const double ex = exp(-x);
        #pragma unroll
        for(int n = L - 1; n >= 0; n--)
            F[n] = (1.0 / (2.0 * n + 1.0)) * fma(x2, F[n + 1], ex);
    }
}

__device__ __forceinline__ BraPrim load_bra_prim(const QuartetCtx & c, int i)
{
    const double * r = c.bprim + (size_t)i * SB_REC;
    BraPrim b;
    b.alpha = r[0]; b.prefac = r[1];
    b.x = r[2]; b.y = r[3]; b.z = r[4];
    if(!c.swapB)
    {
        b.PAx = r[5]; b.PAy = r[6]; b.PAz = r[7];
        b.PBx = r[8]; b.PBy = r[9]; b.PBz = r[10];
        b.a2 = r[11]; b.b2 = r[12];
    }
    else
    {
        b.PAx = r[8]; b.PAy = r[9]; b.PAz = r[10];
        b.PBx = r[5]; b.PBy = r[6]; b.PBz = r[7];
        b.a2 = r[12]; b.b2 = r[11];
    }
    b.screen = r[13]; b.vecmax = r[14]; b.sq = r[15];
    // bra-level test of the reference (OSTEI_Writer.cpp:504-518) applies to
    // the requested bra set P
    b.skip = !c.pq && (b.screen * c.kscreen_max < c.tol2);
    return b;
}

// Screening test of ket primitive j against bra primitive bp (only called
// when screening is on): the reference's 8-wide vector test, plus its
// bra-level test when the requested bra set plays the ket role.  The
// reference's (ss|ss) kernel zeroes the screening values of the lanes past
// the last ket primitive before the test of a partial vector
// (skel/ostei_s_s_s_s.c), so for a ket list clipped inside a vector the
// test of that vector covers the slots below the clip only.
__device__ __forceinline__ bool prim_survives(const QuartetCtx & c, const BraPrim & bp, int j)
{
    const double * r = c.kprim + (size_t)j * SB_REC;
    const double ks = r[13];
    double kv = r[14];
    if(j >= c.kvec0 && j < c.kvec1)
    {
        kv = 0.0;
        for(int s = c.kvec0; s < c.kvec1; s++)
            kv = fmax(kv, c.kprim[(size_t)s * SB_REC + 13]);
    }
    const double v = c.pq ? ks * bp.vecmax : bp.screen * kv;
    if(v < c.tol2)
        return false;
    if(c.pq && ks * c.bscreen_max < c.tol2)
        return false;
    return true;
}

// Ket primitive j against bra primitive bp: screening, then the
// per-primitive-quartet set-up of OSTEI_Writer.cpp:586-702.
__device__ __forceinline__ bool prim_setup(const QuartetCtx & c, const BraPrim & bp, int j,
                                           PrimSetup & s)
{
    const double * r = c.kprim + (size_t)j * SB_REC;
    if(c.check && !prim_survives(c, bp, j))
        return false;
    const double q = r[0];
    const double p = bp.alpha;
    const double sum = p + q;
    const double one_over_sum = 1.0 / sum;
    const double PQx = bp.x - r[2], PQy = bp.y - r[3], PQz = bp.z - r[4];
    double R2 = PQx * PQx;
    R2 = fma(PQy, PQy, R2);
    R2 = fma(PQz, PQz, R2);
    const double alpha = (p * q) * one_over_sum;
    const double one_over_p = 1.0 / p;
    const double one_over_q = 1.0 / q;
    s.oo2p = 0.5 * one_over_p;
    s.oo2q = 0.5 * one_over_q;
    s.oo2pq = 0.5 * one_over_sum;
    s.a_over_p = -alpha * one_over_p;
    s.aopPQx = s.a_over_p * PQx; s.aopPQy = s.a_over_p * PQy; s.aopPQz = s.a_over_p * PQz;
    const double aoq = alpha * one_over_q;
    s.aoqPQx = aoq * PQx; s.aoqPQy = aoq * PQy; s.aoqPQz = aoq * PQz;
    s.a_over_q = -aoq;
    s.PAx = bp.PAx; s.PAy = bp.PAy; s.PAz = bp.PAz;
    s.PBx = bp.PBx; s.PBy = bp.PBy; s.PBz = bp.PBz;
    if(!c.swapK)
    {
        s.QCx = r[5]; s.QCy = r[6]; s.QCz = r[7];
        s.QDx = r[8]; s.QDy = r[9]; s.QDz = r[10];
        s.c2c = r[11]; s.c2d = r[12];
    }
    else
    {
        s.QCx = r[8]; s.QCy = r[9]; s.QCz = r[10];
        s.QDx = r[5]; s.QDy = r[6]; s.QDz = r[7];
        s.c2c = r[12]; s.c2d = r[11];
    }
    s.c2a = bp.a2; s.c2b = bp.b2;
    s.T = R2 * alpha;
    double pf = sqrt(one_over_sum);
    s.prefac = (bp.prefac * r[1]) * pf;
    // mixed precision gate: estimated absolute error of an FP32 VRR for
    // this primitive quartet.  Every (ss|ss)^(m) is at most |prefac|
    // (F_m <= 1); a recursion step adds X and Y multiples of the level below
    // and at most h = L (1/2p + 1/2q + 1/2(p+q)) times the level two below,
    // so the largest value of level k is at most r^k |prefac| with r the
    // root of r^2 = g r + h, g = 1 + max|X| + max|Y|; the HRR multiplies by
    // at most gamp; FP32 rounding adds about 8 (L+1) units of 2^-24 relative
    // to the largest intermediate.
    s.lowprec = false;
    if(c.gate > 0.0)
    {
        const double mx = fmax(fmax(fmax(fabs(s.PAx), fabs(s.PAy)), fmax(fabs(s.PAz), fabs(s.PBx))),
                               fmax(fmax(fabs(s.PBy), fabs(s.PBz)), fmax(fabs(s.QCx), fabs(s.QCy))));
        const double mq = fmax(fmax(fmax(fabs(s.QCz), fabs(s.QDx)), fabs(s.QDy)), fabs(s.QDz));
        const double my = fmax(fmax(fmax(fabs(s.aopPQx), fabs(s.aopPQy)), fabs(s.aopPQz)),
                               fmax(fmax(fabs(s.aoqPQx), fabs(s.aoqPQy)), fabs(s.aoqPQz)));
        const double g = 1.0 + fmax(mx, mq) + my;
        const double h = c.gL * (s.oo2p + s.oo2q + s.oo2pq);
        const double r = 0.5 * (g + sqrt(fma(g, g, 4.0 * h)));
        double est = fabs(s.prefac) * c.gamp * (8.0 * (c.gL + 1) * 5.9604644775390625e-08);
        for(int k = 0; k < c.gL; k++)
            est *= r;
        s.lowprec = est < c.gate;
    }
    return true;
}

// HRR growth factor of a shell quartet for the mixed-precision estimate:
// the transfer multiplies by |AB| (|CD|) once per step, nb (nd) steps.
__device__ __forceinline__ double hrr_amp(const QuartetCtx & c, int nb, int nd)
{
    const double ab = 1.0 + fmax(fmax(fabs(c.AB[0]), fabs(c.AB[1])), fabs(c.AB[2]));
    const double cd = 1.0 + fmax(fmax(fabs(c.CD[0]), fabs(c.CD[1])), fabs(c.CD[2]));
    double r = 1.0;
    for(int k = 0; k < nb; k++) r *= ab;
    for(int k = 0; k < nd; k++) r *= cd;
    return r;
}

// Fill a QuartetCtx for requested bra pair iP and ket pair iQ.
__device__ __forceinline__ void make_ctx(const KernArgs & a, int iP, int iQ, QuartetCtx & c)
{
    const PairSetDev & B = a.pq ? a.Q : a.P;
    const PairSetDev & K = a.pq ? a.P : a.Q;
    const int ib = a.pq ? iQ : iP;
    const int ik = a.pq ? iP : iQ;
    c.bprim = B.prim;
    c.kprim = K.prim;
    c.bi0 = B.pstart[ib];
    c.bi1 = c.bi0 + B.nprim[ib];
    c.kj0 = K.pstart[ik];
    c.kj1 = c.kj0 + K.nprim[ik];
    const double sb = a.swapB ? -1.0 : 1.0;
    const double sk = a.swapK ? -1.0 : 1.0;
    c.AB[0] = sb * B.AB[3 * ib + 0]; c.AB[1] = sb * B.AB[3 * ib + 1]; c.AB[2] = sb * B.AB[3 * ib + 2];
    c.CD[0] = sk * K.AB[3 * ik + 0]; c.CD[1] = sk * K.AB[3 * ik + 1]; c.CD[2] = sk * K.AB[3 * ik + 2];
    c.swapB = a.swapB; c.swapK = a.swapK; c.pq = a.pq;
    c.check = a.check; c.tol2 = a.tol2;
    c.bscreen_max = B.screen_max;
    c.kscreen_max = K.screen_max;
    c.gate = a.gate;
    c.gL = 0;
    c.gamp = 1.0;
    c.oidx = a.oidx;
    c.boys = a.boys;
    c.kvec0 = a.kvec0;
    c.kvec1 = a.kvec1;
    if(a.kvend)
    {
        const int je = __ldg(a.kvend + iP);
        if(je & 7)
        {
            c.kvec0 = je & ~7;
            c.kvec1 = je;
        }
    }
    c.fp32_count = a.fp32_count;
}

// Map a thread to a shell quartet.  MODE 0: the P x Q rectangle of
// simint_compute_eri (or the P x (nQc kets) part of it one launch of a
// chunked call covers), kets visited in the order kord (sorted by primitive
// count so a warp's loops have equal trip counts); output at
// (iP*nQ + iQ)*nout.  MODE 1: an explicit task list.
template<int MODE>
__device__ __forceinline__ bool task_of(const KernArgs & a, long long t, int & iP, int & iQ,
                                        long long & off)
{
    if(t >= a.ntask)
        return false;
    if(MODE == 0)
    {
        iP = (int)(t / a.nQc);
        iQ = a.kord[t - (long long)iP * a.nQc];
        off = ((long long)iP * a.nQ + iQ) * a.nout;
    }
    else if(MODE == 1)
    {
        const int2 tk = a.tasks[t];
        iP = tk.x;
        iQ = tk.y;
        off = a.outoff ? a.outoff[t] : t * (long long)a.nout;
    }
    else
    {
        // largest b with prefix[b] <= tg (binary search over nb+1 entries)
        const long long tg = a.task0 + t;
        int lo = 0, hi = a.nb;
        while(hi - lo > 1)
        {
            const int mid = (lo + hi) >> 1;
            if(__ldg(a.prefix + mid) <= tg) lo = mid; else hi = mid;
        }
        iP = __ldg(a.border + lo);
        iQ = __ldg(a.korder + (int)(tg - __ldg(a.prefix + lo)));
        off = t * (long long)a.nout;
    }
    return true;
}
