// Shared pieces of the table-driven cooperative ERI kernel (coop2.cu) that
// other CTA-wide kernels reuse: the per-class parameter block (accumulator
// layout of the contracted top quartets and the HRR row tables), the HRR in
// shared memory, the Boys evaluation into shared memory and small helpers.
#pragma once

#include <cuda_runtime.h>

#include "simint_b200.h"
#include "ostei_device.cuh"
#include "cartinfo.cuh"

#define C2_MAXL 10
#define C2_MAXS 20
#define C2_NCOEF 32          // per primitive quartet: 6 combos x 4, 1/2(p+q), 4 deriv weights, pad
#define C2_SETUP 16          // primitive quartets set up in parallel
#define C2_MAXN 225          // Cartesian pairs of (g g)

enum { K_O2PQ = 24, K_W1 = 25 };

// One VRR item, 16 bytes:
//   x = dst | src1 << 16                  (offsets of the m = 0 slots in a wave buffer)
//   y = src2 | src3 << 16                 (0 when absent)
//   z = acc index of tag 0 (0xffff = none) | combo << 16 | has2 << 24 | has3 << 25
//       | (mask of tags 1..4) << 26
// One unit computes one auxiliary order m of one element (m is folded into
// the offsets).
//   w = nA | nB << 4 | gE << 8 | gF << 18 (integer factors; Cartesian indices of deriv tags)
typedef int4 C2Item;

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
    const C2Item * items;
    int off_acc, off_prep, off_surv, off_hrr_b, off_hrr_mid;   // shared-memory layout (doubles)
    int prep_stride;              // doubles per prepared primitive quartet
    int off32;                    // offset (doubles) of its FP32 coefficient copy
    int hrr_layer;                // doubles per HRR layer buffer
    int hrr_need;                 // doubles the HRR uses from off_hrr_b (layers + mid)
    int smem_doubles;
    int ordering;
    int res_size;                 // deriv 1: doubles of all target results per CTA
    int res_off[6];
    const int2 * hrr_rows;        // HRR row tables (see c2_hrr_side)
    int hrr_base[6][2];           // per target and side: first row
    int hrr_loff[6][2][6];        // per target and side: row offsets of layers (relative)
    int hrr_nl[6][2];             // per target and side: number of transfer layers
};

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

// One side of the HRR for every column at once, layer by layer in shared
// memory.  in(g, col) gives the tops (functions on the top centre, levels
// lo..lt); out(r, col, v) receives the (ta tb) block, r = pa * nc(tb) + pb.
// rows[loff[sl-1] .. loff[sl]) describe layer sl, one int2 per row:
// x = source A | source B << 16 (function indices on layer 1, rows of the
// previous layer after), y = direction | output row << 2 (last layer).
// Threads form a (row, column) grid.
struct C2SyncAll
{
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// c2_hrr_side for NT threads numbered tid, synchronised by sync() (a CTA
// barrier, or a named barrier of a group of NT threads).
template<int NT, typename IN, typename OUT, typename SYNC>
__device__ void c2_hrr_side_t(int tid, SYNC sync, int right_step, int sl_max, int ncol,
                              const int2 * __restrict__ rows, const int * loff, double X0, double X1,
                              double X2, IN in, OUT out, double * __restrict__ LA, double * __restrict__ LB)
{
    const int TC = ncol < NT ? ncol : NT;
    const int TR = NT / TC;
    const int tc = tid % TC, tr = tid / TC;
    const double Xs[3] = {right_step ? X0 : -X0, right_step ? X1 : -X1, right_step ? X2 : -X2};
    if(sl_max == 0)
    {
        // nothing to transfer: row r of the block is top function rows[r].x
        const int nr = loff[0];
        if(tr < TR)
            for(int r = tr; r < nr; r += TR)
            {
                const int g = __ldg(&rows[r].x);
                for(int col = tc; col < ncol; col += TC)
                    out(r, col, in(g, col));
            }
        sync();
        return;
    }
    double * dst = LA;
    const double * src = LB;
    for(int sl = 1; sl <= sl_max; sl++)
    {
        const int r0 = loff[sl - 1], r1 = loff[sl];
        const bool last = sl == sl_max;
        if(tr < TR)
            #pragma unroll 2
            for(int r = r0 + tr; r < r1; r += TR)
            {
                const int2 e = __ldg(&rows[r]);
                const int a = e.x & 0xffff, b = (int)((unsigned)e.x >> 16);
                const double X = Xs[e.y & 3];
                const int orow = e.y >> 2;
                if(sl == 1)
                {
                    for(int col = tc; col < ncol; col += TC)
                    {
                        const double v = fma(X, in(a, col), in(b, col));
                        if(last) out(orow, col, v);
                        else dst[(r - r0) * ncol + col] = v;
                    }
                }
                else
                {
                    const double * sa = src + a * ncol;
                    const double * sb = src + b * ncol;
                    for(int col = tc; col < ncol; col += TC)
                    {
                        const double v = fma(X, sa[col], sb[col]);
                        if(last) out(orow, col, v);
                        else dst[(r - r0) * ncol + col] = v;
                    }
                }
            }
        sync();
        double * t = (double *)src;
        src = dst;
        dst = t;
    }
}

template<int NT, typename IN, typename OUT>
__device__ __forceinline__ void c2_hrr_side(int right_step, int sl_max, int ncol, const int2 * __restrict__ rows,
                                            const int * loff, double X0, double X1, double X2, IN in, OUT out,
                                            double * __restrict__ LA, double * __restrict__ LB)
{
    c2_hrr_side_t<NT>((int)threadIdx.x, C2SyncAll(), right_step, sl_max, ncol, rows, loff, X0, X1, X2, in, out,
                      LA, LB);
}

// 1/(2n+1), n = 0..31: the same correctly rounded values as the division,
// without a division per order.
__device__ __forceinline__ double c2_recip_odd(int n)
{
    constexpr double r[32] = {
        1.0 / 1, 1.0 / 3, 1.0 / 5, 1.0 / 7, 1.0 / 9, 1.0 / 11, 1.0 / 13, 1.0 / 15, 1.0 / 17, 1.0 / 19,
        1.0 / 21, 1.0 / 23, 1.0 / 25, 1.0 / 27, 1.0 / 29, 1.0 / 31, 1.0 / 33, 1.0 / 35, 1.0 / 37, 1.0 / 39,
        1.0 / 41, 1.0 / 43, 1.0 / 45, 1.0 / 47, 1.0 / 49, 1.0 / 51, 1.0 / 53, 1.0 / 55, 1.0 / 57, 1.0 / 59,
        1.0 / 61, 1.0 / 63};
    return r[n & 31];
}

// Boys values F_0..F_L(T) times prefac into F (shared memory), the
// reference's split: L < 4 every order from the Taylor grid (or the
// asymptotic form for T >= 36.5), L >= 4 F_L then downward recursion
// (boys.h:14-92, boys_taylor.h:14-39, boys_long.h:14-58).
__device__ __forceinline__ void c2_boys(const double * __restrict__ tab, double T, int L, double prefac,
                                        double * __restrict__ F)
{
    if(L < 4)
    {
        if(T >= 0.0 && T < 36.5)
        {
            const int idx = (int)(10.0 * (T + 0.05));
            const double dx = (double)idx * 0.1 - T;
            for(int n = 0; n <= L; n++)
                F[n] = boys_taylor(tab + idx * 32 + n, dx) * prefac;
        }
        else
        {
            const double x1 = 1.0 / T;
            double x2 = sqrt(x1);
            for(int n = 0; n <= L; n++)
            {
                F[n] = (__ldg(tab + SB_BOYS_LONGFAC_OFF + n) * x2) * prefac;
                x2 *= x1;
            }
        }
        return;
    }
    double f;
    if(T >= 0.0 && T < 36.5)
    {
        const int idx = (int)(10.0 * (T + 0.05));
        const double dx = (double)idx * 0.1 - T;
        f = boys_taylor(tab + idx * 32 + L, dx);
    }
    else
        f = __ldg(tab + SB_BOYS_LONGFAC_OFF + L) * pow(T, -((double)L + 0.5));
    const double x2 = 2.0 * T;
    const double ex = exp(-T);
    F[L] = f * prefac;
    for(int n = L - 1; n >= 0; n--)
    {
        f = c2_recip_odd(n) * fma(x2, f, ex);
        F[n] = f * prefac;
    }
}

// Small non-negative integer n as a floating-point value without a
// conversion instruction: the bits of 2^52 + n (resp. 2^23 + n) minus 2^52
// (2^23), exact for n < 2^23.
__device__ __forceinline__ void c2_small(int n, double & d) { d = __hiloint2double(0x43300000, n) - 4503599627370496.0; }
__device__ __forceinline__ void c2_small(int n, float & f) { f = __int_as_float(0x4b000000 | n) - 8388608.0f; }


namespace sb200 {
// Parameters of class am (deriv 0) with the HRR row tables of the current
// device filled in: the accumulator layout and HRR the column kernel shares.
// false when the cooperative kernel's planner does not cover the class.
bool coop2_hrr_params(const int am[4], C2Params & out);
}
