// One-electron integrals on the device: overlap, kinetic energy and nuclear
// attraction over contracted Cartesian shells.
//
// Reference: skel/simint/osoei/ (osoei_overlap.c:9-67, osoei_ke.c:10-68,
// osoei_potential.c:10-219, 1-D terms osoei_terms.c:9-165) behind
// simint_compute_overlap / simint_compute_ke / simint_compute_potential
// (skel/simint/simint_oneelectron.c:4-30).  Output: the ncart(a) x ncart(b)
// block, row-major, Cartesians in the fixed lexicographic order of
// skel/simint/recur_lookup.c (x descending, then y).
//
// Mapping: one warp per shell pair for overlap and kinetic energy, lanes over
// the primitive pairs; one 4-warp block per shell pair for the nuclear
// attraction, threads over the (centre, primitive pair) items.  Threads
// accumulate in registers; warps sum with a butterfly of shuffles and the
// warps of a block in warp order, so results do not depend on scheduling.
//  * overlap / kinetic energy: products of the 1-D Obara-Saika tables
//    S_d(i, j), T_d(i, j) of each primitive pair, as in the reference;
//  * nuclear attraction: the two-centre Obara-Saika recursion of the
//    reference, (a|0)^(m) then (a|b)^(m) with P - A and P - B, for every
//    (centre, primitive pair) item; the step direction is the first non-zero
//    exponent (the reference takes it from its lookup table, which changes
//    only the rounding).  A bra-only recursion followed by one horizontal
//    transfer per shell pair was tried and rejected: its AB terms cancel for
//    distant shells ((f|f) lost 1e-12 against the reference).
// Classes are compile-time (la >= lb; the transposed classes are the same
// blocks transposed, every operator here being symmetric), so the recursion
// indices fold to constants.

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "simint/simint.h"
#include "simint/simint_oneelectron.h"
#include "simint_b200.h"
#include "runtime.h"

namespace sb200 {
namespace {

#define OEI_MAXL 4

__host__ __device__ constexpr int onc(int l) { return ((l + 1) * (l + 2)) / 2; }
// lexicographic position of (x, y, z), l = x + y + z
__host__ __device__ constexpr int olex(int x, int z, int l) { return ((l - x) * (l - x + 1)) / 2 + z; }
// exponents of the k-th Cartesian of level l in that order
__host__ __device__ constexpr int ocx(int l, int k)
{
    int x = l;
    while(k >= l - x + 1) { k -= l - x + 1; x--; }
    return x;
}
__host__ __device__ constexpr int ocz(int l, int k)
{
    int x = l;
    while(k >= l - x + 1) { k -= l - x + 1; x--; }
    return k;
}
struct OeiArgs
{
    const double * shd;        // per shell: x, y, z
    const int4 * shi;          // per shell: am, nprim, first primitive, first basis function
    const double2 * prim;      // (alpha, coef) per primitive
    const int2 * pairs;        // (a, b), am[a] = LA, am[b] = LB
    int npair;
    const double4 * cen;       // (x, y, z, Z) per point charge
    int ncenter;
    double * out;
    long long ld;              // row stride of the matrix (mode 2)
    int mode;                  // 0 block, 1 transposed block, 2 symmetric matrix
    const double * boys;
    signed char pos[OEI_MAXL + 1][onc(OEI_MAXL)];   // output position of each Cartesian
};

__device__ __forceinline__ double warp_sum(double v)
{
    #pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Lanes write the ncart(a) x ncart(b) block `blk` (shared memory) of pair t.
__device__ __forceinline__ void oei_write(const OeiArgs & g, int t, int sa, int sb, int la, int lb,
                                          const double * blk, int lane)
{
    const int na = onc(la), nb = onc(lb);
    for(int k = lane; k < na * nb; k += 32)
    {
        const int u = k / nb, v = k - u * nb;
        if(g.mode == 0)
            g.out[(long long)t * na * nb + k] = blk[k];
        else if(g.mode == 1)
            g.out[(long long)t * na * nb + v * na + u] = blk[k];
        else if(sa != sb || u >= v)
        {
            // a shell with itself: its lower triangle, mirrored, so the
            // matrix is exactly symmetric
            const long long r = g.shi[sa].w + g.pos[la][u], c = g.shi[sb].w + g.pos[lb][v];
            g.out[r * g.ld + c] = blk[k];
            g.out[c * g.ld + r] = blk[k];
        }
    }
}

// Sum of acc over the warp into sm[0..N) (each lane stores its share).
template<int N>
__device__ __forceinline__ void warp_reduce_to(double (&acc)[N], double * sm, int lane)
{
    #pragma unroll
    for(int k = 0; k < N; k++)
    {
        const double v = warp_sum(acc[k]);
        if((k & 31) == lane)
            sm[k] = v;
    }
    __syncwarp();
}

// Overlap (KIND 0) and kinetic energy (KIND 1): osoei_overlap.c:36-64,
// osoei_ke.c:37-65, tables osoei_terms.c:9-165.
template<int LA, int LB, int KIND>
__global__ void __launch_bounds__(128) k_oei_st(const OeiArgs g)
{
    constexpr int NA = onc(LA), NB = onc(LB);
    const int lane = threadIdx.x & 31;
    const int t = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if(t >= g.npair)
        return;
    const int2 pr = g.pairs[t];
    const int4 ia = g.shi[pr.x], ib = g.shi[pr.y];
    const double A[3] = {g.shd[3 * pr.x], g.shd[3 * pr.x + 1], g.shd[3 * pr.x + 2]};
    const double B[3] = {g.shd[3 * pr.y], g.shd[3 * pr.y + 1], g.shd[3 * pr.y + 2]};
    double acc[NA * NB];
    #pragma unroll
    for(int k = 0; k < NA * NB; k++)
        acc[k] = 0.0;
    const int nitem = ia.y * ib.y;
    for(int it = lane; it < nitem; it += 32)
    {
        const int i = it / ib.y, j = it - i * ib.y;
        const double2 pa = g.prim[ia.z + i], pb = g.prim[ib.z + j];
        const double a1 = pa.x, a2 = pb.x;
        const double oop = 1.0 / (a1 + a2), mu = a1 * a2 * oop, o2p = 0.5 * oop;
        double S[3][LA + 1][LB + 1];
        double T[3][LA + 1][LB + 1];
        #pragma unroll
        for(int d = 0; d < 3; d++)
        {
            // P - A = -a2 AB / p and P - B = a1 AB / p: the reference's
            // values (osoei_terms.c:39-41) without the cancellation of
            // forming P first (exact zeros for shells on one centre, whose
            // odd components must vanish)
            const double AB = A[d] - B[d];
            const double PA = -a2 * AB * oop, PB = a1 * AB * oop;
            S[d][0][0] = sqrt(M_PI * oop) * exp(-mu * AB * AB);
            // a1 - 2 a1^2 (PA^2 + 1/2p) (osoei_terms.c:117) equals
            // mu (1 - 2 mu AB^2) with PA = -a2 AB / p: the same value without
            // the cancellation of two terms of size a1 when a1 >> a2, and
            // symmetric in the two exponents (so a transposed class rounds
            // like the direct one)
            if(KIND == 1)
                T[d][0][0] = S[d][0][0] * (mu * (1.0 - 2.0 * mu * AB * AB));
            #pragma unroll
            for(int ii = 1; ii <= LA; ii++)
            {
                double s = PA * S[d][ii - 1][0];
                if(ii > 1)
                    s += (ii - 1) * o2p * S[d][ii - 2][0];
                S[d][ii][0] = s;
                if(KIND == 1)
                {
                    double tt = PA * T[d][ii - 1][0] + 2.0 * mu * s;
                    if(ii > 1)
                        tt += (ii - 1) * o2p * T[d][ii - 2][0] - a2 * oop * (ii - 1) * S[d][ii - 2][0];
                    T[d][ii][0] = tt;
                }
            }
            #pragma unroll
            for(int jj = 1; jj <= LB; jj++)
                #pragma unroll
                for(int ii = 0; ii <= LA; ii++)
                {
                    double s = PB * S[d][ii][jj - 1];
                    if(ii > 0)
                        s += ii * o2p * S[d][ii - 1][jj - 1];
                    if(jj > 1)
                        s += (jj - 1) * o2p * S[d][ii][jj - 2];
                    S[d][ii][jj] = s;
                    if(KIND == 1)
                    {
                        double tt = PB * T[d][ii][jj - 1] + 2.0 * mu * s;
                        if(ii > 0)
                            tt += ii * o2p * T[d][ii - 1][jj - 1];
                        if(jj > 1)
                            tt += (jj - 1) * o2p * T[d][ii][jj - 2] - a1 * oop * (jj - 1) * S[d][ii][jj - 2];
                        T[d][ii][jj] = tt;
                    }
                }
        }
        const double c = pa.y * pb.y;
        #pragma unroll
        for(int u = 0; u < NA; u++)
            #pragma unroll
            for(int v = 0; v < NB; v++)
            {
                const int x1 = ocx(LA, u), z1 = ocz(LA, u), y1 = LA - x1 - z1;
                const int x2 = ocx(LB, v), z2 = ocz(LB, v), y2 = LB - x2 - z2;
                double val;
                if(KIND == 0)
                    val = S[0][x1][x2] * S[1][y1][y2] * S[2][z1][z2];
                else
                    val = T[0][x1][x2] * S[1][y1][y2] * S[2][z1][z2]
                        + S[0][x1][x2] * T[1][y1][y2] * S[2][z1][z2]
                        + S[0][x1][x2] * S[1][y1][y2] * T[2][z1][z2];
                acc[u * NB + v] = fma(c, val, acc[u * NB + v]);
            }
    }
    extern __shared__ double oei_sm[];
    double * sm = oei_sm + (threadIdx.x >> 5) * (NA * NB);
    warp_reduce_to<NA * NB>(acc, sm, lane);
    oei_write(g, t, pr.x, pr.y, LA, LB, sm, lane);
}

// offset of block (|a| = la, |b| = lb) in the two-centre table (a|b)^(m),
// m <= L - la - lb; blocks in order lb = 0..LB (outer), la = 0..LA
__host__ __device__ constexpr int o2off(int LA, int LB, int la, int lb)
{
    int o = 0;
    for(int j = 0; j <= LB; j++)
        for(int i = 0; i <= LA; i++)
        {
            if(j == lb && i == la) return o;
            o += onc(i) * onc(j) * (LA + LB - i - j + 1);
        }
    return o;
}

// Nuclear attraction: -sum_C Z_C (a| 1/|r - C| |b) (osoei_potential.c:10-219):
// the two-centre Obara-Saika recursion of every (centre, primitive pair)
// item, (a|0)^(m) by raising a, then (a|b)^(m) by raising b with P - B (no
// horizontal transfer, whose AB terms cancel for distant shells).
template<int LA, int LB>
__global__ void __launch_bounds__(128) k_oei_v(const OeiArgs g)
{
    constexpr int L = LA + LB;
    constexpr int NA = onc(LA), NB = onc(LB);
    constexpr int NW = o2off(LA, LB, LA, LB) + NA * NB;
    // small tables unroll completely (indices fold, table in registers);
    // large ones ((d|f) and up) keep runtime loops over a local-memory table,
    // which is where the table would live anyway, and compile quickly
    constexpr int UNR = NW <= 320 ? 64 : 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    // one block per shell pair: its items spread over all the block's warps
    // (a pair has thousands of (centre, primitive pair) items, a class may
    // have only hundreds of pairs)
    const int t = blockIdx.x;
    if(t >= g.npair)
        return;
    const int2 pr = g.pairs[t];
    const int4 ia = g.shi[pr.x], ib = g.shi[pr.y];
    const double A[3] = {g.shd[3 * pr.x], g.shd[3 * pr.x + 1], g.shd[3 * pr.x + 2]};
    const double B[3] = {g.shd[3 * pr.y], g.shd[3 * pr.y + 1], g.shd[3 * pr.y + 2]};
    const double AB2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1])
                     + (A[2] - B[2]) * (A[2] - B[2]);
    double acc[NA * NB];
    #pragma unroll
    for(int k = 0; k < NA * NB; k++)
        acc[k] = 0.0;
    const int npp = ia.y * ib.y;
    const int nitem = npp * g.ncenter;
    for(int it = threadIdx.x; it < nitem; it += blockDim.x)
    {
        const int c = it / npp, r = it - c * npp;
        const int i = r / ib.y, j = r - i * ib.y;
        const double2 pa = g.prim[ia.z + i], pb = g.prim[ib.z + j];
        const double4 C = g.cen[c];
        const double a1 = pa.x, a2 = pb.x, p = a1 + a2;
        const double oop = 1.0 / p, mu = a1 * a2 * oop, o2p = 0.5 * oop;
        const double Cx[3] = {C.x, C.y, C.z};
        double PA[3], PB[3], PC[3];
        #pragma unroll
        for(int d = 0; d < 3; d++)
        {
            // as in k_oei_st: P - A, P - B from AB, P - C = (P - A) + (A - C)
            const double AB = A[d] - B[d];
            PA[d] = -a2 * AB * oop;
            PB[d] = a1 * AB * oop;
            PC[d] = PA[d] + (A[d] - Cx[d]);
        }
        const double PC2 = PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2];
        double W[NW];
        boys_split<L>(g.boys, p * PC2, W);          // F_0..F_L in the (0|0) slots
        const double base = 2.0 * M_PI * oop * exp(-mu * AB2);
        #pragma unroll
        for(int m = 0; m <= L; m++)
            W[m] *= base;
        // (a|0)^(m), m <= L - |a|: raise a along its first non-zero exponent
        #pragma unroll UNR
        for(int l = 1; l <= LA; l++)
        {
            const int b0 = o2off(LA, LB, l, 0), b1 = o2off(LA, LB, l - 1, 0);
            const int b2 = l >= 2 ? o2off(LA, LB, l - 2, 0) : 0;
            #pragma unroll UNR
            for(int k = 0; k < onc(l); k++)
            {
                const int x = ocx(l, k), z = ocz(l, k), y = l - x - z;
                const int d = x ? 0 : (y ? 1 : 2);
                const int ed = d == 0 ? x : (d == 1 ? y : z);
                const int k1 = olex(x - (d == 0), z - (d == 2), l - 1);
                const int o0 = b0 + k * (L - l + 1);
                const int o1 = b1 + k1 * (L - l + 2);
                const int o2 = ed >= 2 ? b2 + olex(x - 2 * (d == 0), z - 2 * (d == 2), l - 2) * (L - l + 3) : 0;
                #pragma unroll UNR
                for(int m = 0; m <= L - l; m++)
                {
                    double v = PA[d] * W[o1 + m] - PC[d] * W[o1 + m + 1];
                    if(ed >= 2)
                        v += (ed - 1) * o2p * (W[o2 + m] - W[o2 + m + 1]);
                    W[o0 + m] = v;
                }
            }
        }
        // (a|b)^(m), m <= L - |a| - |b|: raise b along its first non-zero exponent
        #pragma unroll UNR
        for(int lb = 1; lb <= LB; lb++)
            #pragma unroll UNR
            for(int la = 0; la <= LA; la++)
            {
                const int nm = L - la - lb + 1;
                const int b0 = o2off(LA, LB, la, lb), b1 = o2off(LA, LB, la, lb - 1);
                const int b2 = lb >= 2 ? o2off(LA, LB, la, lb - 2) : 0;
                const int b3 = la >= 1 ? o2off(LA, LB, la - 1, lb - 1) : 0;
                #pragma unroll UNR
                for(int kb = 0; kb < onc(lb); kb++)
                {
                    const int xb = ocx(lb, kb), zb = ocz(lb, kb), yb = lb - xb - zb;
                    const int d = xb ? 0 : (yb ? 1 : 2);
                    const int bd = (d == 0 ? xb : (d == 1 ? yb : zb)) - 1;   // exponent of b - 1_d
                    const int kb1 = olex(xb - (d == 0), zb - (d == 2), lb - 1);
                    const int kb2 = bd >= 1 ? olex(xb - 2 * (d == 0), zb - 2 * (d == 2), lb - 2) : 0;
                    #pragma unroll UNR
                    for(int ka = 0; ka < onc(la); ka++)
                    {
                        const int xa = ocx(la, ka), za = ocz(la, ka), ya = la - xa - za;
                        const int ad = d == 0 ? xa : (d == 1 ? ya : za);
                        const int o0 = b0 + (ka * onc(lb) + kb) * nm;
                        const int o1 = b1 + (ka * onc(lb - 1) + kb1) * (nm + 1);
                        const int o3 = ad >= 1 ? b3 + (olex(xa - (d == 0), za - (d == 2), la - 1) * onc(lb - 1) + kb1) * (nm + 2) : 0;
                        const int o2 = bd >= 1 ? b2 + (ka * onc(lb - 2) + kb2) * (nm + 2) : 0;
                        #pragma unroll UNR
                        for(int m = 0; m < nm; m++)
                        {
                            double v = PB[d] * W[o1 + m] - PC[d] * W[o1 + m + 1];
                            if(ad >= 1)
                                v += ad * o2p * (W[o3 + m] - W[o3 + m + 1]);
                            if(bd >= 1)
                                v += bd * o2p * (W[o2 + m] - W[o2 + m + 1]);
                            W[o0 + m] = v;
                        }
                    }
                }
            }
        const double f = -C.w * pa.y * pb.y;
        #pragma unroll
        for(int k = 0; k < NA * NB; k++)
            acc[k] = fma(f, W[o2off(LA, LB, LA, LB) + k], acc[k]);
    }
    // warp sums, then the warps' sums in warp order (deterministic)
    extern __shared__ double oei_sm[];
    warp_reduce_to<NA * NB>(acc, oei_sm + warp * (NA * NB), lane);
    __syncthreads();
    if(warp != 0)
        return;
    for(int k = lane; k < NA * NB; k += 32)
    {
        double v = oei_sm[k];
        for(int w = 1; w < nwarp; w++)
            v += oei_sm[w * (NA * NB) + k];
        oei_sm[k] = v;
    }
    __syncwarp();
    oei_write(g, t, pr.x, pr.y, LA, LB, oei_sm, lane);
}

typedef void (*OeiKern)(OeiArgs);

struct OeiTable
{
    OeiKern k[3][OEI_MAXL + 1][OEI_MAXL + 1] = {};
};

template<int LA, int LB>
void oei_register(OeiTable & t)
{
    t.k[0][LA][LB] = k_oei_st<LA, LB, 0>;
    t.k[1][LA][LB] = k_oei_st<LA, LB, 1>;
    t.k[2][LA][LB] = k_oei_v<LA, LB>;
}

const OeiTable & oei_table()
{
    static OeiTable t = [] {
        OeiTable x;
        oei_register<0, 0>(x);
        oei_register<1, 0>(x); oei_register<1, 1>(x);
        oei_register<2, 0>(x); oei_register<2, 1>(x); oei_register<2, 2>(x);
        oei_register<3, 0>(x); oei_register<3, 1>(x); oei_register<3, 2>(x); oei_register<3, 3>(x);
        oei_register<4, 0>(x); oei_register<4, 1>(x); oei_register<4, 2>(x); oei_register<4, 3>(x);
        oei_register<4, 4>(x);
        return x;
    }();
    return t;
}

// Working memory of the one-electron calls of one host thread.  The inputs
// of a call stay in `dev` until its kernels are done (`done` is waited on
// before the next call overwrites them).
struct OeiBufs
{
    DevBuf dev;
    HostBuf host;
    cudaEvent_t done = nullptr;
    bool pending = false;
    ~OeiBufs()
    {
        if(pending && done)
            cudaEventSynchronize(done);
        dev.release();
        host.release();
        if(done)
            cudaEventDestroy(done);
    }
};

OeiBufs & oei_bufs()
{
    static thread_local OeiBufs b;
    return b;
}

size_t a256(size_t n) { return (n + 255) & ~(size_t)255; }

// Upload shells, primitives, centres and the pair list; return the device
// views.  `pairs` hold (a, b) with am[a] >= am[b], grouped by class.
int oei_upload(OeiBufs & B, int nshell, const simint_shell * const * shells, int ncenter,
               const double * Z, const double * x, const double * y, const double * z,
               const std::vector<int2> & pairs, size_t out_bytes, cudaStream_t stream,
               OeiArgs & g, double ** dout)
{
    if(!B.done && cudaEventCreateWithFlags(&B.done, cudaEventDisableTiming) != cudaSuccess)
    {
        set_error("cudaEventCreate failed");
        return SIMINT_B200_ERR_CUDA;
    }
    if(B.pending)
    {
        cudaEventSynchronize(B.done);
        B.pending = false;
    }
    int nprim = 0;
    for(int s = 0; s < nshell; s++)
        nprim += shells[s]->nprim;
    const size_t o_shd = 0;
    const size_t o_shi = a256(o_shd + sizeof(double) * 3 * (size_t)nshell);
    const size_t o_prim = a256(o_shi + sizeof(int4) * (size_t)nshell);
    const size_t o_pair = a256(o_prim + sizeof(double2) * (size_t)std::max(nprim, 1));
    const size_t o_cen = a256(o_pair + sizeof(int2) * std::max<size_t>(pairs.size(), 1));
    const size_t o_out = a256(o_cen + sizeof(double4) * (size_t)std::max(ncenter, 1));
    const size_t up = o_out;
    const size_t tot = o_out + a256(out_bytes);
    // the staging buffer also receives the block of a per-pair call
    if(!B.dev.reserve(tot) || !B.host.reserve(std::max(up, out_bytes)))
    {
        set_error("out of memory in a one-electron call");
        return SIMINT_B200_ERR_CUDA;
    }
    char * h = (char *)B.host.ptr;
    double * shd = (double *)(h + o_shd);
    int4 * shi = (int4 *)(h + o_shi);
    double2 * prim = (double2 *)(h + o_prim);
    int p = 0, ao = 0;
    for(int s = 0; s < nshell; s++)
    {
        const simint_shell * S = shells[s];
        shd[3 * s] = S->x; shd[3 * s + 1] = S->y; shd[3 * s + 2] = S->z;
        shi[s] = make_int4(S->am, S->nprim, p, ao);
        for(int k = 0; k < S->nprim; k++)
            prim[p + k] = make_double2(S->alpha[k], S->coef[k]);
        p += S->nprim;
        ao += onc(S->am);
    }
    if(!pairs.empty())
        memcpy(h + o_pair, pairs.data(), sizeof(int2) * pairs.size());
    double4 * cen = (double4 *)(h + o_cen);
    for(int c = 0; c < ncenter; c++)
        cen[c] = make_double4(x[c], y[c], z[c], Z[c]);
    char * d = (char *)B.dev.ptr;
    if(cudaMemcpyAsync(d, h, up, cudaMemcpyHostToDevice, stream) != cudaSuccess)
    {
        set_error("one-electron upload failed");
        return SIMINT_B200_ERR_CUDA;
    }
    g = OeiArgs{};
    g.shd = (const double *)(d + o_shd);
    g.shi = (const int4 *)(d + o_shi);
    g.prim = (const double2 *)(d + o_prim);
    g.pairs = (const int2 *)(d + o_pair);
    g.cen = (const double4 *)(d + o_cen);
    g.ncenter = ncenter;
    g.boys = boys_table();
    *dout = (double *)(d + o_out);
    return 0;
}

int oei_launch(int kind, int la, int lb, OeiArgs g, int first, int npair, cudaStream_t stream)
{
    if(npair <= 0)
        return 0;
    OeiKern k = oei_table().k[kind][la][lb];
    g.pairs += first;
    g.npair = npair;
    if(g.mode != 2)
        g.out += (long long)first * onc(la) * onc(lb);
    const int threads = 128;
    // overlap, kinetic energy: a warp per shell pair; nuclear attraction: a
    // block per shell pair
    const long long blocks = kind == 2 ? npair : ((long long)npair * 32 + threads - 1) / threads;
    const size_t smem = sizeof(double) * (threads / 32) * onc(la) * onc(lb);
    k<<<(unsigned)blocks, threads, smem, stream>>>(g);
    count_launch(1);
    if(cudaGetLastError() != cudaSuccess)
    {
        set_error("one-electron kernel launch failed");
        return SIMINT_B200_ERR_CUDA;
    }
    return 1;
}

void lex_positions(OeiArgs & g, int ord)
{
    for(int l = 0; l <= OEI_MAXL; l++)
        for(int k = 0; k < onc(l); k++)
        {
            const int xx = ocx(l, k), zz = ocz(l, k);
            g.pos[l][k] = (signed char)(ord < 0 ? k : cart_index(xx, l - xx - zz, zz, ord));
        }
}

// One shell pair through the reference's per-pair interface: host shells and
// centres in, the ncart(a) x ncart(b) block out.
int oei_pair(int kind, int ncenter, const double * Z, const double * x, const double * y,
             const double * z, const simint_shell * sa, const simint_shell * sb, double * integrals)
{
    init_tables();
    if(ensure_device() < 0)
        return SIMINT_B200_ERR_NODEVICE;
    if(!sa || !sb || !integrals || ncenter < 0 || (kind == 2 && ncenter > 0 && (!Z || !x || !y || !z)))
    {
        set_error("bad argument to a one-electron call");
        return SIMINT_B200_ERR_ARG;
    }
    if(sa->am < 0 || sb->am < 0 || sa->am > OEI_MAXL || sb->am > OEI_MAXL)
    {
        set_error("one-electron integrals are built for am <= 4");
        return SIMINT_B200_ERR_CLASS;
    }
    Workspace & w = workspace();
    if(!w.stream && cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess)
    {
        set_error("cudaStreamCreate failed");
        return SIMINT_B200_ERR_CUDA;
    }
    const bool swap = sa->am < sb->am;
    const simint_shell * sh[2] = {swap ? sb : sa, swap ? sa : sb};
    const int la = sh[0]->am, lb = sh[1]->am;
    const int n = onc(la) * onc(lb);
    std::vector<int2> pairs(1, make_int2(0, 1));
    OeiBufs & B = oei_bufs();
    OeiArgs g;
    double * dout = nullptr;
    int rc = oei_upload(B, 2, sh, kind == 2 ? ncenter : 0, Z, x, y, z, pairs, sizeof(double) * n,
                        w.stream, g, &dout);
    if(rc < 0)
        return rc;
    g.out = dout;
    g.mode = swap ? 1 : 0;
    rc = oei_launch(kind, la, lb, g, 0, 1, w.stream);
    if(rc < 0)
        return rc;
    double * hout = (double *)((char *)B.host.ptr);   // inputs already copied: reuse the staging
    cudaMemcpyAsync(hout, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, w.stream);
    if(cudaStreamSynchronize(w.stream) != cudaSuccess)
    {
        set_error("one-electron kernel failed");
        return SIMINT_B200_ERR_CUDA;
    }
    memcpy(integrals, hout, sizeof(double) * n);
    return 1;
}

} // namespace
} // namespace sb200

using namespace sb200;

// simint_oneelectron.c:4-11 -> osoei_overlap.c:9-67
extern "C" int simint_compute_overlap(struct simint_shell * a, struct simint_shell * b,
                                      double * integrals)
{
    return oei_pair(0, 0, nullptr, nullptr, nullptr, nullptr, a, b, integrals);
}

// simint_oneelectron.c:14-19 -> osoei_ke.c:10-68
extern "C" int simint_compute_ke(struct simint_shell * a, struct simint_shell * b,
                                 double * integrals)
{
    return oei_pair(1, 0, nullptr, nullptr, nullptr, nullptr, a, b, integrals);
}

// simint_oneelectron.c:22-30 -> osoei_potential.c:10-219
extern "C" int simint_compute_potential(int ncenter, double * Z, double * x, double * y, double * z,
                                        struct simint_shell const * sh1, struct simint_shell const * sh2,
                                        double * integrals)
{
    return oei_pair(2, ncenter, Z, x, y, z, sh1, sh2, integrals);
}

extern "C" int simint_b200_oei_matrix(int kind, int nshell, struct simint_shell const * shells,
                                      int ncenter, const double * Z, const double * x,
                                      const double * y, const double * z, double * dev_out,
                                      void * stream_)
{
    init_tables();
    if(ensure_device() < 0)
        return SIMINT_B200_ERR_NODEVICE;
    if(kind < 0 || kind > 2 || nshell < 0 || (nshell > 0 && !shells) || !dev_out || ncenter < 0
       || (kind == 2 && ncenter > 0 && (!Z || !x || !y || !z)))
    {
        set_error("bad argument to simint_b200_oei_matrix");
        return SIMINT_B200_ERR_ARG;
    }
    std::vector<const simint_shell *> sh(nshell);
    std::vector<std::vector<int2>> bycls((OEI_MAXL + 1) * (OEI_MAXL + 1));
    for(int s = 0; s < nshell; s++)
    {
        sh[s] = &shells[s];
        if(shells[s].am < 0 || shells[s].am > OEI_MAXL)
        {
            set_error("one-electron integrals are built for am <= 4");
            return SIMINT_B200_ERR_CLASS;
        }
    }
    for(int i = 0; i < nshell; i++)
        for(int j = 0; j <= i; j++)
        {
            int a = i, b = j;
            if(shells[a].am < shells[b].am)
                std::swap(a, b);
            bycls[shells[a].am * (OEI_MAXL + 1) + shells[b].am].push_back(make_int2(a, b));
        }
    std::vector<int2> pairs;
    std::vector<int> first(bycls.size() + 1, 0);
    for(size_t c = 0; c < bycls.size(); c++)
    {
        first[c] = (int)pairs.size();
        pairs.insert(pairs.end(), bycls[c].begin(), bycls[c].end());
    }
    first[bycls.size()] = (int)pairs.size();
    cudaStream_t stream = (cudaStream_t)stream_;
    OeiBufs & B = oei_bufs();
    OeiArgs g;
    double * dscr = nullptr;
    int rc = oei_upload(B, nshell, sh.data(), kind == 2 ? ncenter : 0, Z, x, y, z, pairs, 0, stream,
                        g, &dscr);
    if(rc < 0)
        return rc;
    int nbf = 0;
    for(int s = 0; s < nshell; s++)
        nbf += onc(shells[s].am);
    g.out = dev_out;
    g.ld = nbf;
    g.mode = 2;
    lex_positions(g, ordering());
    int nl = 0;
    for(int la = 0; la <= OEI_MAXL; la++)
        for(int lb = 0; lb <= la; lb++)
        {
            const int c = la * (OEI_MAXL + 1) + lb;
            rc = oei_launch(kind, la, lb, g, first[c], first[c + 1] - first[c], stream);
            if(rc < 0)
                return rc;
            nl += rc;
        }
    cudaEventRecord(B.done, stream);
    B.pending = true;
    return nl;
}
