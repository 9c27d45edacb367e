// Batched, device-resident ERI sweeps over a whole basis.
//
// The reference's callers express a sweep as many simint_compute_eri calls
// (one bra pair against a ket list, skel/test/benchmark_eri.cpp:135-216, or
// Psi4/GTFock integral loops).  Here a basis is uploaded once:
//   * shell pairs (i >= j) are grouped into pair classes (la >= lb) and built
//     with primitive Schwarz screening (values computed on the GPU),
//   * every shell pair gets its Schwarz bound Q_ab = sqrt(max |(ab|ab)|)
//     (simint_shellscreen_schwarz, shell_screen.c:48-83), also on the GPU,
//   * pairs are sorted by Q_ab, so for each bra pair the surviving ket pairs
//     (Q_ab Q_cd >= tol) are a prefix of the sorted ket list; a prefix-sum
//     array over bra pairs is the whole task list of a quartet class
//     (kernels decode task t by binary search: no explicit quartet list),
//   * inside a quartet the reference's primitive screening applies with the
//     same tolerance (pairs built with SIMINT_SCREEN_SCHWARZ).
// A sweep launches one kernel per class (or per output chunk), adds a
// checksum kernel per launch, and is captured into one CUDA graph.

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "simint/simint.h"
#include "simint_b200.h"
#include "runtime.h"

using namespace sb200;

namespace {

struct PairClass
{
    int la = 0, lb = 0;
    std::vector<int> sa, sb;         // shell indices of the two functions
    simint_multi_shellpair P;        // host pair data (Schwarz screened)
    DevBuf dev;                      // packed records + sorted order
    PairSetDev view;
    std::vector<double> Q;           // Schwarz bound per pair
    std::vector<int> order;          // pair indices by decreasing Q
    const int * dorder = nullptr;
    DevBuf dsh;                      // (sa, sb) per pair on the device (J/K digestion)
};

struct QClass
{
    int bx = 0, ky = 0;              // pair classes of bra and ket
    int req[4];
    long long ntask = 0, nprimq = 0, nfull = 0;
    int nout = 0;
    long long offset = 0;
    std::vector<long long> prefix;   // nb + 1
    std::vector<int> border;         // bra pair of each b
    bool has_perm = false;           // task order by primitive count uploaded
    bool ssss = false;               // (ss|ss) with screening: per-row clipped-vector ends uploaded
    DevBuf dev;                      // prefix, border, task order, (ss|ss) row ends
};

// Tasks of a class up to this count get a heaviest-first visiting order.
#define SWEEP_PERM_MAX (64LL << 20)
// Per class in the basis' queue buffer: the work queue, then the counter of
// primitive quartets run in FP32.
#define SWEEP_QSTRIDE (sizeof(WorkQueue) + sizeof(unsigned long long))

// A launch's queue: every task published and the queue closed (the status
// word and the FP32 counter keep what earlier launches of the sweep left).
__global__ void k_queue_reset(WorkQueue * q, long long ntask, unsigned long long spin_limit)
{
    q->next = 0;
    q->published = (unsigned long long)ntask;
    q->closed = 1;
    q->spin_limit = spin_limit;
}

// A queue in a given state, for the probe of the bounded wait.
__global__ void k_queue_set(WorkQueue * q, long long published, int closed, unsigned long long spin_limit)
{
    q->next = 0;
    q->published = (unsigned long long)published;
    q->closed = (unsigned)closed;
    q->status = 0;
    q->spin_limit = spin_limit;
}

__global__ void k_checksum(const double * __restrict__ v, long long n, double * __restrict__ sums)
{
    double s = 0.0, a = 0.0;
    for(long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
        i += (long long)gridDim.x * blockDim.x)
    {
        const double x = v[i];
        s += x;
        a += fabs(x);
    }
    for(int o = 16; o > 0; o >>= 1)
    {
        s += __shfl_down_sync(0xffffffffu, s, o);
        a += __shfl_down_sync(0xffffffffu, a, o);
    }
    if((threadIdx.x & 31) == 0)
    {
        atomicAdd(sums, s);
        atomicAdd(sums + 1, a);
    }
}

// primitive quartets that survive the reference's primitive screening
template<int MODE>
__global__ void k_count_primq(const KernArgs a, unsigned long long * count)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int iP, iQ;
    long long off;
    unsigned long long n = 0;
    if(task_of<MODE>(a, t, iP, iQ, off))
    {
        QuartetCtx c;
        make_ctx(a, iP, iQ, c);
        for(int i = c.bi0; i < c.bi1; ++i)
        {
            const BraPrim bp = load_bra_prim(c, i);
            if(c.check && bp.skip)
                continue;
            if(!c.check)
            {
                n += c.kj1 - c.kj0;
                continue;
            }
            for(int j = c.kj0; j < c.kj1; ++j)
                n += prim_survives(c, bp, j) ? 1 : 0;
        }
    }
    for(int o = 16; o > 0; o >>= 1)
        n += __shfl_down_sync(0xffffffffu, n, o);
    if((threadIdx.x & 31) == 0 && n)
        atomicAdd(count, n);
}

} // namespace

#define SWEEP_SIDE 3                      // side streams besides the caller's

struct simint_b200_basis
{
    int nshell = 0;
    double tol = 0.0;
    std::vector<simint_shell> shells;      // copies (storage owned by caller)
    std::vector<PairClass> pcs;
    std::vector<QClass> qcs;
    long long total_out = 0;
    DevBuf dsums;
    DevBuf dqueue;                         // per class: WorkQueue + FP32 counter (SWEEP_QSTRIDE)
    std::map<std::array<long long, 3>, cudaGraphExec_t> graphs;
    std::map<std::array<long long, 3>, int> eager_done;
    long long graph_epoch = -1;            // settings_epoch() the graphs were built under
    cudaStream_t own_stream = nullptr;
    // concurrent class streams of a full-layout sweep (fork/join around the
    // classes); each side stream has its own scratch workspace
    DevBuf daooff;                          // first basis function of every shell (J/K digestion)
    int nbf = 0;
    cudaStream_t side[SWEEP_SIDE] = {};
    cudaEvent_t fork = nullptr, join[SWEEP_SIDE] = {};
    Workspace side_ws[SWEEP_SIDE];
    int nlaunch = 0;
};

static void fill_args(const simint_b200_basis * b, const QClass & q, KernArgs & a);

static void layout_outputs(simint_b200_basis * b)
{
    b->total_out = 0;
    for(auto & q : b->qcs)
    {
        q.offset = b->total_out;
        b->total_out += q.ntask * q.nout;
    }
}

static size_t perm_offset(const QClass & q)
{
    const size_t szp = (q.prefix.size() * sizeof(long long) + 255) & ~(size_t)255;
    return szp + ((q.border.size() * sizeof(int) + 255) & ~(size_t)255);
}

// Task lists of class q on the device: prefix, border and (up to
// SWEEP_PERM_MAX tasks) the visiting order of the CTA-per-quartet kernels'
// work queue -- tasks by decreasing primitive-pair product (a stable
// counting sort), so the longest shell quartets start first and the short
// ones fill the tail of the launch.
static size_t kvend_offset(const QClass & q)
{
    return perm_offset(q) + (q.has_perm ? (((size_t)q.ntask * sizeof(int) + 255) & ~(size_t)255) : 0);
}

static int upload_tasks(QClass & q, const PairClass & X, const PairClass & Y, bool screened)
{
    const size_t szp = (q.prefix.size() * sizeof(long long) + 255) & ~(size_t)255;
    const size_t off = perm_offset(q);
    q.has_perm = q.ntask > 0 && q.ntask <= SWEEP_PERM_MAX;
    const size_t szperm = q.has_perm ? (size_t)q.ntask * sizeof(int) : 0;
    // (ss|ss): the reference kernel's vector test at each row's clip (see
    // ssss_clip_vector) needs the end of the row's ket primitives, per bra pair
    q.ssss = screened && !q.req[0] && !q.req[1] && !q.req[2] && !q.req[3];
    const size_t szkv = q.ssss ? (size_t)X.P.nshell12 * sizeof(int) : 0;
    if(!q.dev.reserve(kvend_offset(q) + szkv + 8))
    {
        set_error("out of memory building task lists");
        return SIMINT_B200_ERR_CUDA;
    }
    cudaMemcpy(q.dev.ptr, q.prefix.data(), q.prefix.size() * sizeof(long long), cudaMemcpyHostToDevice);
    cudaMemcpy((char *)q.dev.ptr + szp, q.border.data(), q.border.size() * sizeof(int), cudaMemcpyHostToDevice);
    if(q.has_perm)
    {
        int maxw = 1;
        for(int ip : q.border)
            maxw = std::max(maxw, X.P.nprim12[ip]);
        int maxk = 1;
        for(int iq = 0; iq < Y.P.nshell12; iq++)
            maxk = std::max(maxk, Y.P.nprim12[iq]);
        const int nkey = maxw * maxk + 1;
        std::vector<long long> cnt(nkey + 1, 0);
        auto key = [&](size_t r, long long i) {
            return nkey - 1 - X.P.nprim12[q.border[r]] * Y.P.nprim12[Y.order[(size_t)i]];
        };
        for(size_t r = 0; r + 1 < q.prefix.size(); r++)
            for(long long i = 0; i < q.prefix[r + 1] - q.prefix[r]; i++)
                cnt[key(r, i) + 1]++;
        for(int k = 0; k < nkey; k++)
            cnt[k + 1] += cnt[k];
        std::vector<int> perm((size_t)q.ntask);
        long long t = 0;
        for(size_t r = 0; r + 1 < q.prefix.size(); r++)
            for(long long i = 0; i < q.prefix[r + 1] - q.prefix[r]; i++, t++)
                perm[(size_t)cnt[key(r, i)]++] = (int)t;
        cudaMemcpy((char *)q.dev.ptr + off, perm.data(), szperm, cudaMemcpyHostToDevice);
    }
    if(q.ssss)
    {
        std::vector<int> ystart, kv((size_t)X.P.nshell12, 0);
        int npad = 0;
        pair_starts(&Y.P, ystart, npad);
        for(size_t r = 0; r + 1 < q.prefix.size(); r++)
        {
            const long long n = q.prefix[r + 1] - q.prefix[r];
            const int last = Y.order[(size_t)n - 1];
            kv[(size_t)q.border[r]] = ystart[(size_t)last] + Y.P.nprim12[last];
        }
        cudaMemcpy((char *)q.dev.ptr + kvend_offset(q), kv.data(), szkv, cudaMemcpyHostToDevice);
    }
    return 0;
}

static void fill_args(const simint_b200_basis * b, const QClass & q, KernArgs & a)
{
    memset(&a, 0, sizeof(a));
    const PairClass & X = b->pcs[q.bx];
    const PairClass & Y = b->pcs[q.ky];
    a.P = X.view;
    a.Q = Y.view;
    a.check = b->tol > 0.0;
    a.tol2 = b->tol * b->tol;
    a.nout = q.nout;
    a.prefix = (const long long *)q.dev.ptr;
    a.border = (const int *)((const char *)q.dev.ptr + ((q.prefix.size() * sizeof(long long) + 255) & ~(size_t)255));
    a.korder = Y.dorder;
    a.nb = (int)q.border.size();
    a.kvend = q.ssss ? (const int *)((const char *)q.dev.ptr + kvend_offset(q)) : nullptr;
}

extern "C" simint_b200_basis * simint_b200_basis_create(int nshell, struct simint_shell const * shells,
                                                        double screen_tol, int max_am)
{
    init_tables();
    if(ensure_device() < 0)
        return nullptr;
    if(nshell <= 0 || !shells || max_am < 0 || max_am > SIMINT_OSTEI_MAXAM)
    {
        set_error("bad argument to simint_b200_basis_create");
        return nullptr;
    }
    simint_b200_basis * b = new simint_b200_basis;
    b->nshell = nshell;
    b->tol = screen_tol;
    b->shells.assign(shells, shells + nshell);
    Workspace & w = workspace();
    if(!w.stream)
        cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking);
    std::vector<std::vector<int>> byam(max_am + 1);
    for(int s = 0; s < nshell; s++)
        if(shells[s].am <= max_am)
            byam[shells[s].am].push_back(s);
    // pair classes
    for(int la = 0; la <= max_am; la++)
        for(int lb = 0; lb <= la; lb++)
        {
            if(byam[la].empty() || byam[lb].empty())
                continue;
            PairClass pc;
            pc.la = la;
            pc.lb = lb;
            for(int i : byam[la])
                for(int j : byam[lb])
                {
                    if(la == lb && j > i)
                        continue;
                    pc.sa.push_back(i);
                    pc.sb.push_back(j);
                }
            b->pcs.push_back(std::move(pc));
        }
    for(auto & pc : b->pcs)
    {
        const int n = (int)pc.sa.size();
        std::vector<simint_shell> AB(2 * (size_t)n);
        for(int k = 0; k < n; k++)
        {
            AB[2 * k] = shells[pc.sa[k]];
            AB[2 * k + 1] = shells[pc.sb[k]];
        }
        simint_initialize_multi_shellpair(&pc.P);
        simint_create_multi_shellpair2(n, AB.data(), &pc.P,
                                       screen_tol > 0.0 ? SIMINT_SCREEN_SCHWARZ : SIMINT_SCREEN_NONE);
        PackedLayout L;
        size_t sz = (pack_pairs(&pc.P, nullptr, L) + 255) & ~(size_t)255;
        const size_t szo = ((size_t)n * sizeof(int) + 255) & ~(size_t)255;
        const size_t szq = (size_t)n * sizeof(double);
        if(!pc.dev.reserve(sz + szo + szq) || !w.hstage.reserve(sz))
        {
            set_error("out of memory building the basis");
            simint_b200_basis_free(b);
            return nullptr;
        }
        pack_pairs(&pc.P, (char *)w.hstage.ptr, L);
        cudaMemcpy(pc.dev.ptr, w.hstage.ptr, sz, cudaMemcpyHostToDevice);
        pc.view = device_view((const char *)pc.dev.ptr, L, pc.P.screen_max);
        // Schwarz bound of every contracted pair
        double * dq = (double *)((char *)pc.dev.ptr + sz + szo);
        if(pair_diag_max(pc.view, pc.la, pc.lb, n, dq, w.stream) != 0)
        {
            simint_b200_basis_free(b);
            return nullptr;
        }
        pc.Q.resize(n);
        cudaMemcpy(pc.Q.data(), dq, n * sizeof(double), cudaMemcpyDeviceToHost);
        for(auto & v : pc.Q)
            v = std::sqrt(v);
        pc.order.resize(n);
        std::iota(pc.order.begin(), pc.order.end(), 0);
        std::stable_sort(pc.order.begin(), pc.order.end(), [&](int x, int y) { return pc.Q[x] > pc.Q[y]; });
        // Store the pairs in that order: a row's kets are then a prefix of
        // the set, exactly the clipped sorted list a caller of
        // simint_compute_eri passes, and the 8-wide vector screening groups
        // the same primitives as it does for that caller.
        bool sorted = true;
        for(int k = 0; k < n && sorted; k++)
            sorted = pc.order[k] == k;
        if(!sorted)
        {
            simint_multi_shellpair S;
            simint_initialize_multi_shellpair(&S);
            permute_multi_shellpair(&pc.P, pc.order.data(), &S);
            simint_free_multi_shellpair(&pc.P);
            pc.P = S;
            std::vector<int> sa(n), sbv(n);
            std::vector<double> q(n);
            for(int k = 0; k < n; k++)
            {
                sa[k] = pc.sa[pc.order[k]];
                sbv[k] = pc.sb[pc.order[k]];
                q[k] = pc.Q[pc.order[k]];
            }
            pc.sa.swap(sa);
            pc.sb.swap(sbv);
            pc.Q.swap(q);
            std::iota(pc.order.begin(), pc.order.end(), 0);
            const size_t sz2 = (pack_pairs(&pc.P, nullptr, L) + 255) & ~(size_t)255;
            if(!pc.dev.reserve(sz2 + szo) || !w.hstage.reserve(sz2))
            {
                set_error("out of memory building the basis");
                simint_b200_basis_free(b);
                return nullptr;
            }
            pack_pairs(&pc.P, (char *)w.hstage.ptr, L);
            cudaMemcpy(pc.dev.ptr, w.hstage.ptr, sz2, cudaMemcpyHostToDevice);
            pc.view = device_view((const char *)pc.dev.ptr, L, pc.P.screen_max);
            sz = sz2;
        }
        cudaMemcpy((char *)pc.dev.ptr + sz, pc.order.data(), n * sizeof(int), cudaMemcpyHostToDevice);
        pc.dorder = (const int *)((char *)pc.dev.ptr + sz);
    }
    // quartet classes: bra class >= ket class in (la+lb, la) order
    std::vector<int> cls(b->pcs.size());
    std::iota(cls.begin(), cls.end(), 0);
    std::stable_sort(cls.begin(), cls.end(), [&](int x, int y) {
        const auto & X = b->pcs[x];
        const auto & Y = b->pcs[y];
        return std::make_pair(X.la + X.lb, X.la) > std::make_pair(Y.la + Y.lb, Y.la);
    });
    for(size_t xi = 0; xi < cls.size(); xi++)
        for(size_t yi = xi; yi < cls.size(); yi++)
        {
            QClass q;
            q.bx = cls[xi];
            q.ky = cls[yi];
            const PairClass & X = b->pcs[q.bx];
            const PairClass & Y = b->pcs[q.ky];
            q.req[0] = X.la; q.req[1] = X.lb; q.req[2] = Y.la; q.req[3] = Y.lb;
            q.nout = ncart_of(X.la) * ncart_of(X.lb) * ncart_of(Y.la) * ncart_of(Y.lb);
            std::vector<double> qy(Y.order.size());
            for(size_t k = 0; k < qy.size(); k++)
                qy[k] = Y.Q[Y.order[k]];
            long long tot = 0;
            q.prefix.push_back(0);
            for(size_t bb = 0; bb < X.order.size(); bb++)
            {
                const double qb = X.Q[X.order[bb]];
                // ket pairs with qb * q >= tol: a prefix of the decreasing list
                long long cut = (long long)qy.size();
                if(screen_tol > 0.0)
                {
                    cut = std::upper_bound(qy.begin(), qy.end(), screen_tol / std::max(qb, 1e-300),
                                           [](double t, double v) { return v < t; }) - qy.begin();
                    // exact test at the boundary (division rounding)
                    while(cut > 0 && qb * qy[cut - 1] < screen_tol) cut--;
                    while(cut < (long long)qy.size() && qb * qy[cut] >= screen_tol) cut++;
                }
                long long cnt = (q.bx == q.ky) ? std::min<long long>((long long)bb + 1, cut) : cut;
                if(cnt <= 0)
                    continue;
                q.border.push_back(X.order[bb]);
                tot += cnt;
                q.prefix.push_back(tot);
            }
            q.ntask = tot;
            q.nfull = tot;
            if(tot == 0)
                continue;
            if(upload_tasks(q, X, Y, screen_tol > 0.0) != 0)
            {
                simint_b200_basis_free(b);
                return nullptr;
            }
            b->qcs.push_back(std::move(q));
        }
    layout_outputs(b);
    if(!b->dsums.reserve(2 * sizeof(double) * std::max<size_t>(1, b->qcs.size())) ||
       !b->dqueue.reserve(SWEEP_QSTRIDE * std::max<size_t>(1, b->qcs.size())))
    {
        set_error("out of device memory for the sweep's checksums and queues");
        simint_b200_basis_free(b);
        return nullptr;
    }
    cudaMemset(b->dqueue.ptr, 0, SWEEP_QSTRIDE * std::max<size_t>(1, b->qcs.size()));
    cudaError_t e = cudaDeviceSynchronize();
    if(e != cudaSuccess)
    {
        set_error(std::string("CUDA error building the basis: ") + cudaGetErrorString(e));
        simint_b200_basis_free(b);
        return nullptr;
    }
    return b;
}

extern "C" int simint_b200_basis_subsample(simint_b200_basis * b, long long maxq)
{
    if(!b || maxq <= 0)
        return SIMINT_B200_ERR_ARG;
    for(auto & g : b->graphs)
        cudaGraphExecDestroy(g.second);
    b->graphs.clear();
    b->eager_done.clear();
    for(auto & q : b->qcs)
    {
        if(q.ntask <= maxq)
            continue;
        const long long stride = (q.ntask + maxq - 1) / maxq;
        std::vector<long long> pre(1, 0);
        std::vector<int> bor;
        const int nb = (int)q.border.size();
        for(int r = 0; r < nb; r += (int)stride)
        {
            bor.push_back(q.border[r]);
            pre.push_back(pre.back() + (q.prefix[r + 1] - q.prefix[r]));
        }
        q.prefix.swap(pre);
        q.border.swap(bor);
        q.ntask = q.prefix.back();
        q.nprimq = 0;
        if(upload_tasks(q, b->pcs[q.bx], b->pcs[q.ky], b->tol > 0.0) != 0)
            return SIMINT_B200_ERR_CUDA;
    }
    layout_outputs(b);
    return 0;
}

extern "C" int simint_b200_basis_nrows(simint_b200_basis const * b, int k)
{
    if(!b || k < 0 || k >= (int)b->qcs.size())
        return SIMINT_B200_ERR_ARG;
    return (int)b->qcs[k].border.size();
}

extern "C" int simint_b200_basis_row(simint_b200_basis const * b, int k, int r,
                                     long long * first, long long * n)
{
    if(!b || k < 0 || k >= (int)b->qcs.size() || r < 0 || r >= (int)b->qcs[k].border.size())
        return SIMINT_B200_ERR_ARG;
    *first = b->qcs[k].prefix[r];
    *n = b->qcs[k].prefix[r + 1] - b->qcs[k].prefix[r];
    return 0;
}

extern "C" int simint_b200_basis_subsample_stride(simint_b200_basis * b, int stride, int offset)
{
    if(!b || stride < 1 || offset < 0)
        return SIMINT_B200_ERR_ARG;
    for(auto & g : b->graphs)
        cudaGraphExecDestroy(g.second);
    b->graphs.clear();
    b->eager_done.clear();
    for(auto & q : b->qcs)
    {
        std::vector<long long> pre(1, 0);
        std::vector<int> bor;
        const int nb = (int)q.border.size();
        for(int r = offset % stride; r < nb; r += stride)
        {
            bor.push_back(q.border[r]);
            pre.push_back(pre.back() + (q.prefix[r + 1] - q.prefix[r]));
        }
        q.prefix.swap(pre);
        q.border.swap(bor);
        q.ntask = q.prefix.back();
        q.nprimq = 0;
        if(upload_tasks(q, b->pcs[q.bx], b->pcs[q.ky], b->tol > 0.0) != 0)
            return SIMINT_B200_ERR_CUDA;
    }
    layout_outputs(b);
    return 0;
}

extern "C" long long simint_b200_basis_class_full(simint_b200_basis const * b, int k)
{
    if(k < 0 || k >= (int)b->qcs.size())
        return SIMINT_B200_ERR_ARG;
    return b->qcs[k].nfull;
}

extern "C" long long simint_b200_basis_count_primq(simint_b200_basis * b)
{
    unsigned long long * dcount = nullptr;
    if(cudaMalloc(&dcount, sizeof(unsigned long long)) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    long long tot = 0;
    for(auto & q : b->qcs)
    {
        KernArgs a;
        fill_args(b, q, a);
        a.ntask = q.ntask;
        cudaMemset(dcount, 0, sizeof(unsigned long long));
        k_count_primq<2><<<(unsigned)((q.ntask + 127) / 128), 128>>>(a, dcount);
        unsigned long long c = 0;
        cudaMemcpy(&c, dcount, sizeof(c), cudaMemcpyDeviceToHost);
        q.nprimq = (long long)c;
        tot += q.nprimq;
    }
    cudaFree(dcount);
    return tot;
}

extern "C" void simint_b200_basis_free(simint_b200_basis * b)
{
    if(!b)
        return;
    for(auto & g : b->graphs)
        cudaGraphExecDestroy(g.second);
    for(auto & pc : b->pcs)
    {
        simint_free_multi_shellpair(&pc.P);
        pc.dev.release();
    }
    for(auto & q : b->qcs)
        q.dev.release();
    for(auto & pc : b->pcs)
        pc.dsh.release();
    b->daooff.release();
    b->dsums.release();
    b->dqueue.release();
    for(int i = 0; i < SWEEP_SIDE; i++)
    {
        if(b->side[i]) cudaStreamDestroy(b->side[i]);
        if(b->join[i]) cudaEventDestroy(b->join[i]);
        b->side_ws[i].dscratch.release();
    }
    if(b->fork) cudaEventDestroy(b->fork);
    delete b;
}

extern "C" long long simint_b200_basis_nquartets(simint_b200_basis const * b)
{
    long long n = 0;
    for(auto & q : b->qcs) n += q.ntask;
    return n;
}

extern "C" long long simint_b200_basis_nprimquartets(simint_b200_basis const * b)
{
    long long n = 0;
    for(auto & q : b->qcs) n += q.nprimq;
    return n;
}

extern "C" long long simint_b200_basis_output_size(simint_b200_basis const * b)
{
    return b->total_out;
}

extern "C" int simint_b200_basis_nclass(simint_b200_basis const * b)
{
    return (int)b->qcs.size();
}

extern "C" int simint_b200_basis_class_info(simint_b200_basis const * b, int k, int am[4],
                                            long long * nquart, long long * nprimq,
                                            int * nout, long long * offset)
{
    if(k < 0 || k >= (int)b->qcs.size())
        return SIMINT_B200_ERR_ARG;
    const QClass & q = b->qcs[k];
    if(am) memcpy(am, q.req, sizeof(q.req));
    if(nquart) *nquart = q.ntask;
    if(nprimq) *nprimq = q.nprimq;
    if(nout) *nout = q.nout;
    if(offset) *offset = q.offset;
    return 0;
}

extern "C" int simint_b200_basis_quartet(simint_b200_basis const * b, int k, long long t, int sh[4])
{
    if(k < 0 || k >= (int)b->qcs.size() || t < 0 || t >= b->qcs[k].ntask)
        return SIMINT_B200_ERR_ARG;
    const QClass & q = b->qcs[k];
    const int bi = (int)(std::upper_bound(q.prefix.begin(), q.prefix.end(), t) - q.prefix.begin()) - 1;
    const int ip = q.border[bi];
    const PairClass & X = b->pcs[q.bx];
    const PairClass & Y = b->pcs[q.ky];
    const int iq = Y.order[(size_t)(t - q.prefix[bi])];
    sh[0] = X.sa[ip]; sh[1] = X.sb[ip];
    sh[2] = Y.sa[iq]; sh[3] = Y.sb[iq];
    return 0;
}

extern "C" int simint_b200_basis_class_kets(simint_b200_basis const * b, int k, int * shells)
{
    if(!b || k < 0 || k >= (int)b->qcs.size())
        return SIMINT_B200_ERR_ARG;
    const PairClass & Y = b->pcs[b->qcs[k].ky];
    const int n = (int)Y.sa.size();
    if(shells)
        for(int i = 0; i < n; i++)
        {
            shells[2 * i] = Y.sa[(size_t)Y.order[(size_t)i]];
            shells[2 * i + 1] = Y.sb[(size_t)Y.order[(size_t)i]];
        }
    return n;
}

extern "C" int simint_b200_basis_class_quartets(simint_b200_basis const * b, int k, int * sh)
{
    if(!b || !sh || k < 0 || k >= (int)b->qcs.size())
        return SIMINT_B200_ERR_ARG;
    const QClass & q = b->qcs[k];
    const PairClass & X = b->pcs[q.bx];
    const PairClass & Y = b->pcs[q.ky];
    long long t = 0;
    for(size_t r = 0; r + 1 < q.prefix.size(); r++)
    {
        const int ip = q.border[r];
        for(long long i = 0; i < q.prefix[r + 1] - q.prefix[r]; i++, t++)
        {
            const int iq = Y.order[(size_t)i];
            sh[4 * t] = X.sa[ip]; sh[4 * t + 1] = X.sb[ip];
            sh[4 * t + 2] = Y.sa[iq]; sh[4 * t + 3] = Y.sb[iq];
        }
    }
    return 0;
}

static WorkQueue * class_queue(simint_b200_basis * b, size_t k)
{
    return (WorkQueue *)((char *)b->dqueue.ptr + k * SWEEP_QSTRIDE);
}

static unsigned long long * class_fp32(simint_b200_basis * b, size_t k)
{
    return (unsigned long long *)((char *)b->dqueue.ptr + k * SWEEP_QSTRIDE + sizeof(WorkQueue));
}

// Polls of about a microsecond a CTA waits on its launch's queue: every task
// is published before the launch, so no wait happens in a sweep.
#define SWEEP_SPIN_LIMIT 1000000ull

// Issue the launches of class k (ERI chunks + checksums) on `stream`.
// J/K digestion of a streamed sweep (simint_b200_basis_compute_jk): each
// chunk of a class's integrals is contracted right after it is computed,
// while it is still in L2.
struct JKJob
{
    const double * D;
    double *J, *K;
};
static int jk_chunk(simint_b200_basis * b, size_t k, const double * out, long long t0, long long cn,
                    const JKJob & job, cudaStream_t stream);

static int issue_class(simint_b200_basis * b, size_t k, int prec, double * dout, long long cap,
                       cudaStream_t stream, const JKJob * jk = nullptr)
{
    int nl = 0;
    const bool full = cap >= b->total_out;
    double * dsums = (double *)b->dsums.ptr;
    QClass & q = b->qcs[k];
    const long long chunk = full ? q.ntask : std::max<long long>(1, cap / q.nout);
    // SIMINT_B200_SWEEP_QUEUE=0: static grid-stride task order instead
    static const bool queue_on = [] {
        const char * e = getenv("SIMINT_B200_SWEEP_QUEUE");
        return !(e && atoi(e) == 0);
    }();
    const bool queued = queue_on && class_uses_queue(q.req, 0, prec);
    for(long long t0 = 0; t0 < q.ntask; t0 += chunk)
    {
        const long long cn = std::min(chunk, q.ntask - t0);
        KernArgs a;
        fill_args(b, q, a);
        a.ntask = cn;
        a.task0 = t0;
        a.out = full ? dout + q.offset + t0 * q.nout : dout;
        a.gate = gate();
        a.fp32_count = class_fp32(b, k);
        if(queued)
        {
            // CTA-per-quartet kernels take their shell quartets from the
            // class's work queue, heaviest first when the launch covers the
            // whole class
            a.wq = class_queue(b, k);
            k_queue_reset<<<1, 1, 0, stream>>>(a.wq, cn, SWEEP_SPIN_LIMIT);
            count_launch(1);
            nl++;
            if(q.has_perm && cn == q.ntask)
                a.tperm = (const int *)((const char *)q.dev.ptr + perm_offset(q));
        }
        int rc = launch_class(a, q.req, 0, 2, prec, stream);
        if(rc != 0)
            return rc;
        nl++;
        const long long n = cn * q.nout;
        const unsigned blocks = (unsigned)std::min<long long>(148 * 8, (n + 255) / 256);
        k_checksum<<<blocks, 256, 0, stream>>>(a.out, n, dsums + 2 * k);
        count_launch(1);
        nl++;
        if(jk)
        {
            rc = jk_chunk(b, k, a.out, t0, cn, *jk, stream);
            if(rc < 0)
                return rc;
            nl += rc;
        }
    }
    return nl;
}

// Issue every launch of one sweep on `stream`.  events: optional per-class
// start/stop pairs (eager runs only).
static int issue_sweep(simint_b200_basis * b, int prec, double * dout, long long cap,
                       cudaStream_t stream, cudaEvent_t * events)
{
    int nl = 0;
    cudaMemsetAsync(b->dsums.ptr, 0, 2 * sizeof(double) * b->qcs.size(), stream);
    cudaMemsetAsync(b->dqueue.ptr, 0, SWEEP_QSTRIDE * b->qcs.size(), stream);
    if(!events && cap >= b->total_out)
    {
        // full layout: classes write disjoint output ranges, so they run on
        // SWEEP_SIDE + 1 streams at once (small classes fill the GPU while
        // large ones run).  Classes go to the least loaded stream, largest
        // estimated cost first.
        if(!b->fork)
        {
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
            for(int i = 0; i < SWEEP_SIDE; i++)
            {
                cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
                cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
            }
        }
        std::vector<size_t> order(b->qcs.size());
        std::iota(order.begin(), order.end(), 0);
        // cost estimate from the task lists only (the same assignment on the
        // eager run that sizes the workspaces and on the captured run)
        auto cost = [&](size_t k) {
            const QClass & q = b->qcs[k];
            const int L = q.req[0] + q.req[1] + q.req[2] + q.req[3];
            return (double)q.ntask * q.nout * (1.0 + L);
        };
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return cost(x) > cost(y); });
        double load[SWEEP_SIDE + 1] = {};
        cudaEventRecord(b->fork, stream);
        for(int i = 0; i < SWEEP_SIDE; i++)
            cudaStreamWaitEvent(b->side[i], b->fork, 0);
        int rc = 0;
        for(size_t k : order)
        {
            int s = 0;
            for(int i = 1; i <= SWEEP_SIDE; i++)
                if(load[i] < load[s]) s = i;
            load[s] += cost(k);
            set_workspace_override(s ? &b->side_ws[s - 1] : nullptr);
            const int r = issue_class(b, k, prec, dout, cap, s ? b->side[s - 1] : stream);
            set_workspace_override(nullptr);
            if(r < 0)
            {
                rc = r;
                break;
            }
            nl += r;
        }
        for(int i = 0; i < SWEEP_SIDE; i++)
        {
            cudaEventRecord(b->join[i], b->side[i]);
            cudaStreamWaitEvent(stream, b->join[i], 0);
        }
        return rc < 0 ? rc : nl;
    }
    for(size_t k = 0; k < b->qcs.size(); k++)
    {
        if(events)
            cudaEventRecord(events[2 * k], stream);
        const int r = issue_class(b, k, prec, dout, cap, stream);
        if(r < 0)
            return r;
        nl += r;
        if(events)
            cudaEventRecord(events[2 * k + 1], stream);
    }
    return nl;
}

extern "C" int simint_b200_basis_autotune(simint_b200_basis * b, int prec, double * dev_out,
                                          long long dev_out_doubles, void * stream_)
{
    if(!b || !dev_out || dev_out_doubles <= 0)
        return SIMINT_B200_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    for(auto & g : b->graphs)
        cudaGraphExecDestroy(g.second);
    b->graphs.clear();
    b->eager_done.clear();
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaMemsetAsync(b->dsums.ptr, 0, 2 * sizeof(double) * b->qcs.size(), stream);
    for(size_t k = 0; k < b->qcs.size(); k++)
    {
        QClass & q = b->qcs[k];
        if(q.ntask == 0)
            continue;
        std::vector<int> cand;
        if(has_straight(q.req))
        {
            cand.push_back(VAR_STRAIGHT);
            if(prec == SIMINT_B200_PREC_MIXED)
                cand.push_back(VAR_STRAIGHT64);
        }
        if(has_warp(q.req, 2))
        {
            cand.push_back(VAR_WARP);
            if(prec == SIMINT_B200_PREC_MIXED)
                cand.push_back(VAR_WARP64);
        }
        for(int v : {81, 82, 83})
            if(col_supported(q.req, 0, v))
            {
                cand.push_back(v);
                if(prec == SIMINT_B200_PREC_MIXED)
                    cand.push_back(v + 100);
            }
        for(int v : {21, 22, 24, 28, 41, 42, 44, 48, 61, 62, 64, 68})
            if(coop2_supported(q.req, 0, v))
            {
                cand.push_back(v);
                if(prec == SIMINT_B200_PREC_MIXED)
                    cand.push_back(v + 100);      // the same kernel without the FP32 path
            }
        if(cand.empty())
            continue;
        int best = cand[0];
        float bestms = 1e30f;
        for(int v : cand)
        {
            set_variant(q.req, 0, prec, v);
            cudaEventRecord(e0, stream);
            if(issue_class(b, k, prec, dev_out, dev_out_doubles, stream) < 0)
                continue;
            cudaEventRecord(e1, stream);
            cudaEventSynchronize(e1);
            float warm = 0;
            cudaEventElapsedTime(&warm, e0, e1);
            // a candidate whose first run (which includes loading its
            // kernel) takes over twice the best time so far plus a
            // millisecond is not timed again
            if(warm > 2.0f * bestms + 1.0f)
                continue;
            float ms = 1e30f;
            for(int rep = 0; rep < 2; rep++)
            {
                cudaEventRecord(e0, stream);
                issue_class(b, k, prec, dev_out, dev_out_doubles, stream);
                cudaEventRecord(e1, stream);
                cudaEventSynchronize(e1);
                float t = 0;
                cudaEventElapsedTime(&t, e0, e1);
                ms = std::min(ms, t);
            }
            if(ms < bestms)
            {
                bestms = ms;
                best = v;
            }
        }
        set_variant(q.req, 0, prec, best);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    save_tune_file();
    const cudaError_t e = cudaStreamSynchronize(stream);
    if(e != cudaSuccess)
    {
        set_error(std::string("autotune: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    return 0;
}

extern "C" int simint_b200_variant(const int am[4], int deriv, int prec)
{
    return variant_of(am, deriv, prec);
}

extern "C" int simint_b200_basis_compute(simint_b200_basis * b, int prec, double * dev_out,
                                         long long dev_out_doubles, void * stream_)
{
    if(!b || !dev_out || dev_out_doubles <= 0)
        return SIMINT_B200_ERR_ARG;
    cudaStream_t stream = (cudaStream_t)stream_;
    if(b->graph_epoch != settings_epoch())
    {
        // a kernel variant, the ordering or the precision gate changed:
        // graphs captured before bake in the old choice
        cudaStreamSynchronize(stream);
        for(auto & g : b->graphs)
            cudaGraphExecDestroy(g.second);
        b->graphs.clear();
        b->eager_done.clear();
        b->graph_epoch = settings_epoch();
    }
    const std::array<long long, 3> key = {prec, (long long)(uintptr_t)dev_out, dev_out_doubles};
    auto it = b->graphs.find(key);
    if(it != b->graphs.end())
    {
        if(cudaGraphLaunch(it->second, stream) != cudaSuccess)
        {
            set_error("cudaGraphLaunch failed");
            return SIMINT_B200_ERR_CUDA;
        }
        count_launch(b->nlaunch);
        return b->nlaunch;
    }
    if(!b->eager_done.count(key))
    {
        // first use: run eagerly so every table and scratch buffer exists
        int nl = issue_sweep(b, prec, dev_out, dev_out_doubles, stream, nullptr);
        if(nl < 0)
            return nl;
        b->eager_done[key] = 1;
        b->nlaunch = nl;
        return nl;
    }
    // second use: capture the sweep into a CUDA graph and replay it
    cudaStream_t cs = stream;
    bool own = false;
    if(!cs)
    {
        cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
        own = true;
    }
    cudaGraph_t graph;
    if(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    {
        set_error("cudaStreamBeginCapture failed");
        return SIMINT_B200_ERR_CUDA;
    }
    const long long before = simint_b200_launch_count();
    int nl = issue_sweep(b, prec, dev_out, dev_out_doubles, cs, nullptr);
    count_launch(-(simint_b200_launch_count() - before));   // captured, not launched
    cudaError_t e = cudaStreamEndCapture(cs, &graph);
    if(nl < 0)
        return nl;
    if(e != cudaSuccess)
    {
        set_error(std::string("graph capture failed: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if(e != cudaSuccess)
    {
        set_error(std::string("graph instantiate failed: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    b->graphs[key] = exec;
    if(own)
    {
        cudaStreamSynchronize(cs);
        cudaStreamDestroy(cs);
    }
    b->nlaunch = nl;
    cudaGraphLaunch(exec, stream);
    count_launch(nl);
    return nl;
}

// Status words of the classes' work queues: SIMINT_B200_ERR_TIMEOUT when a
// wait of the last sweep ran out.
static int queue_status(simint_b200_basis * b)
{
    std::vector<char> h(SWEEP_QSTRIDE * b->qcs.size());
    if(h.empty())
        return 0;
    if(cudaMemcpy(h.data(), b->dqueue.ptr, h.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    for(size_t k = 0; k < b->qcs.size(); k++)
    {
        WorkQueue w;
        memcpy(&w, h.data() + k * SWEEP_QSTRIDE, sizeof(w));
        if(w.status)
        {
            set_error("a work-queue wait ran out");
            return SIMINT_B200_ERR_TIMEOUT;
        }
    }
    return 0;
}

extern "C" int simint_b200_basis_checksums(simint_b200_basis * b, double * sums)
{
    if(!b || !sums)
        return SIMINT_B200_ERR_ARG;
    cudaDeviceSynchronize();
    if(cudaMemcpy(sums, b->dsums.ptr, 2 * sizeof(double) * b->qcs.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    return queue_status(b);
}

extern "C" int simint_b200_basis_fp32_counts(simint_b200_basis * b, long long * counts)
{
    if(!b || !counts)
        return SIMINT_B200_ERR_ARG;
    cudaDeviceSynchronize();
    std::vector<char> h(SWEEP_QSTRIDE * b->qcs.size());
    if(!h.empty() && cudaMemcpy(h.data(), b->dqueue.ptr, h.size(), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    for(size_t k = 0; k < b->qcs.size(); k++)
    {
        unsigned long long c = 0;
        memcpy(&c, h.data() + k * SWEEP_QSTRIDE + sizeof(WorkQueue), sizeof(c));
        counts[k] = (long long)c;
    }
    return 0;
}

extern "C" int simint_b200_basis_queue_probe(simint_b200_basis * b, int k, long long published, int closed,
                                             int wait_ms, double * dev_out, long long dev_out_doubles)
{
    if(!b || k < 0 || k >= (int)b->qcs.size() || !dev_out || published < 0 || wait_ms < 0)
        return SIMINT_B200_ERR_ARG;
    QClass & q = b->qcs[k];
    if(dev_out_doubles < q.ntask * q.nout || published > q.ntask)
        return SIMINT_B200_ERR_ARG;
    if(!class_uses_queue(q.req, 0, SIMINT_B200_PREC_FP64))
    {
        set_error("the class's kernel does not take work from a queue");
        return SIMINT_B200_ERR_ARG;
    }
    Workspace & w = workspace();
    if(!w.stream)
        cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking);
    KernArgs a;
    fill_args(b, q, a);
    a.ntask = q.ntask;
    a.task0 = 0;
    a.out = dev_out;
    a.wq = class_queue(b, (size_t)k);
    k_queue_set<<<1, 1, 0, w.stream>>>(a.wq, published, closed, 1000ull * (unsigned long long)wait_ms);
    count_launch(1);
    int rc = launch_class(a, q.req, 0, 2, SIMINT_B200_PREC_FP64, w.stream);
    if(rc != 0)
        return rc;
    const cudaError_t e = cudaStreamSynchronize(w.stream);
    if(e != cudaSuccess)
    {
        set_error(std::string("queue probe: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    WorkQueue hq;
    if(cudaMemcpy(&hq, a.wq, sizeof(hq), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    if(hq.status)
    {
        set_error("a work-queue wait ran out");
        return SIMINT_B200_ERR_TIMEOUT;
    }
    return (int)std::min<long long>(published, 0x7fffffff);
}

extern "C" int simint_b200_basis_class_times(simint_b200_basis * b, int prec, double * dev_out,
                                             long long dev_out_doubles, void * stream_, float * ms)
{
    cudaStream_t stream = (cudaStream_t)stream_;
    std::vector<cudaEvent_t> ev(2 * b->qcs.size());
    for(auto & e : ev)
        cudaEventCreate(&e);
    int nl = issue_sweep(b, prec, dev_out, dev_out_doubles, stream, ev.data());
    cudaStreamSynchronize(stream);
    for(size_t k = 0; k < b->qcs.size() && nl >= 0; k++)
        cudaEventElapsedTime(&ms[k], ev[2 * k], ev[2 * k + 1]);
    for(auto & e : ev)
        cudaEventDestroy(e);
    return nl;
}


// ---------------------------------------------------------------------
// Fock-matrix digestion of a full-layout sweep: Coulomb and exchange
// matrices J_pq = sum_rs (pq|rs) D_rs, K_pq = sum_rs (pr|qs) D_rs for a
// symmetric density D, from the shell quartets the sweep computed (each
// unordered shell pair once, each unordered pair of pairs once).  Every
// quartet is scaled by its degeneracy (2 for a != b, 2 for c != d, 2 when
// the bra and ket pairs differ) and adds its contributions to the raw J and
// K; the symmetrised halves (J = (Jr + Jr^T)/4, K = (Kr + Kr^T)/8) are the
// full sums.
// ---------------------------------------------------------------------
namespace {

struct JKArgs
{
    const long long * prefix;
    const int * border;
    const int * korder;
    int nb;
    long long ntask;
    const int2 * shX, * shY;
    const int * aooff;
    int na, nbb, nc, nd;
    int same_class;                 // bra and ket pair classes equal (unique pair-pairs)
    const double * out;             // integrals of tasks task0 .. task0 + ntask - 1
    long long task0;
    const double * D;
    double * J, * K;
    int nbf;
};

// One warp per shell quartet: the quartet's integrals are staged in shared
// memory (coalesced), then each of the six contractions gives every lane
// outer elements (p,q), (r,s), ... to sum over the inner pair; one atomic
// add per outer element.
// Shell quartet t of a class: its position in the task list and the
// degeneracy factor (2 for a != b, 2 for c != d, 2 when the bra and ket
// pairs differ).
__device__ __forceinline__ void jk_quartet(const JKArgs & g, long long t, int2 & ab, int2 & cd, double & sc)
{
    int lo = 0, hi = g.nb;
    while(hi - lo > 1)
    {
        const int mid = (lo + hi) >> 1;
        if(__ldg(g.prefix + mid) <= t) lo = mid; else hi = mid;
    }
    const int iP = __ldg(g.border + lo);
    const int iQ = __ldg(g.korder + (int)(t - __ldg(g.prefix + lo)));
    ab = g.shX[iP];
    cd = g.shY[iQ];
    sc = (ab.x != ab.y ? 2.0 : 1.0) * (cd.x != cd.y ? 2.0 : 1.0)
       * ((g.same_class && iP == iQ) ? 1.0 : 2.0);
}

// Density sub-blocks a quartet (ab|cd) reads, staged next to its integrals:
// D[c][d], D[a][b], D[b][d], D[a][c], D[b][c], D[a][d] (row-major, in that
// order); jk_dsize doubles in all.
__host__ __device__ __forceinline__ int jk_dsize(int na, int nb, int nc, int nd)
{
    return nc * nd + na * nb + nb * nd + na * nc + nb * nc + na * nd;
}

__device__ __forceinline__ void jk_stage_d(const JKArgs & g, int2 ab, int2 cd, double * Ds, int k0, int stride)
{
    const int o[4] = {g.aooff[ab.x], g.aooff[ab.y], g.aooff[cd.x], g.aooff[cd.y]};
    const int nn[4] = {g.na, g.nbb, g.nc, g.nd};
    // (row shell, column shell) of the six blocks: 0 = a, 1 = b, 2 = c, 3 = d
    const int rs[6] = {2, 0, 1, 0, 1, 0}, cs[6] = {3, 1, 3, 2, 2, 3};
    int base = 0;
    #pragma unroll
    for(int b = 0; b < 6; b++)
    {
        const int nr = nn[rs[b]], nc = nn[cs[b]], orow = o[rs[b]], ocol = o[cs[b]];
        for(int e = k0; e < nr * nc; e += stride)
        {
            const int r = e / nc, c = e - r * nc;
            Ds[base + e] = __ldg(g.D + (size_t)(orow + r) * g.nbf + ocol + c);
        }
        base += nr * nc;
    }
}

// The six contractions of one staged quartet I (scaled by its degeneracy)
// with its staged density blocks Ds, output elements over threads k0,
// k0 + stride, ...; one atomic add each.
__device__ __forceinline__ void jk_passes(const JKArgs & g, int2 ab, int2 cd, const double * I,
                                          const double * Ds, int k0, int stride)
{
    const int oA = g.aooff[ab.x], oB = g.aooff[ab.y], oC = g.aooff[cd.x], oD = g.aooff[cd.y];
    const int na = g.na, nb = g.nbb, nc = g.nc, nd = g.nd, n = g.nbf;
    const double * Dcd = Ds;
    const double * Dab = Dcd + nc * nd;
    const double * Dbd = Dab + na * nb;
    const double * Dac = Dbd + nb * nd;
    const double * Dbc = Dac + na * nc;
    const double * Dad = Dbc + nb * nc;
    // J(p,q) += sum_rs D(r,s) I ; J(r,s) += sum_pq D(p,q) I
    for(int e = k0; e < na * nb; e += stride)
    {
        const int p = e / nb, q = e - p * nb;
        const double * row = I + e * nc * nd;
        double a = 0.0;
        for(int rs2 = 0; rs2 < nc * nd; rs2++)
            a = fma(Dcd[rs2], row[rs2], a);
        atomicAdd(g.J + (oA + p) * n + oB + q, a);
    }
    for(int e = k0; e < nc * nd; e += stride)
    {
        const int r = e / nd, s2 = e - r * nd;
        double a = 0.0;
        for(int pq = 0; pq < na * nb; pq++)
            a = fma(Dab[pq], I[pq * nc * nd + e], a);
        atomicAdd(g.J + (oC + r) * n + oD + s2, a);
    }
    // K(p,r) += D(q,s) I ; K(q,s) += D(p,r) I ; K(p,s) += D(q,r) I ; K(q,r) += D(p,s) I
    for(int e = k0; e < na * nc; e += stride)
    {
        const int p = e / nc, r = e - p * nc;
        double a = 0.0;
        for(int q = 0; q < nb; q++)
            for(int s2 = 0; s2 < nd; s2++)
                a = fma(Dbd[q * nd + s2], I[((p * nb + q) * nc + r) * nd + s2], a);
        atomicAdd(g.K + (oA + p) * n + oC + r, a);
    }
    for(int e = k0; e < nb * nd; e += stride)
    {
        const int q = e / nd, s2 = e - q * nd;
        double a = 0.0;
        for(int p = 0; p < na; p++)
            for(int r = 0; r < nc; r++)
                a = fma(Dac[p * nc + r], I[((p * nb + q) * nc + r) * nd + s2], a);
        atomicAdd(g.K + (oB + q) * n + oD + s2, a);
    }
    for(int e = k0; e < na * nd; e += stride)
    {
        const int p = e / nd, s2 = e - p * nd;
        double a = 0.0;
        for(int q = 0; q < nb; q++)
            for(int r = 0; r < nc; r++)
                a = fma(Dbc[q * nc + r], I[((p * nb + q) * nc + r) * nd + s2], a);
        atomicAdd(g.K + (oA + p) * n + oD + s2, a);
    }
    for(int e = k0; e < nb * nc; e += stride)
    {
        const int q = e / nc, r = e - q * nc;
        double a = 0.0;
        for(int p = 0; p < na; p++)
            for(int s2 = 0; s2 < nd; s2++)
                a = fma(Dad[p * nd + s2], I[((p * nb + q) * nc + r) * nd + s2], a);
        atomicAdd(g.K + (oB + q) * n + oC + r, a);
    }
}

// WPB warps per block, one shell quartet per warp, the quartet's integrals
// and density blocks staged in the warp's shared memory.
template<int WPB>
__global__ void __launch_bounds__(32 * WPB) k_jk(const JKArgs g)
{
    extern __shared__ double jsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long t = (long long)blockIdx.x * WPB + warp;
    if(t >= g.ntask)
        return;
    int2 ab, cd;
    double sc;
    jk_quartet(g, g.task0 + t, ab, cd, sc);
    const int nout = g.na * g.nbb * g.nc * g.nd;
    double * I = jsm + (size_t)warp * (nout + jk_dsize(g.na, g.nbb, g.nc, g.nd));
    double * Ds = I + nout;
    const double * src = g.out + t * (long long)nout;
    for(int k = lane; k < nout; k += 32)
        I[k] = __ldg(src + k) * sc;
    jk_stage_d(g, ab, cd, Ds, lane, 32);
    __syncwarp();
    jk_passes(g, ab, cd, I, Ds, lane, 32);
}

// Classes whose quartet fills more than 24 KB of shared memory: one block of
// NT threads per shell quartet (a warp alone would leave the SM with 2-4
// warps), the six contractions spread over all NT threads.
template<int NT>
__global__ void __launch_bounds__(NT) k_jkb(const JKArgs g)
{
    extern __shared__ double jsm[];
    const long long t = blockIdx.x;
    int2 ab, cd;
    double sc;
    jk_quartet(g, g.task0 + t, ab, cd, sc);
    const int nout = g.na * g.nbb * g.nc * g.nd;
    double * Ds = jsm + nout;
    const double * src = g.out + t * (long long)nout;
    for(int k = threadIdx.x; k < nout; k += NT)
        jsm[k] = __ldg(src + k) * sc;
    jk_stage_d(g, ab, cd, Ds, threadIdx.x, NT);
    __syncthreads();
    jk_passes(g, ab, cd, jsm, Ds, threadIdx.x, NT);
}

__global__ void k_jk_sym(double * __restrict__ J, double * __restrict__ K, int n)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= (long long)n * n)
        return;
    const int i = (int)(t / n), j = (int)(t - (long long)i * n);
    if(j < i)
        return;
    const double ja = J[(size_t)i * n + j], jb = J[(size_t)j * n + i];
    const double ka = K[(size_t)i * n + j], kb = K[(size_t)j * n + i];
    J[(size_t)i * n + j] = J[(size_t)j * n + i] = 0.25 * (ja + jb);
    K[(size_t)i * n + j] = K[(size_t)j * n + i] = 0.125 * (ka + kb);
}

} // namespace

extern "C" int simint_b200_basis_nbf(simint_b200_basis const * b)
{
    if(!b)
        return SIMINT_B200_ERR_ARG;
    int n = 0;
    for(const auto & s : b->shells)
        n += ncart_of(s.am);
    return n;
}

// Shell offsets and pair shell lists of the digestion (once per basis);
// every shell must take part in the sweep (none above its max_am).
static int jk_prepare(simint_b200_basis * b)
{
    if(!b->daooff.ptr)
    {
        std::vector<int> off(b->shells.size());
        int o = 0;
        for(size_t s = 0; s < b->shells.size(); s++)
        {
            off[s] = o;
            o += ncart_of(b->shells[s].am);
        }
        if(!b->daooff.reserve(off.size() * sizeof(int)))
            return SIMINT_B200_ERR_CUDA;
        cudaMemcpy(b->daooff.ptr, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice);
        for(auto & pc : b->pcs)
        {
            std::vector<int2> sh(pc.sa.size());
            for(size_t k = 0; k < sh.size(); k++)
                sh[k] = make_int2(pc.sa[k], pc.sb[k]);
            if(!pc.dsh.reserve(std::max<size_t>(1, sh.size()) * sizeof(int2)))
                return SIMINT_B200_ERR_CUDA;
            cudaMemcpy(pc.dsh.ptr, sh.data(), sh.size() * sizeof(int2), cudaMemcpyHostToDevice);
        }
        b->nbf = simint_b200_basis_nbf(b);
    }
    for(const auto & sh : b->shells)
    {
        bool found = false;
        for(const auto & pc : b->pcs)
            if(pc.la == sh.am || pc.lb == sh.am)
                found = true;
        if(!found)
        {
            set_error("a shell of the basis is above the sweep's max_am");
            return SIMINT_B200_ERR_ARG;
        }
    }
    return 0;
}

// Shared memory of the digestion of one quartet of class q (integrals and
// density blocks), or 0 when it exceeds 227 KB.
static size_t jk_quartet_bytes(const QClass & q)
{
    const size_t per = ((size_t)q.nout + jk_dsize(ncart_of(q.req[0]), ncart_of(q.req[1]), ncart_of(q.req[2]),
                                                   ncart_of(q.req[3]))) * sizeof(double);
    return per > 227 * 1024 ? 0 : per;
}

// Contract tasks t0 .. t0 + cn - 1 of class k, whose integrals are at out,
// into the raw J and K sums.  Returns the launches (1) or an error.
static int jk_launch(simint_b200_basis * b, size_t k, const double * out, long long t0, long long cn,
                     const JKJob & job, cudaStream_t stream)
{
    const QClass & q = b->qcs[k];
    KernArgs a;
    fill_args(b, q, a);
    JKArgs g;
    g.prefix = a.prefix;
    g.border = a.border;
    g.korder = a.korder;
    g.nb = a.nb;
    g.ntask = cn;
    g.task0 = t0;
    g.shX = (const int2 *)b->pcs[q.bx].dsh.ptr;
    g.shY = (const int2 *)b->pcs[q.ky].dsh.ptr;
    g.aooff = (const int *)b->daooff.ptr;
    g.na = ncart_of(q.req[0]); g.nbb = ncart_of(q.req[1]); g.nc = ncart_of(q.req[2]); g.nd = ncart_of(q.req[3]);
    g.same_class = q.bx == q.ky;
    g.out = out;
    g.D = job.D;
    g.J = job.J;
    g.K = job.K;
    g.nbf = b->nbf;
    // the quartet's integrals and density blocks are staged in shared
    // memory: one quartet per warp, 4 warps per block, while they fit
    // 96 KB; else one quartet per 256-thread block, up to 227 KB (about
    // 28 000 integrals per shell quartet: (gg|gd), (gf|gf), (gg|ff))
    const size_t per_warp = jk_quartet_bytes(q);
    if(!per_warp)
    {
        set_error("J/K digestion: class too large for the digestion kernel");
        return SIMINT_B200_ERR_CLASS;
    }
    if(4 * per_warp <= 96 * 1024)
    {
        cudaFuncSetAttribute(k_jk<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
        k_jk<4><<<(unsigned)((cn + 3) / 4), 128, 4 * per_warp, stream>>>(g);
    }
    else
    {
        cudaFuncSetAttribute(k_jkb<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        k_jkb<256><<<(unsigned)cn, 256, per_warp, stream>>>(g);
    }
    count_launch(1);
    return 1;
}

static int jk_chunk(simint_b200_basis * b, size_t k, const double * out, long long t0, long long cn,
                    const JKJob & job, cudaStream_t stream)
{
    return jk_launch(b, k, out, t0, cn, job, stream);
}

static int jk_finish(simint_b200_basis * b, const JKJob & job, cudaStream_t stream)
{
    const long long nn = (long long)b->nbf * b->nbf;
    k_jk_sym<<<(unsigned)((nn + 255) / 256), 256, 0, stream>>>(job.J, job.K, b->nbf);
    count_launch(1);
    const cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess)
    {
        set_error(std::string("J/K digestion: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    return 1;
}

extern "C" int simint_b200_basis_jk(simint_b200_basis * b, const double * dev_out, long long dev_out_doubles,
                                    const double * dev_D, double * dev_J, double * dev_K, void * stream_)
{
    if(!b || !dev_out || !dev_D || !dev_J || !dev_K || dev_out_doubles < b->total_out)
    {
        set_error("simint_b200_basis_jk needs the full-layout output of the sweep");
        return SIMINT_B200_ERR_ARG;
    }
    cudaStream_t stream = (cudaStream_t)stream_;
    int rc = jk_prepare(b);
    if(rc < 0)
        return rc;
    const int nbf = b->nbf;
    cudaMemsetAsync(dev_J, 0, (size_t)nbf * nbf * sizeof(double), stream);
    cudaMemsetAsync(dev_K, 0, (size_t)nbf * nbf * sizeof(double), stream);
    const JKJob job = {dev_D, dev_J, dev_K};
    int nl = 0;
    for(size_t k = 0; k < b->qcs.size(); k++)
    {
        const QClass & q = b->qcs[k];
        if(q.ntask == 0)
            continue;
        rc = jk_launch(b, k, dev_out + q.offset, 0, q.ntask, job, stream);
        if(rc < 0)
            return rc;
        nl += rc;
    }
    rc = jk_finish(b, job, stream);
    return rc < 0 ? rc : nl + rc;
}

extern "C" int simint_b200_basis_compute_jk(simint_b200_basis * b, int prec, const double * dev_D,
                                            double * dev_J, double * dev_K, double * dev_scratch,
                                            long long scratch_doubles, void * stream_)
{
    if(!b || !dev_D || !dev_J || !dev_K || !dev_scratch || scratch_doubles <= 0)
    {
        set_error("bad argument to simint_b200_basis_compute_jk");
        return SIMINT_B200_ERR_ARG;
    }
    if(prec != SIMINT_B200_PREC_FP64 && prec != SIMINT_B200_PREC_MIXED)
        return SIMINT_B200_ERR_ARG;
    for(const auto & q : b->qcs)
        if(q.ntask > 0 && (scratch_doubles < q.nout || !jk_quartet_bytes(q)))
        {
            set_error(scratch_doubles < q.nout ? "scratch buffer smaller than one quartet of a class"
                                               : "J/K digestion: class too large for the digestion kernel");
            return scratch_doubles < q.nout ? SIMINT_B200_ERR_ARG : SIMINT_B200_ERR_CLASS;
        }
    cudaStream_t stream = (cudaStream_t)stream_;
    int rc = jk_prepare(b);
    if(rc < 0)
        return rc;
    const int nbf = b->nbf;
    cudaMemsetAsync(dev_J, 0, (size_t)nbf * nbf * sizeof(double), stream);
    cudaMemsetAsync(dev_K, 0, (size_t)nbf * nbf * sizeof(double), stream);
    cudaMemsetAsync(b->dsums.ptr, 0, 2 * sizeof(double) * b->qcs.size(), stream);
    cudaMemsetAsync(b->dqueue.ptr, 0, SWEEP_QSTRIDE * b->qcs.size(), stream);
    const JKJob job = {dev_D, dev_J, dev_K};
    int nl = 0;
    long long maxout = 1;
    for(const auto & q : b->qcs)
        if(q.ntask > 0)
            maxout = std::max<long long>(maxout, q.nout);
    const int ns = SWEEP_SIDE + 1;
    const long long part = scratch_doubles / ns;
    if(scratch_doubles >= b->total_out || part < maxout)
    {
        // one stream: a scratch buffer that holds the whole sweep is used as
        // the full layout (each class digested from its own range), a
        // smaller one streams every class through it
        for(size_t k = 0; k < b->qcs.size(); k++)
        {
            if(b->qcs[k].ntask == 0)
                continue;
            rc = issue_class(b, k, prec, dev_scratch, scratch_doubles, stream, &job);
            if(rc < 0)
                return rc;
            nl += rc;
        }
    }
    else
    {
        // the classes on SWEEP_SIDE + 1 streams at once, as a full-layout
        // sweep runs them, each stream streaming its classes through its own
        // part of the scratch buffer (J and K take atomic adds from all)
        if(!b->fork)
        {
            cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
            for(int i = 0; i < SWEEP_SIDE; i++)
            {
                cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
                cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
            }
        }
        std::vector<size_t> order(b->qcs.size());
        std::iota(order.begin(), order.end(), 0);
        auto cost = [&](size_t k) {
            const QClass & q = b->qcs[k];
            const int L = q.req[0] + q.req[1] + q.req[2] + q.req[3];
            return (double)q.ntask * q.nout * (1.0 + L);
        };
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return cost(x) > cost(y); });
        double load[SWEEP_SIDE + 1] = {};
        cudaEventRecord(b->fork, stream);
        for(int i = 0; i < SWEEP_SIDE; i++)
            cudaStreamWaitEvent(b->side[i], b->fork, 0);
        for(size_t k : order)
        {
            if(b->qcs[k].ntask == 0)
                continue;
            int sidx = 0;
            for(int i = 1; i <= SWEEP_SIDE; i++)
                if(load[i] < load[sidx]) sidx = i;
            load[sidx] += cost(k);
            set_workspace_override(sidx ? &b->side_ws[sidx - 1] : nullptr);
            rc = issue_class(b, k, prec, dev_scratch + sidx * part, part, sidx ? b->side[sidx - 1] : stream, &job);
            set_workspace_override(nullptr);
            if(rc < 0)
                break;
            nl += rc;
        }
        for(int i = 0; i < SWEEP_SIDE; i++)
        {
            cudaEventRecord(b->join[i], b->side[i]);
            cudaStreamWaitEvent(stream, b->join[i], 0);
        }
        if(rc < 0)
            return rc;
    }
    rc = jk_finish(b, job, stream);
    return rc < 0 ? rc : nl + rc;
}
