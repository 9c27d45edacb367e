// Host runtime of the B200 Simint engine: simint_init/finalize,
// simint_compute_eri(_deriv) and the run-time dispatch to the generated
// per-class kernels.
//
// Reference behaviour kept (skel/simint/ostei/ostei.c:10-41,
// skel/simint/simint_eri.c:4-22): the tolerance is squared, a pair-level
// test returns -1 without writing when P.screen_max*Q.screen_max < tol^2,
// the result count is nshell12_clip(P)*nshell12_clip(Q), output is
// bra-pair-major then Cartesian a,b,c,d row major.
//
// Everything else is B200-specific: the pair SoA is packed into 128-byte
// primitive records, uploaded with one copy per pair set, one thread
// computes one shell quartet, kets are visited in order of primitive count,
// and the result comes back with one device-to-host copy.

#include <cuda_runtime.h>
#include <algorithm>
#include <csignal>
#include <execinfo.h>
#include <unistd.h>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "simint/simint.h"
#include "simint_b200.h"
#include "kernels.h"
#include "runtime.h"
#include "hostpool.h"
#include "gen/boys_grid.inc"

namespace sb200 {
void load_tune_file();

static std::mutex g_mutex;
static bool g_initialised = false;
static int g_ordering = SIMINT_B200_ORDERING_PSI4;
static int g_precision = SIMINT_B200_PREC_FP64;
static double g_gate = 0.0;
static KernelTable g_table;
static std::map<std::array<int, 4>, int> g_unique;     // unique class -> index in g_table
static std::vector<double *> g_boys_dev;              // per device: Boys tables
static thread_local std::string t_last_error;
static thread_local long long t_launches = 0;

void set_error(const std::string & s)
{
    t_last_error = s;
}

void count_launch(long long n) { t_launches += n; }

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }
int ncart_of(int l) { return ncart(l); }

// Psi4 position of (i,j,k) inside its shell
static int psi4_index(int i, int j, int k)
{
    const int l = i + j + k;
    (void)j;
    return ((l - i) * (l - i + 1)) / 2 + k;
}

int cart_index(int i, int j, int k, int ordering)
{
    const int l = i + j + k;
    if(ordering == SIMINT_B200_ORDERING_GAMESS && (l == 2 || l == 3))
    {
        // generator/Ordering_GAMESS.cpp:20-41
        static const int g2[6][3] = {{2,0,0},{0,2,0},{0,0,2},{1,1,0},{1,0,1},{0,1,1}};
        static const int g3[10][3] = {{3,0,0},{0,3,0},{0,0,3},{2,1,0},{2,0,1},
                                      {1,2,0},{0,2,1},{1,0,2},{0,1,2},{1,1,1}};
        const int n = ncart(l);
        for(int t = 0; t < n; t++)
        {
            const int * g = (l == 2) ? g2[t] : g3[t];
            if(g[0] == i && g[1] == j && g[2] == k)
                return t;
        }
    }
    return psi4_index(i, j, k);
}

void carts(int l, std::vector<std::array<int, 3>> & out)
{
    out.clear();
    for(int i = l; i >= 0; i--)
        for(int j = l - i; j >= 0; j--)
            out.push_back({i, j, l - i - j});
}

UniqueMap unique_of(const int am[4])
{
    // emit.unique_class: canonical (a>=b, c>=d, (a+b, a) >= (c+d, c))
    UniqueMap u;
    int a = am[0], b = am[1], c = am[2], d = am[3];
    int sb = a < b, sk = c < d;
    if(sb) std::swap(a, b);
    if(sk) std::swap(c, d);
    int pq = (a + b < c + d) || (a + b == c + d && a < c);
    if(pq)
    {
        std::swap(a, c);
        std::swap(b, d);
        std::swap(sb, sk);
    }
    u.am[0] = a; u.am[1] = b; u.am[2] = c; u.am[3] = d;
    u.swapB = sb; u.swapK = sk; u.pq = pq;
    return u;
}

// Output index table: for the unique class element n (Psi4 order), the
// position inside the requested class's shell-quartet block.
std::vector<unsigned short> make_oidx(const int req[4], const UniqueMap & u, int ordering)
{
    std::vector<std::array<int, 3>> ca, cb, cc, cd;
    carts(u.am[0], ca); carts(u.am[1], cb); carts(u.am[2], cc); carts(u.am[3], cd);
    std::vector<unsigned short> o;
    o.reserve(ca.size() * cb.size() * cc.size() * cd.size());
    for(auto & gA : ca) for(auto & gB : cb) for(auto & gC : cc) for(auto & gD : cd)
    {
        std::array<int, 3> b0 = u.swapB ? gB : gA, b1 = u.swapB ? gA : gB;
        std::array<int, 3> k0 = u.swapK ? gD : gC, k1 = u.swapK ? gC : gD;
        std::array<int, 3> p0, p1, q0, q1;
        if(!u.pq) { p0 = b0; p1 = b1; q0 = k0; q1 = k1; }
        else      { q0 = b0; q1 = b1; p0 = k0; p1 = k1; }
        const int i0 = cart_index(p0[0], p0[1], p0[2], ordering);
        const int i1 = cart_index(p1[0], p1[1], p1[2], ordering);
        const int i2 = cart_index(q0[0], q0[1], q0[2], ordering);
        const int i3 = cart_index(q1[0], q1[1], q1[2], ordering);
        o.push_back((unsigned short)(((i0 * ncart(req[1]) + i1) * ncart(req[2]) + i2) * ncart(req[3]) + i3));
    }
    return o;
}

const ClassKernels * find_kernels(const UniqueMap & u)
{
    auto it = g_unique.find({u.am[0], u.am[1], u.am[2], u.am[3]});
    if(it == g_unique.end())
        return nullptr;
    return &g_table.list[it->second];
}

int ensure_device()
{
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess)
    {
        cudaGetLastError();
        set_error("no CUDA device available");
        return -1;
    }
    int ndev = 0;
    if(cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0)
    {
        cudaGetLastError();
        set_error("no CUDA device available");
        return -1;
    }
    std::lock_guard<std::mutex> lk(g_mutex);
    if((int)g_boys_dev.size() < ndev)
        g_boys_dev.resize(ndev, nullptr);
    if(!g_boys_dev[dev])
    {
        double * d = nullptr;
        const size_t n1 = sizeof(simint_b200_boys_grid_host), n2 = sizeof(simint_b200_boys_longfac_host);
        if(cudaMalloc(&d, n1 + n2) != cudaSuccess ||
           cudaMemcpy(d, simint_b200_boys_grid_host, n1, cudaMemcpyHostToDevice) != cudaSuccess ||
           cudaMemcpy((char *)d + n1, simint_b200_boys_longfac_host, n2, cudaMemcpyHostToDevice) != cudaSuccess)
        {
            set_error(std::string("Boys table upload failed: ") + cudaGetErrorString(cudaGetLastError()));
            return -1;
        }
        g_boys_dev[dev] = d;
    }
    return dev;
}

const double * boys_table()
{
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mutex);
    return dev < (int)g_boys_dev.size() ? g_boys_dev[dev] : nullptr;
}

int ordering() { return g_ordering; }
int precision() { return g_precision; }
double gate() { return g_gate; }

void init_tables()
{
    std::lock_guard<std::mutex> lk(g_mutex);
    if(g_initialised)
        return;
    simint_b200_register_generated(g_table);
    for(size_t k = 0; k < g_table.list.size(); k++)
    {
        const auto & e = g_table.list[k];
        g_unique[{e.am[0], e.am[1], e.am[2], e.am[3]}] = (int)k;
    }
    load_tune_file();
    const char * o = getenv("SIMINT_B200_ORDERING");
    if(o && (!strcmp(o, "gamess") || !strcmp(o, "GAMESS") || !strcmp(o, "1")))
        g_ordering = SIMINT_B200_ORDERING_GAMESS;
    g_initialised = true;
}

// ---------------------------------------------------------------------
// Per-thread device workspace (grow-only)
// ---------------------------------------------------------------------

static thread_local Workspace * t_ws_override = nullptr;

Workspace & workspace()
{
    static thread_local Workspace w;
    return t_ws_override ? *t_ws_override : w;
}

void set_workspace_override(Workspace * w) { t_ws_override = w; }

bool DevBuf::reserve(size_t n)
{
    if(n <= cap)
        return true;
    if(ptr)
    {
        // kernels queued by asynchronous entry points may still use it
        cudaDeviceSynchronize();
        cudaFree(ptr);
    }
    ptr = nullptr;
    cap = 0;
    size_t want = std::max(n, (size_t)4096);
    want = (want * 5) / 4;
    if(cudaMalloc(&ptr, want) != cudaSuccess)
    {
        cudaGetLastError();
        ptr = nullptr;
        return false;
    }
    cap = want;
    return true;
}

void DevBuf::release()
{
    if(ptr)
        cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
}

bool HostBuf::reserve(size_t n)
{
    if(n <= cap)
        return true;
    if(ptr)
        cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    size_t want = (std::max(n, (size_t)4096) * 5) / 4;
    if(cudaMallocHost(&ptr, want) != cudaSuccess)
    {
        cudaGetLastError();
        ptr = nullptr;
        return false;
    }
    cap = want;
    return true;
}

void HostBuf::release()
{
    if(ptr)
        cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
}

Workspace::~Workspace()
{
    // device buffers are released by simint_finalize on the owning thread;
    // at process exit the driver reclaims them.
}

// Padded slot layout of a multi-shell-pair (shell.c:538-570): after every
// 16 shell pairs the slot index is rounded up to a multiple of 8.
void pair_starts(const simint_multi_shellpair * P, std::vector<int> & start, int & npad)
{
    start.resize(P->nshell12);
    int idx = 0;
    for(int p = 0; p < P->nshell12; p++)
    {
        start[p] = idx;
        idx += P->nprim12[p];
        if(((p + 1) % SIMINT_NSHELL_SIMD) == 0 || p + 1 >= P->nshell12)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    npad = idx;
}

// Pack one pair set into host staging memory: records, starts, counts, AB.
// Records of padded slots [g0, g1) (multiples of 8, the vector-screening
// groups) into rec (slot 0 of rec = slot g0), on the calling thread (pair
// sets large enough for packing to matter are page-locked and go up by DMA).
void pack_records(const simint_multi_shellpair * P, int npad, int g0, int g1, double * rec)
{
    const bool has_screen = P->screen != nullptr;
    g1 = std::min(g1, npad);
    if(g1 <= g0)
        return;
    auto body = [&](size_t b0, size_t b1) {
        for(int g = g0 + (int)b0 * 8; g < std::min(g0 + (int)b1 * 8, g1); g += 8)
        {
            double m = 0.0;
            const int ge = std::min(g + 8, g1);
            for(int s = g; s < ge; s++)
            {
                double * r = rec + (size_t)(s - g0) * SB_REC;
                r[0] = P->alpha[s]; r[1] = P->prefac[s];
                r[2] = P->x[s]; r[3] = P->y[s]; r[4] = P->z[s];
                r[5] = P->PA_x[s]; r[6] = P->PA_y[s]; r[7] = P->PA_z[s];
                r[8] = P->PB_x[s]; r[9] = P->PB_y[s]; r[10] = P->PB_z[s];
                r[11] = P->alpha2 ? P->alpha2[s] : 0.0;
                r[12] = P->beta2 ? P->beta2[s] : 0.0;
                const double sc = has_screen ? P->screen[s] : 0.0;
                r[13] = sc;
                r[15] = has_screen ? std::sqrt(std::max(sc, 0.0)) : INFINITY;
                m = std::max(m, sc);
            }
            for(int s = g; s < ge; s++)
                rec[(size_t)(s - g0) * SB_REC + 14] = m;
        }
    };
    body(0, (size_t)(g1 - g0 + 7) / 8);
}

// Layout of the packed pair set: records, then starts, counts and AB at
// 256-byte aligned offsets; optionally the padded start of every pair.
static size_t pack_layout(const simint_multi_shellpair * P, PackedLayout & L, std::vector<int> * start_out)
{
    std::vector<int> start;
    int npad = 0;
    pair_starts(P, start, npad);
    L.npad = npad;
    L.npair = P->nshell12;
    L.off_rec = 0;
    L.off_start = (size_t)npad * SB_REC * sizeof(double);
    L.off_nprim = L.off_start + ((P->nshell12 * sizeof(int) + 255) & ~(size_t)255);
    L.off_AB = L.off_nprim + ((P->nshell12 * sizeof(int) + 255) & ~(size_t)255);
    if(start_out)
        start_out->swap(start);
    return L.off_AB + 3 * (size_t)P->nshell12 * sizeof(double);
}

static void pack_meta(const simint_multi_shellpair * P, const PackedLayout & L, const std::vector<int> & start,
                      char * dst)
{
    memcpy(dst + L.off_start, start.data(), P->nshell12 * sizeof(int));
    memcpy(dst + L.off_nprim, P->nprim12, P->nshell12 * sizeof(int));
    double * ab = (double *)(dst + L.off_AB);
    for(int p = 0; p < P->nshell12; p++)
    {
        ab[3 * p + 0] = P->AB_x[p];
        ab[3 * p + 1] = P->AB_y[p];
        ab[3 * p + 2] = P->AB_z[p];
    }
}

// Pack one pair set into host staging memory: records, starts, counts, AB.
size_t pack_pairs(const simint_multi_shellpair * P, char * dst, PackedLayout & L)
{
    std::vector<int> start;
    const size_t total = pack_layout(P, L, &start);
    if(!dst)
        return total;
    pack_records(P, L.npad, 0, L.npad, (double *)(dst + L.off_rec));
    pack_meta(P, L, start, dst);
    return total;
}

// Byte offsets of a pair set's arrays inside its allocation (-1: absent).
struct SoaOffsets
{
    long long x, y, z, pax, pay, paz, pbx, pby, pbz, alpha, prefac, screen, a2, b2, abx, aby, abz, nprim12;
};

// The device records of pack_records, built from a device copy of the pair
// set's arrays: one thread per padded slot, the vector maximum of field 14
// over the aligned group of 8 slots (lanes 8k..8k+7 of a warp).
__global__ void k_soa_records(const char * __restrict__ soa, const SoaOffsets o, int npad,
                              double * __restrict__ rec)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = s < npad;
    auto A = [&](long long off) { return __ldg((const double *)(soa + off) + s); };
    const double sc = (in && o.screen >= 0) ? A(o.screen) : 0.0;
    double m = sc;
    #pragma unroll
    for(int d = 1; d < 8; d <<= 1)
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, d));
    if(!in)
        return;
    double * r = rec + (size_t)s * SB_REC;
    r[0] = A(o.alpha); r[1] = A(o.prefac);
    r[2] = A(o.x); r[3] = A(o.y); r[4] = A(o.z);
    r[5] = A(o.pax); r[6] = A(o.pay); r[7] = A(o.paz);
    r[8] = A(o.pbx); r[9] = A(o.pby); r[10] = A(o.pbz);
    r[11] = o.a2 >= 0 ? A(o.a2) : 0.0;
    r[12] = o.b2 >= 0 ? A(o.b2) : 0.0;
    r[13] = sc;
    r[14] = fmax(m, 0.0);
    r[15] = o.screen >= 0 ? sqrt(fmax(sc, 0.0)) : INFINITY;
}

__global__ void k_soa_meta(const char * __restrict__ soa, const SoaOffsets o, int npair, int * __restrict__ nprim,
                           double * __restrict__ ab)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if(p >= npair)
        return;
    nprim[p] = __ldg((const int *)(soa + o.nprim12) + p);
    ab[3 * p + 0] = __ldg((const double *)(soa + o.abx) + p);
    ab[3 * p + 1] = __ldg((const double *)(soa + o.aby) + p);
    ab[3 * p + 2] = __ldg((const double *)(soa + o.abz) + p);
}

// Whether every array of P lies inside its own allocation [ptr, ptr +
// memsize) with its full extent (npad slots, npair pairs): only then is one
// DMA of the allocation a copy of the pair set.  (A caller may point an
// array elsewhere, e.g. at a private copy of the screening values.)
bool pair_arrays_in_block(const simint_multi_shellpair * P, int npad)
{
    const char * b = (const char *)P->ptr;
    const char * e = b + P->memsize;
    auto in = [&](const void * a, size_t n) {
        const char * c = (const char *)a;
        return !a || (c >= b && c + n <= e);
    };
    const size_t dp = (size_t)npad * sizeof(double), dq = (size_t)P->nshell12 * sizeof(double);
    return in(P->x, dp) && in(P->y, dp) && in(P->z, dp) && in(P->PA_x, dp) && in(P->PA_y, dp) &&
           in(P->PA_z, dp) && in(P->PB_x, dp) && in(P->PB_y, dp) && in(P->PB_z, dp) && in(P->alpha, dp) &&
           in(P->prefac, dp) && in(P->screen, dp) && in(P->alpha2, dp) && in(P->beta2, dp) &&
           in(P->AB_x, dq) && in(P->AB_y, dq) && in(P->AB_z, dq) &&
           in(P->nprim12, (size_t)P->nshell12 * sizeof(int)) && P->x && P->alpha && P->prefac && P->nprim12;
}

// Pair set P (arrays in page-locked host memory) into the packed layout L at
// dpack on `stream`: the arrays the records need (2a and 2b only for
// derivatives) into dsoa at their offsets in the allocation, one DMA per run
// of adjacent arrays; the pair starts from hstart (page-locked,
// start.size() ints, kept until the stream has run); the records and
// metadata built on the device.
int upload_pinned_pairs(const simint_multi_shellpair * P, const PackedLayout & L, const std::vector<int> & start,
                        char * dpack, DevBuf & dsoa, int * hstart, cudaStream_t stream, int deriv)
{
    if(!dsoa.reserve(P->memsize))
    {
        set_error("out of device memory for pair data");
        return SIMINT_B200_ERR_CUDA;
    }
    const char * base = (const char *)P->ptr;
    auto off = [&](const void * a) { return a ? (long long)((const char *)a - base) : -1LL; };
    SoaOffsets o;
    o.x = off(P->x); o.y = off(P->y); o.z = off(P->z);
    o.pax = off(P->PA_x); o.pay = off(P->PA_y); o.paz = off(P->PA_z);
    o.pbx = off(P->PB_x); o.pby = off(P->PB_y); o.pbz = off(P->PB_z);
    o.alpha = off(P->alpha); o.prefac = off(P->prefac); o.screen = off(P->screen);
    // 2a and 2b only weigh derivative integrals
    o.a2 = deriv ? off(P->alpha2) : -1;
    o.b2 = deriv ? off(P->beta2) : -1;
    o.abx = off(P->AB_x); o.aby = off(P->AB_y); o.abz = off(P->AB_z); o.nprim12 = off(P->nprim12);
    // one DMA per run of adjacent arrays the records need
    const size_t dprim = (size_t)L.npad * sizeof(double), dpair = (size_t)L.npair * sizeof(double);
    std::vector<std::pair<long long, size_t>> r;
    for(long long a : {o.x, o.y, o.z, o.pax, o.pay, o.paz, o.pbx, o.pby, o.pbz, o.alpha, o.prefac, o.screen,
                       o.a2, o.b2})
        if(a >= 0)
            r.push_back({a, dprim});
    for(long long a : {o.abx, o.aby, o.abz})
        if(a >= 0)
            r.push_back({a, dpair});
    if(o.nprim12 >= 0)
        r.push_back({o.nprim12, (size_t)L.npair * sizeof(int)});
    std::sort(r.begin(), r.end());
    for(size_t k = 0; k < r.size();)
    {
        long long a = r[k].first, e = a + (long long)r[k].second;
        size_t m = k + 1;
        for(; m < r.size() && r[m].first <= e; m++)
            e = std::max(e, r[m].first + (long long)r[m].second);
        cudaMemcpyAsync((char *)dsoa.ptr + a, (const char *)P->ptr + a, (size_t)(e - a), cudaMemcpyHostToDevice,
                        stream);
        k = m;
    }
    memcpy(hstart, start.data(), (size_t)L.npair * sizeof(int));
    cudaMemcpyAsync(dpack + L.off_start, hstart, (size_t)L.npair * sizeof(int), cudaMemcpyHostToDevice, stream);
    k_soa_records<<<(unsigned)((L.npad + 255) / 256), 256, 0, stream>>>((const char *)dsoa.ptr, o, L.npad,
                                                                      (double *)(dpack + L.off_rec));
    k_soa_meta<<<(unsigned)((L.npair + 255) / 256), 256, 0, stream>>>((const char *)dsoa.ptr, o, L.npair,
                                                                    (int *)(dpack + L.off_nprim),
                                                                    (double *)(dpack + L.off_AB));
    count_launch(2);
    return 0;
}

PairSetDev device_view(const char * base, const PackedLayout & L, double screen_max)
{
    PairSetDev d;
    d.prim = (const double *)(base + L.off_rec);
    d.pstart = (const int *)(base + L.off_start);
    d.nprim = (const int *)(base + L.off_nprim);
    d.AB = (const double *)(base + L.off_AB);
    d.screen_max = screen_max;
    d.npair = L.npair;
    return d;
}

// Device copy of an output-index table, cached per (device, class, variant).
const unsigned short * oidx_table(const int req[4], const UniqueMap & u, int ord)
{
    static std::mutex m;
    static std::map<std::array<int, 7>, unsigned short *> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::array<int, 7> key = {dev, req[0], req[1], req[2], req[3], ord, 0};
    std::lock_guard<std::mutex> lk(m);
    auto it = cache.find(key);
    if(it != cache.end())
        return it->second;
    std::vector<unsigned short> h = make_oidx(req, u, ord);
    unsigned short * d = nullptr;
    if(cudaMalloc(&d, h.size() * sizeof(unsigned short)) != cudaSuccess)
    {
        cudaGetLastError();
        return nullptr;
    }
    cudaMemcpy(d, h.data(), h.size() * sizeof(unsigned short), cudaMemcpyHostToDevice);
    cache[key] = d;
    return d;
}

} // namespace sb200

using namespace sb200;

// =====================================================================
// C API
// =====================================================================

// Opt-in crash report (SIMINT_B200_SEGV_TRACE=1): a segmentation fault in
// any thread prints that thread's call stack (addresses inside the loaded
// libraries) on stderr before the process ends as it would have.
static void segv_report(int sig)
{
    void * frames[64];
    const int n = backtrace(frames, 64);
    static const char msg[] = "simint_b200: fatal signal, call stack:\n";
    if(write(2, msg, sizeof(msg) - 1) < 0) {}
    backtrace_symbols_fd(frames, n, 2);
    signal(sig, SIG_DFL);
    raise(sig);
}

extern "C" void simint_init(void)
{
    init_tables();
    static std::once_flag once;
    std::call_once(once, [] {
        const char * e = getenv("SIMINT_B200_SEGV_TRACE");
        if(e && atoi(e) != 0)
            signal(SIGSEGV, segv_report);
    });
}

extern "C" void simint_finalize(void)
{
    Workspace & w = workspace();
    w.dpair.release();
    w.dout.release();
    w.dkord.release();
    w.hstage.release();
    w.hout.release();
    if(w.stream)
    {
        cudaStreamDestroy(w.stream);
        w.stream = nullptr;
    }
}

extern "C" int simint_b200_set_ordering(int o)
{
    if(o != SIMINT_B200_ORDERING_PSI4 && o != SIMINT_B200_ORDERING_GAMESS)
        return SIMINT_B200_ERR_ARG;
    if(g_ordering != o)
        sb200::bump_settings_epoch();
    g_ordering = o;
    return 0;
}

extern "C" int simint_b200_get_ordering(void) { return g_ordering; }

extern "C" int simint_b200_set_precision(int mode, double gate)
{
    if(mode != SIMINT_B200_PREC_FP64 && mode != SIMINT_B200_PREC_MIXED)
        return SIMINT_B200_ERR_ARG;
    if(g_precision != mode || g_gate != gate)
        sb200::bump_settings_epoch();
    g_precision = mode;
    g_gate = gate;
    return 0;
}

extern "C" int simint_b200_get_precision(void) { return g_precision; }

extern "C" const char * simint_b200_last_error(void) { return t_last_error.c_str(); }

extern "C" long long simint_b200_launch_count(void) { return t_launches; }

extern "C" size_t simint_eri_worksize(int derorder, int maxam)
{
    return simint_ostei_worksize(derorder, maxam);
}

extern "C" size_t simint_eri_workmem(int derorder, int maxam)
{
    return simint_ostei_workmem(derorder, maxam);
}

namespace sb200 {

// Untuned default: the register kernel while its contracted tops fit
// registers (above ~200 accumulators it spills), else the cooperative kernel
// (the column kernel runs where the autotuner or a caller chooses it).
static int default_variant(const int req[4], int deriv, const ClassKernels * k)
{
    (void)req;
    (void)deriv;
    return (k && k->ntop <= 200) ? VAR_STRAIGHT : VAR_COOP2;
}

// Launch the kernel of class req for the prepared arguments a (P, Q,
// tasks or kord, ntask, check, tol2, out, nout filled by the caller).
int launch_class(KernArgs & a, const int req[4], int deriv, int mode, int prec,
                 cudaStream_t stream)
{
    for(int k = 0; k < 4; k++)
        if(req[k] < 0 || req[k] > SIMINT_OSTEI_MAXAM)
        {
            set_error("angular momentum outside 0..SIMINT_OSTEI_MAXAM");
            return SIMINT_B200_ERR_CLASS;
        }
    if(a.ntask == 0)
        return 0;
    const UniqueMap u = unique_of(req);
    a.swapB = u.swapB; a.swapK = u.swapK; a.pq = u.pq;
    a.boys = boys_table();
    const ClassKernels * k = deriv == 0 ? find_kernels(u) : nullptr;
    int v = variant_of(req, deriv, prec);
    if(v >= 100)
    {
        // the FP64 form of a variant, chosen for a class in mixed mode
        v -= 100;
        prec = SIMINT_B200_PREC_FP64;
        a.gate = 0.0;
    }
    if(v == VAR_DEFAULT)
        v = default_variant(req, deriv, k);
    // a small rectangle (one simint_compute_eri call) gives a thread-per-
    // quartet kernel a handful of CTAs: the warp-per-quartet form of the
    // same register kernel spreads it over 32x the threads
    if(mode == 0 && a.ntask < 16384 && k && k->fnw[0][0])
    {
        if(v == VAR_STRAIGHT)
            v = VAR_WARP;
        else if(v == VAR_STRAIGHT64)
            v = VAR_WARP64;
    }
    if((v == VAR_STRAIGHT || v == VAR_STRAIGHT64) && k)
    {
        a.oidx = oidx_table(req, u, ordering());
        if(!a.oidx)
        {
            set_error("cannot allocate output index table");
            return SIMINT_B200_ERR_CUDA;
        }
        const int threads = 128;
        const long long blocks = (a.ntask + threads - 1) / threads;
        KernFn fn = k->fn[mode][(prec == SIMINT_B200_PREC_MIXED && v == VAR_STRAIGHT) ? 1 : 0];
        fn<<<(unsigned)blocks, threads, 0, stream>>>(a);
        count_launch(1);
        return 0;
    }
    if((v == VAR_WARP || v == VAR_WARP64) && k && k->fnw[mode][0])
    {
        a.oidx = oidx_table(req, u, ordering());
        if(!a.oidx)
        {
            set_error("cannot allocate output index table");
            return SIMINT_B200_ERR_CUDA;
        }
        const int threads = 128;           // 4 shell quartets per block
        const long long blocks = (a.ntask + 3) / 4;
        KernFn fn = k->fnw[mode][(prec == SIMINT_B200_PREC_MIXED && v == VAR_WARP) ? 1 : 0];
        fn<<<(unsigned)blocks, threads, 0, stream>>>(a);
        count_launch(1);
        return 0;
    }
    if(col_is_variant(v) && col_supported(req, deriv, v))
        return launch_col(a, req, mode, prec, stream, v);
    if(coop2_is_variant(v) && coop2_supported(req, deriv, v))
        return launch_coop2(a, req, deriv, mode, prec, stream, v);
    if(v == VAR_COOP1 && coop_supported(req, deriv))
        return launch_coop(a, req, deriv, mode, stream);
    if(v == VAR_GENERIC)
        return launch_generic(a, req, u, deriv, mode, stream);
    if(coop2_supported(req, deriv))
        return launch_coop2(a, req, deriv, mode, prec, stream);
    if(coop_supported(req, deriv))
        return launch_coop(a, req, deriv, mode, stream);
    return launch_generic(a, req, u, deriv, mode, stream);
}

// Whether launch_class runs class req on a CTA-per-quartet kernel that takes
// its shell quartets from KernArgs::wq (the cooperative and column kernels):
// the same choice of kernel as launch_class.
bool class_uses_queue(const int req[4], int deriv, int prec)
{
    const UniqueMap u = unique_of(req);
    const ClassKernels * k = deriv == 0 ? find_kernels(u) : nullptr;
    int v = variant_of(req, deriv, prec);
    if(v >= 100)
        v -= 100;
    if(v == VAR_DEFAULT)
        v = default_variant(req, deriv, k);
    if((v == VAR_STRAIGHT || v == VAR_STRAIGHT64) && k)
        return false;
    if((v == VAR_WARP || v == VAR_WARP64) && k && k->fnw[2][0])
        return false;
    if(col_is_variant(v) && col_supported(req, deriv, v))
        return true;
    if(coop2_is_variant(v) && coop2_supported(req, deriv, v))
        return true;
    if(v == VAR_COOP1 && coop_supported(req, deriv))
        return false;
    if(v == VAR_GENERIC)
        return false;
    return coop2_supported(req, deriv);
}

// The reference's (ss|ss) kernel (skel/ostei_s_s_s_s.c) sets the screening
// values of the lanes past the last ket primitive to zero before testing a
// partial last vector -- in the caller's pair data: later calls that reach
// further into the same ket list see the zeros.  For a ket list clipped
// inside a vector (nshell12_clip < nshell12) the first call's test of that
// vector therefore covers only its slots below the clip.  [v0, v1) are those
// slots (padded primitive indices of Q), or an empty range when the call is
// not (ss|ss), is not clipped or the clip ends on a vector boundary.  The
// caller's data is left unchanged here.
void ssss_clip_vector(const simint_multi_shellpair * P, const simint_multi_shellpair * Q, int & v0, int & v1)
{
    v0 = v1 = 0;
    if(P->am1 || P->am2 || Q->am1 || Q->am2 || Q->nshell12_clip >= Q->nshell12 || Q->nshell12_clip <= 0)
        return;
    int idx = 0;
    for(int p = 0; p < Q->nshell12_clip; p++)
    {
        idx += Q->nprim12[p];
        if(((p + 1) % SIMINT_NSHELL_SIMD) == 0 && p + 1 < Q->nshell12_clip)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    if(idx % SIMINT_SIMD_LEN == 0)
        return;
    v0 = idx - idx % SIMINT_SIMD_LEN;
    v1 = idx;
}

// Run one P x Q rectangle on the device.  dP/dQ already hold packed pair
// data; writes nout doubles per shell quartet to dout.
int launch_rectangle(const simint_multi_shellpair * P, const PairSetDev & dP,
                     const simint_multi_shellpair * Q, const PairSetDev & dQ,
                     const int * dkord, double screen_tol, int deriv, int prec, double gatev,
                     double * dout, cudaStream_t stream, int nqc)
{
    const int req[4] = {P->am1, P->am2, Q->am1, Q->am2};
    const int nc = ncart(req[0]) * ncart(req[1]) * ncart(req[2]) * ncart(req[3]);
    KernArgs a;
    memset(&a, 0, sizeof(a));
    a.P = dP;
    a.Q = dQ;
    a.kord = dkord;
    a.nQ = Q->nshell12_clip;
    a.nQc = nqc < 0 ? a.nQ : nqc;
    a.ntask = (long long)P->nshell12_clip * a.nQc;
    a.check = (screen_tol > 0.0) && P->screen && Q->screen;
    a.tol2 = screen_tol * screen_tol;
    a.gate = (prec == SIMINT_B200_PREC_MIXED) ? gatev : 0.0;
    a.out = dout;
    a.nout = nc * (deriv ? 12 : 1);
    if(a.check)
        ssss_clip_vector(P, Q, a.kvec0, a.kvec1);
    return launch_class(a, req, deriv, 0, prec, stream);
}

} // namespace sb200

// Large calls: the ket pairs go through the device in chunks (multiples of
// 16 pairs, so chunk records are whole padded groups) so host packing of
// chunk k+1 and the copy of chunk k-1's results into the caller's memory run
// while the GPU uploads, computes and downloads chunk k.  Results are the
// same as the one-shot path (each chunk's kets in primitive-count order).
// Opt-in phase trace of the host-buffer entry points (environment variable
// SIMINT_B200_TRACE=1): one line per simint_compute_eri call on stderr with
// the host time spent packing pair records, issuing the uploads, issuing the
// kernels and the download, waiting for the GPU and copying results into the
// caller's memory, and (one-shot calls) the device time of the kernels and of
// the download between CUDA events on the call's stream.
namespace {
struct CallTrace
{
    typedef std::chrono::steady_clock clk;
    bool on;
    clk::time_point t0;
    double pack = 0.0, upload = 0.0, issue = 0.0, wait = 0.0, copy = 0.0;
    float kern = -1.0f, down = -1.0f;     // device time of the kernels and of the download
    CallTrace() : on(enabled()), t0(on ? clk::now() : clk::time_point()) {}
    // device-side marks on the call's stream (events of the calling thread)
    cudaEvent_t * events()
    {
        thread_local cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
        if(!ev[0])
            for(int i = 0; i < 3; i++)
                if(cudaEventCreate(&ev[i]) != cudaSuccess)
                {
                    cudaGetLastError();
                    ev[i] = nullptr;
                }
        return ev;
    }
    void mark(int i, cudaStream_t s)
    {
        if(on && events()[i])
            cudaEventRecord(events()[i], s);
    }
    // after the stream has been synchronised
    void device_times()
    {
        if(!on)
            return;
        cudaEvent_t * ev = events();
        if(ev[0] && ev[1] && ev[2])
        {
            if(cudaEventElapsedTime(&kern, ev[0], ev[1]) != cudaSuccess ||
               cudaEventElapsedTime(&down, ev[1], ev[2]) != cudaSuccess)
            {
                cudaGetLastError();
                kern = down = -1.0f;
            }
        }
    }
    static bool enabled()
    {
        static const bool e = [] {
            const char * v = getenv("SIMINT_B200_TRACE");
            return v && atoi(v) != 0;
        }();
        return e;
    }
    template<typename F>
    void time(double & acc, F && f)
    {
        if(!on)
        {
            f();
            return;
        }
        const clk::time_point a = clk::now();
        f();
        acc += std::chrono::duration<double, std::milli>(clk::now() - a).count();
    }
    void report(const simint_multi_shellpair * P, const simint_multi_shellpair * Q, size_t outbytes,
                bool pipelined) const
    {
        if(!on)
            return;
        const double tot = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
        fprintf(stderr, "simint_b200 trace: (%d %d|%d %d) bra %d ket %d out %.1f MB pipelined %d: "
                "total %.3f ms, pack %.3f, upload %.3f, launch %.3f, wait %.3f, copy %.3f; device: kernels %.3f, "
                "download %.3f\n", P->am1, P->am2, Q->am1, Q->am2, P->nshell12_clip, Q->nshell12_clip,
                outbytes / 1e6, pipelined ? 1 : 0, tot, pack, upload, issue, wait, copy, kern, down);
    }
};
} // namespace

// Ket pairs c0 .. c1-1 of Q in decreasing primitive count, equal counts in
// list order (a stable counting sort; a comparison sort for counts above
// 4096), into out.
static void kets_by_nprim(const simint_multi_shellpair * Q, int c0, int c1, int * out)
{
    int mx = 0;
    for(int q = c0; q < c1; q++)
        mx = std::max(mx, Q->nprim12[q]);
    if(mx > 4096)
    {
        for(int q = c0; q < c1; q++) out[q - c0] = q;
        std::stable_sort(out, out + (c1 - c0), [Q](int x, int y) { return Q->nprim12[x] > Q->nprim12[y]; });
        return;
    }
    std::vector<int> first(mx + 2, 0);
    for(int q = c0; q < c1; q++)
        first[mx - std::max(Q->nprim12[q], 0) + 1]++;
    for(int v = 1; v <= mx + 1; v++)
        first[v] += first[v - 1];
    for(int q = c0; q < c1; q++)
        out[first[mx - std::max(Q->nprim12[q], 0)]++] = q;
}

static int compute_eri_pipelined(int deriv, const simint_multi_shellpair * P, const simint_multi_shellpair * Q,
                                 double screen_tol, double * integrals, int nc)
{
    Workspace & w = workspace();
    const int nP = P->nshell12_clip, nQ = Q->nshell12_clip;
    const size_t outbytes = (size_t)nP * nQ * nc * sizeof(double);
    // few chunks: each launch must still fill the GPU
    const size_t moved = outbytes + (size_t)Q->nprim * SB_REC * sizeof(double);
    const int nch = (int)std::min<size_t>(4, std::max<size_t>(2, moved / ((size_t)32 << 20)));
    const int cq = std::max(16, ((nQ + nch - 1) / nch + 15) & ~15);
    PackedLayout LP, LQ;
    std::vector<int> qstart;
    const size_t szP = (pack_pairs(P, nullptr, LP) + 255) & ~(size_t)255;
    const size_t szQ = (pack_layout(Q, LQ, &qstart) + 255) & ~(size_t)255;
    const size_t szK = ((size_t)nQ * sizeof(int) + 255) & ~(size_t)255;
    // staging: P | Q meta (records area unused) | two chunk slots (records + kord)
    size_t maxrec = 0;
    for(int c0 = 0; c0 < nQ; c0 += cq)
    {
        const int c1 = std::min(nQ, c0 + cq);
        const int g0 = qstart[c0], g1 = c1 >= nQ ? LQ.npad : qstart[c1];
        maxrec = std::max(maxrec, (size_t)(g1 - g0) * SB_REC * sizeof(double));
    }
    const size_t slot = ((maxrec + (size_t)cq * sizeof(int)) + 255) & ~(size_t)255;
    if(!w.hstage.reserve(szP + szQ + 2 * slot) || !w.dpair.reserve(szP + szQ + szK) || !w.dout.reserve(outbytes)
       || !w.hout.reserve(outbytes))
    {
        set_error("out of memory for a pipelined call");
        return SIMINT_B200_ERR_CUDA;
    }
    CallTrace tr;
    char * h = (char *)w.hstage.ptr;
    char * d = (char *)w.dpair.ptr;
    const bool pinP = pair_data_pinned(P) && pair_arrays_in_block(P, LP.npad);
    const bool pinQ = pair_data_pinned(Q) && pair_arrays_in_block(Q, LQ.npad);
    std::vector<int> pstart;
    if(pinP)
        pack_layout(P, LP, &pstart);
    tr.time(tr.pack, [&] {
        if(!pinP)
            pack_pairs(P, h, LP);
        if(!pinQ)
            pack_meta(Q, LQ, qstart, h + szP);
    });
    if(pinP || pinQ)
    {
        if(!w.dsoa.reserve(std::max(pinP ? P->memsize : 0, pinQ ? Q->memsize : 0)))
        {
            set_error("out of device memory for pair data");
            return SIMINT_B200_ERR_CUDA;
        }
    }
    // P, and Q's starts/counts/AB (everything after the records); a pinned
    // Q goes up whole, its records built on the device
    int rc0 = pinP ? upload_pinned_pairs(P, LP, pstart, d, w.dsoa, (int *)h, w.stream, deriv)
                   : (cudaMemcpyAsync(d, h, szP, cudaMemcpyHostToDevice, w.stream), 0);
    if(rc0 == 0)
        rc0 = pinQ ? upload_pinned_pairs(Q, LQ, qstart, d + szP, w.dsoa, (int *)(h + szP), w.stream, deriv)
                   : (cudaMemcpyAsync(d + szP + LQ.off_start, h + szP + LQ.off_start, szQ - LQ.off_start,
                                      cudaMemcpyHostToDevice, w.stream), 0);
    if(rc0 != 0)
    {
        cudaStreamSynchronize(w.stream);
        return rc0;
    }
    const PairSetDev dP = device_view(d, LP, P->screen_max);
    const PairSetDev dQ = device_view(d + szP, LQ, Q->screen_max);
    int * dkord = (int *)(d + szP + szQ);
    if(!w.dstream && cudaStreamCreateWithFlags(&w.dstream, cudaStreamNonBlocking) != cudaSuccess)
    {
        set_error("cudaStreamCreate failed");
        cudaStreamSynchronize(w.stream);
        return SIMINT_B200_ERR_CUDA;
    }
    static thread_local std::vector<cudaEvent_t> ev;
    const int nchunk = (nQ + cq - 1) / cq;
    while((int)ev.size() < 2 * nchunk + 2)
    {
        cudaEvent_t e;
        if(cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
        {
            set_error("cudaEventCreate failed");
            cudaStreamSynchronize(w.stream);
            return SIMINT_B200_ERR_CUDA;
        }
        ev.push_back(e);
    }
    const size_t rowbytes = (size_t)nQ * nc * sizeof(double);
    auto copy_out = [&](int k) {
        const int c0 = k * cq, c1 = std::min(nQ, c0 + cq);
        const size_t off = (size_t)c0 * nc * sizeof(double), len = (size_t)(c1 - c0) * nc * sizeof(double);
        if(nP == 1)
            parallel_copy((char *)integrals + off, (char *)w.hout.ptr + off, len);
        else
            parallel_for((size_t)nP, 1, [&](size_t r0, size_t r1) {
                for(size_t r = r0; r < r1; r++)
                    memcpy((char *)integrals + r * rowbytes + off, (char *)w.hout.ptr + r * rowbytes + off, len);
            });
    };
    int rc = 0;
    for(int k = 0; k < nchunk && rc == 0; k++)
    {
        const int c0 = k * cq, c1 = std::min(nQ, c0 + cq);
        const int g0 = qstart[c0], g1 = c1 >= nQ ? LQ.npad : qstart[c1];
        char * hs = h + szP + szQ + (size_t)(k & 1) * slot;
        if(k >= 2)
            tr.time(tr.wait, [&] { cudaEventSynchronize(ev[k & 1]); });   // staging slot of chunk k-2 uploaded
        const size_t recbytes = pinQ ? 0 : (size_t)(g1 - g0) * SB_REC * sizeof(double);
        int * kk = (int *)(hs + recbytes);
        tr.time(tr.pack, [&] {
            if(!pinQ)
                pack_records(Q, LQ.npad, g0, g1, (double *)hs);
            kets_by_nprim(Q, c0, c1, kk);
        });
        if(recbytes)
            cudaMemcpyAsync(d + szP + (size_t)g0 * SB_REC * sizeof(double), hs, recbytes, cudaMemcpyHostToDevice,
                            w.stream);
        cudaMemcpyAsync(dkord + c0, kk, (size_t)(c1 - c0) * sizeof(int), cudaMemcpyHostToDevice, w.stream);
        cudaEventRecord(ev[k & 1], w.stream);
        rc = launch_rectangle(P, dP, Q, dQ, dkord + c0, screen_tol, deriv, precision(), gate(),
                              (double *)w.dout.ptr, w.stream, c1 - c0);
        if(rc < 0)
            break;
        rc = 0;
        // the download of chunk k overlaps the upload and kernel of chunk k+1
        const size_t off = (size_t)c0 * nc * sizeof(double), len = (size_t)(c1 - c0) * nc * sizeof(double);
        cudaEventRecord(ev[2 + nchunk + k], w.stream);
        cudaStreamWaitEvent(w.dstream, ev[2 + nchunk + k], 0);
        if(nP == 1)
            cudaMemcpyAsync((char *)w.hout.ptr + off, (char *)w.dout.ptr + off, len, cudaMemcpyDeviceToHost,
                            w.dstream);
        else
            cudaMemcpy2DAsync((char *)w.hout.ptr + off, rowbytes, (char *)w.dout.ptr + off, rowbytes, len, nP,
                              cudaMemcpyDeviceToHost, w.dstream);
        cudaEventRecord(ev[2 + k], w.dstream);
        if(k >= 1)
        {
            tr.time(tr.wait, [&] { cudaEventSynchronize(ev[2 + k - 1]); });
            tr.time(tr.copy, [&] { copy_out(k - 1); });
        }
    }
    cudaError_t e = cudaSuccess, e2 = cudaSuccess;
    tr.time(tr.wait, [&] {
        e = cudaStreamSynchronize(w.stream);
        e2 = cudaStreamSynchronize(w.dstream);
    });
    if(e == cudaSuccess)
        e = e2;
    if(e == cudaSuccess)
        e = cudaGetLastError();
    if(rc < 0)
        return rc;
    if(e != cudaSuccess)
    {
        set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    tr.time(tr.copy, [&] { copy_out(nchunk - 1); });
    tr.report(P, Q, outbytes, true);
    return nP * nQ;
}

extern "C" int simint_compute_eri_deriv(int deriv,
                                        struct simint_multi_shellpair const * P,
                                        struct simint_multi_shellpair const * Q,
                                        double screen_tol, double * work, double * integrals)
{
    (void)work;
    if(!P || !Q || !integrals || deriv < 0 || deriv > SIMINT_OSTEI_MAXDER)
    {
        set_error("bad argument to simint_compute_eri_deriv");
        return SIMINT_B200_ERR_ARG;
    }
    // pair-level early exit (ostei.c:16-19)
    const double tol2 = screen_tol * screen_tol;
    if(screen_tol > 0.0 && (P->screen_max * Q->screen_max) < tol2)
        return -1;
    init_tables();
    if(ensure_device() < 0)
        return SIMINT_B200_ERR_NODEVICE;
    Workspace & w = workspace();
    if(!w.stream && cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess)
    {
        set_error("cudaStreamCreate failed");
        return SIMINT_B200_ERR_CUDA;
    }
    const long long nquart = (long long)P->nshell12_clip * Q->nshell12_clip;
    if(nquart == 0)
        return 0;
    {
        const int nc = ncart(P->am1) * ncart(P->am2) * ncart(Q->am1) * ncart(Q->am2) * (deriv ? 12 : 1);
        // pipelined when the call moves >= 16 MB (results down plus ket
        // records up: long ket lists of small classes are upload-bound)
        const size_t moved = (size_t)nquart * nc * sizeof(double) + (size_t)Q->nprim * SB_REC * sizeof(double);
        if(moved >= ((size_t)16 << 20) && Q->nshell12_clip >= 64)
            return compute_eri_pipelined(deriv, P, Q, screen_tol, integrals, nc);
    }
    CallTrace tr;
    PackedLayout LP, LQ;
    std::vector<int> pstart, qstart;
    const size_t szP = (pack_layout(P, LP, &pstart) + 255) & ~(size_t)255;
    const size_t szQ = (pack_layout(Q, LQ, &qstart) + 255) & ~(size_t)255;
    // pair sets in page-locked memory go up as their arrays in one DMA and
    // become records on the device; the others are packed on the host
    const bool pinP = pair_data_pinned(P) && pair_arrays_in_block(P, LP.npad);
    const bool pinQ = pair_data_pinned(Q) && pair_arrays_in_block(Q, LQ.npad);
    // ket order: by primitive count (descending), stable
    std::vector<int> kord(Q->nshell12_clip);
    kets_by_nprim(Q, 0, Q->nshell12_clip, kord.data());
    const size_t szK = (kord.size() * sizeof(int) + 255) & ~(size_t)255;
    if(!w.hstage.reserve(szP + szQ + szK) || !w.dpair.reserve(szP + szQ + szK))
    {
        set_error("out of memory for pair data");
        return SIMINT_B200_ERR_CUDA;
    }
    char * h = (char *)w.hstage.ptr;
    tr.time(tr.pack, [&] {
        if(!pinP)
        {
            pack_records(P, LP.npad, 0, LP.npad, (double *)(h + LP.off_rec));
            pack_meta(P, LP, pstart, h);
        }
        if(!pinQ)
        {
            pack_records(Q, LQ.npad, 0, LQ.npad, (double *)(h + szP + LQ.off_rec));
            pack_meta(Q, LQ, qstart, h + szP);
        }
        memcpy(h + szP + szQ, kord.data(), kord.size() * sizeof(int));
    });
    char * d = (char *)w.dpair.ptr;
    int rc_up = 0;
    tr.time(tr.upload, [&] {
        if(pinP || pinQ)
        {
            if(!w.dsoa.reserve(std::max(pinP ? P->memsize : 0, pinQ ? Q->memsize : 0)))
            {
                set_error("out of device memory for pair data");
                rc_up = SIMINT_B200_ERR_CUDA;
                return;
            }
            // the unused host staging of a pinned set holds its pair starts
            rc_up = pinP ? upload_pinned_pairs(P, LP, pstart, d, w.dsoa, (int *)h, w.stream, deriv)
                         : (cudaMemcpyAsync(d, h, szP, cudaMemcpyHostToDevice, w.stream), 0);
            if(rc_up == 0)
                rc_up = pinQ ? upload_pinned_pairs(Q, LQ, qstart, d + szP, w.dsoa, (int *)(h + szP), w.stream,
                                                   deriv)
                             : (cudaMemcpyAsync(d + szP, h + szP, szQ, cudaMemcpyHostToDevice, w.stream), 0);
            if(rc_up == 0)
                cudaMemcpyAsync(d + szP + szQ, h + szP + szQ, szK, cudaMemcpyHostToDevice, w.stream);
        }
        else
            cudaMemcpyAsync(d, h, szP + szQ + szK, cudaMemcpyHostToDevice, w.stream);
    });
    if(rc_up != 0)
    {
        // copies already queued read the staging buffer: let them finish
        // before the next call reuses it
        cudaStreamSynchronize(w.stream);
        return rc_up;
    }
    const PairSetDev dP = device_view(d, LP, P->screen_max);
    const PairSetDev dQ = device_view(d + szP, LQ, Q->screen_max);
    const int nc = ncart(P->am1) * ncart(P->am2) * ncart(Q->am1) * ncart(Q->am2) * (deriv ? 12 : 1);
    const size_t outbytes = (size_t)nquart * nc * sizeof(double);
    if(!w.dout.reserve(outbytes))
    {
        set_error("out of device memory for the output");
        return SIMINT_B200_ERR_CUDA;
    }
    int r = 0;
    // results through the pinned staging buffer (full-speed DMA; a copy
    // into pageable memory would go through the driver's own staging and
    // return only when done), then into the caller's memory on the host
    // threads
    const bool staged = w.hout.reserve(outbytes);
    tr.time(tr.issue, [&] {
        tr.mark(0, w.stream);
        r = launch_rectangle(P, dP, Q, dQ, (const int *)(d + szP + szQ), screen_tol, deriv,
                             precision(), gate(), (double *)w.dout.ptr, w.stream);
        tr.mark(1, w.stream);
        if(r >= 0)
            cudaMemcpyAsync(staged ? w.hout.ptr : (void *)integrals, w.dout.ptr, outbytes,
                            cudaMemcpyDeviceToHost, w.stream);
        tr.mark(2, w.stream);
    });
    if(r < 0)
    {
        cudaStreamSynchronize(w.stream);
        return r;
    }
    cudaError_t e = cudaSuccess;
    tr.time(tr.wait, [&] { e = cudaStreamSynchronize(w.stream); });
    if(e == cudaSuccess)
        e = cudaGetLastError();
    if(e != cudaSuccess)
    {
        set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    tr.device_times();
    if(staged)
        tr.time(tr.copy, [&] { parallel_copy(integrals, w.hout.ptr, outbytes); });
    tr.report(P, Q, outbytes, false);
    return (int)nquart;
}

namespace sb200 {

// Identity ket order per device for the device-resident entry point; grown
// (never shrunk) under a lock, so kernels already queued keep a valid
// buffer until the device is synchronised before a regrowth.
static const int * identity_kord(long long n)
{
    static std::mutex m;
    static std::map<int, std::pair<int *, long long>> bufs;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(m);
    auto & b = bufs[dev];
    if(b.second >= n)
        return b.first;
    long long cap = std::max<long long>(n, 1 << 16);
    std::vector<int> h(cap);
    for(long long k = 0; k < cap; k++)
        h[k] = (int)k;
    if(b.first)
    {
        cudaDeviceSynchronize();
        cudaFree(b.first);
        b = {nullptr, 0};
    }
    int * d = nullptr;
    if(cudaMalloc(&d, cap * sizeof(int)) != cudaSuccess)
        return nullptr;
    if(cudaMemcpy(d, h.data(), cap * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
    {
        cudaFree(d);
        return nullptr;
    }
    b = {d, cap};
    return d;
}

} // namespace sb200

extern "C" int simint_b200_compute_eri_device(int deriv,
                                              struct simint_multi_shellpair const * P, const void * dev_P,
                                              struct simint_multi_shellpair const * Q, const void * dev_Q,
                                              double screen_tol, double * dev_integrals, void * stream)
{
    if(!P || !Q || !dev_P || !dev_Q || !dev_integrals || deriv < 0 || deriv > SIMINT_OSTEI_MAXDER)
    {
        set_error("bad argument to simint_b200_compute_eri_device");
        return SIMINT_B200_ERR_ARG;
    }
    const double tol2 = screen_tol * screen_tol;
    if(screen_tol > 0.0 && (P->screen_max * Q->screen_max) < tol2)
        return -1;
    init_tables();
    if(ensure_device() < 0)
        return SIMINT_B200_ERR_NODEVICE;
    const long long nquart = (long long)P->nshell12_clip * Q->nshell12_clip;
    if(nquart == 0)
        return 0;
    const int * kord = identity_kord(Q->nshell12_clip);
    if(!kord)
    {
        set_error("cannot allocate the ket order");
        return SIMINT_B200_ERR_CUDA;
    }
    PackedLayout LP, LQ;
    pack_pairs(P, nullptr, LP);
    pack_pairs(Q, nullptr, LQ);
    const PairSetDev dP = device_view((const char *)dev_P, LP, P->screen_max);
    const PairSetDev dQ = device_view((const char *)dev_Q, LQ, Q->screen_max);
    int r = launch_rectangle(P, dP, Q, dQ, kord, screen_tol, deriv, precision(), gate(),
                             dev_integrals, (cudaStream_t)stream);
    if(r < 0)
        return r;
    cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess)
    {
        set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
        return SIMINT_B200_ERR_CUDA;
    }
    return (int)nquart;
}

extern "C" int simint_compute_eri(struct simint_multi_shellpair const * P,
                                  struct simint_multi_shellpair const * Q,
                                  double screen_tol, double * work, double * integrals)
{
    return simint_compute_eri_deriv(0, P, Q, screen_tol, work, integrals);
}

extern "C" long long simint_b200_count_primq(struct simint_multi_shellpair const * P,
                                             struct simint_multi_shellpair const * Q, double screen_tol)
{
    const double tol2 = screen_tol * screen_tol;
    if(screen_tol > 0.0 && P->screen_max * Q->screen_max < tol2)
        return 0;
    const bool check = screen_tol > 0.0 && P->screen && Q->screen;
    std::vector<int> ps, qs;
    int npP = 0, npQ = 0;
    pair_starts(P, ps, npP);
    pair_starts(Q, qs, npQ);
    std::vector<double> vmax((npQ + 7) / 8, 0.0);
    if(check)
    {
        for(int j = 0; j < npQ; j++)
            vmax[j / 8] = std::max(vmax[j / 8], Q->screen[j]);
        int v0, v1;
        ssss_clip_vector(P, Q, v0, v1);
        if(v1 > v0)
        {
            vmax[v0 / 8] = 0.0;
            for(int j = v0; j < v1; j++)
                vmax[v0 / 8] = std::max(vmax[v0 / 8], Q->screen[j]);
        }
    }
    long long n = 0;
    for(int ab = 0; ab < P->nshell12_clip; ab++)
        for(int i = ps[ab]; i < ps[ab] + P->nprim12[ab]; i++)
        {
            if(check && P->screen[i] * Q->screen_max < tol2)
                continue;
            for(int cd = 0; cd < Q->nshell12_clip; cd++)
                for(int j = qs[cd]; j < qs[cd] + Q->nprim12[cd]; j++)
                    if(!check || P->screen[i] * vmax[j / 8] >= tol2)
                        n++;
        }
    return n;
}

namespace sb200 {

static std::mutex g_var_mutex;
static std::map<std::array<int, 6>, int> g_variant;
static std::atomic<long long> g_settings_epoch{0};

long long settings_epoch() { return g_settings_epoch.load(); }
void bump_settings_epoch() { g_settings_epoch++; }

int variant_of(const int req[4], int deriv, int prec)
{
    std::lock_guard<std::mutex> lk(g_var_mutex);
    auto it = g_variant.find({req[0], req[1], req[2], req[3], deriv, prec});
    return it == g_variant.end() ? VAR_DEFAULT : it->second;
}

void set_variant(const int req[4], int deriv, int prec, int v)
{
    std::lock_guard<std::mutex> lk(g_var_mutex);
    g_variant[{req[0], req[1], req[2], req[3], deriv, prec}] = v;
    g_settings_epoch++;
}

bool has_straight(const int req[4])
{
    return find_kernels(unique_of(req)) != nullptr;
}

bool has_warp(const int req[4], int mode)
{
    const ClassKernels * k = find_kernels(unique_of(req));
    return k && k->fnw[mode][0];
}

// Tuning cache: a small JSON object {"a,b,c,d,deriv,prec": variant, ...}
// at $SIMINT_B200_TUNE_FILE, read at simint_init and written by the
// autotuner.
void load_tune_file()
{
    const char * f = getenv("SIMINT_B200_TUNE_FILE");
    if(!f)
        return;
    FILE * fp = fopen(f, "r");
    if(!fp)
        return;
    char line[256];
    while(fgets(line, sizeof(line), fp))
    {
        int q[6], v;
        if(sscanf(line, " \"%d,%d,%d,%d,%d,%d\": %d", &q[0], &q[1], &q[2], &q[3], &q[4], &q[5], &v) == 7)
            set_variant(q, q[4], q[5], v);
    }
    fclose(fp);
}

void save_tune_file()
{
    const char * f = getenv("SIMINT_B200_TUNE_FILE");
    if(!f)
        return;
    FILE * fp = fopen(f, "w");
    if(!fp)
        return;
    std::lock_guard<std::mutex> lk(g_var_mutex);
    fprintf(fp, "{\n");
    size_t n = 0;
    for(auto & e : g_variant)
    {
        fprintf(fp, "  \"%d,%d,%d,%d,%d,%d\": %d%s\n", e.first[0], e.first[1], e.first[2], e.first[3],
                e.first[4], e.first[5], e.second, ++n < g_variant.size() ? "," : "");
    }
    fprintf(fp, "}\n");
    fclose(fp);
}

} // namespace sb200

extern "C" int simint_b200_set_variant(const int am[4], int deriv, int prec, int variant)
{
    using namespace sb200;
    if(!am || (deriv != 0 && deriv != 1) ||
       (prec != SIMINT_B200_PREC_FP64 && prec != SIMINT_B200_PREC_MIXED))
        return SIMINT_B200_ERR_ARG;
    for(int k = 0; k < 4; k++)
        if(am[k] < 0 || am[k] > SIMINT_OSTEI_MAXAM)
            return SIMINT_B200_ERR_CLASS;
    bool ok = false;
    switch(variant)
    {
        case VAR_DEFAULT:
        case VAR_GENERIC:
            ok = true;
            break;
        case VAR_STRAIGHT:
        case VAR_STRAIGHT64:
            ok = deriv == 0 && has_straight(am);
            break;
        case VAR_WARP:
        case VAR_WARP64:
            ok = deriv == 0 && has_warp(am, 0) && has_warp(am, 2);
            break;
        case VAR_COOP1:
            ok = coop_supported(am, deriv);
            break;
        case 21: case 22: case 24: case 28:
        case 41: case 42: case 44: case 48:
        case 61: case 62: case 64: case 68:
            ok = coop2_supported(am, deriv, variant);
            break;
        case 81: case 82: case 83:
            ok = col_supported(am, deriv, variant);
            break;
        case 181: case 182: case 183:
            ok = prec == SIMINT_B200_PREC_MIXED && col_supported(am, deriv, variant - 100);
            break;
        case 121: case 122: case 124: case 128:
        case 141: case 142: case 144: case 148:
        case 161: case 162: case 164: case 168:
            ok = prec == SIMINT_B200_PREC_MIXED && coop2_supported(am, deriv, variant - 100);
            break;
        default:
            ok = false;
    }
    if(!ok)
    {
        set_error("kernel variant not available for this class");
        return SIMINT_B200_ERR_ARG;
    }
    set_variant(am, deriv, prec, variant);
    return 0;
}
