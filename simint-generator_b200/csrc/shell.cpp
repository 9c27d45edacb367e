// Shells and multi-shell-pairs: the host side of the drop-in API.
//
// Layout and arithmetic follow skel/simint/shell/shell.c (allocation
// :131-185, normalisation :248-278, pair fill :425-582, concatenation
// :605-873); screening values follow skel/simint/shell/shell_screen.c.
// Differences: Schwarz primitive screening evaluates all diagonal (ab|ab)
// integrals of a pair list in one GPU launch instead of one library call per
// primitive pair, and the screen padding never writes past the array end
// (shell_screen.c:207-212 rounds a per-pair local index).

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

#include "simint/simint.h"
#include "simint_b200.h"

// Pair data of at least this many bytes lives in page-locked host memory
// (when a CUDA device is present and SIMINT_B200_PIN_PAIRS is not 0): the
// compute calls then copy a pair set's arrays to the device with one DMA
// and build the device records there, instead of packing them on the host.
#define PAIR_PIN_MIN ((size_t)256 << 10)

namespace {
std::mutex g_pin_mutex;
std::unordered_set<const void *> g_pinned;

bool pin_enabled()
{
    static const bool on = [] {
        const char * e = getenv("SIMINT_B200_PIN_PAIRS");
        if(e && atoi(e) == 0)
            return false;
        int n = 0;
        if(cudaGetDeviceCount(&n) != cudaSuccess)
        {
            cudaGetLastError();
            return false;
        }
        return n > 0;
    }();
    return on;
}

void * pair_alloc(size_t n)
{
    if(n >= PAIR_PIN_MIN && pin_enabled())
    {
        void * p = nullptr;
        if(cudaHostAlloc(&p, n, cudaHostAllocPortable) == cudaSuccess)
        {
            std::lock_guard<std::mutex> lk(g_pin_mutex);
            g_pinned.insert(p);
            return p;
        }
        cudaGetLastError();
    }
    return SIMINT_ALLOC(n);
}

void pair_free(void * p)
{
    bool pinned;
    {
        std::lock_guard<std::mutex> lk(g_pin_mutex);
        pinned = g_pinned.erase(p) > 0;
    }
    if(pinned)
        cudaFreeHost(p);
    else
        SIMINT_FREE(p);
}
} // namespace

namespace sb200 {
bool pair_data_pinned(const simint_multi_shellpair * P)
{
    if(!P->ptr)
        return false;
    std::lock_guard<std::mutex> lk(g_pin_mutex);
    return g_pinned.count(P->ptr) > 0;
}
}

#define SQRT_TWO_PI_52 5.91496717279561287782347843505365022963403204272156069835237
#define SQRT_TWO_TIMES_PI_52 24.739429451193148050228357586821944304008810699990039583

// pi^(3/2) (2l-1)!! / 2^l   (skel/simint/shell/shell_constants.c:13-36)
static double norm_fac(int l)
{
    double df = 1.0;
    for(int k = 2 * l - 1; k > 0; k -= 2)
        df *= k;
    return std::pow(M_PI, 1.5) * df / std::ldexp(1.0, l);
}

extern "C" {

void simint_initialize_shell(struct simint_shell * G)
{
    G->ptr = NULL;
    G->memsize = 0;
}

void simint_initialize_shells(int n, struct simint_shell * G)
{
    for(int i = 0; i < n; i++)
        simint_initialize_shell(G + i);
}

void simint_allocate_shell(int nprim, struct simint_shell * G)
{
    const size_t memsize = 2 * (size_t)nprim * sizeof(double);
    if(G->memsize < memsize)
    {
        simint_free_shell(G);
        G->ptr = malloc(memsize);
        G->memsize = memsize;
    }
    G->alpha = (double *)G->ptr;
    G->coef = (double *)G->ptr + nprim;
}

void simint_free_shell(struct simint_shell * G)
{
    if(G->ptr != NULL)
        free(G->ptr);
    simint_initialize_shell(G);
}

void simint_free_shells(int n, struct simint_shell * G)
{
    for(int i = 0; i < n; i++)
        simint_free_shell(G + i);
}

void simint_copy_shell(struct simint_shell const * src, struct simint_shell * dest)
{
    simint_allocate_shell(src->nprim, dest);
    dest->nprim = src->nprim;
    dest->am = src->am;
    dest->x = src->x;
    dest->y = src->y;
    dest->z = src->z;
    memcpy(dest->alpha, src->alpha, src->nprim * sizeof(double));
    memcpy(dest->coef, src->coef, src->nprim * sizeof(double));
}

void simint_normalize_shells(int n, struct simint_shell * G)
{
    for(int i = 0; i < n; ++i)
    {
        const double m = (double)G[i].am + 1.5;
        const double m2 = 0.5 * m;
        double sum = 0.0;
        for(int j = 0; j < G[i].nprim; j++)
            for(int k = 0; k < G[i].nprim; k++)
            {
                const double a1 = G[i].alpha[j], c1 = G[i].coef[j];
                const double a2 = G[i].alpha[k], c2 = G[i].coef[k];
                sum += (c1 * c2 * std::pow(a1 * a2, m2)) / (std::pow(a1 + a2, m));
            }
        const double norm = 1.0 / std::sqrt(sum * norm_fac(G[i].am));
        for(int j = 0; j < G[i].nprim; ++j)
            G[i].coef[j] *= norm * std::pow(G[i].alpha[j], m2);
    }
}

void simint_create_shell(int nprim, int am, double x, double y, double z,
                         double const * alpha, double const * coef, struct simint_shell * G)
{
    simint_allocate_shell(nprim, G);
    G->am = am;
    G->nprim = nprim;
    G->x = x;
    G->y = y;
    G->z = z;
    memcpy(G->alpha, alpha, nprim * sizeof(double));
    memcpy(G->coef, coef, nprim * sizeof(double));
}

void simint_create_zero_shell(struct simint_shell * G)
{
    const double alpha[1] = {0.0};
    const double coef[1] = {1.0};
    simint_create_shell(1, 0, 0.0, 0.0, 0.0, alpha, coef, G);
}

void simint_initialize_multi_shellpair(struct simint_multi_shellpair * P)
{
    P->ptr = NULL;
    P->memsize = 0;
}

void simint_initialize_multi_shellpairs(int n, struct simint_multi_shellpair * P)
{
    for(int i = 0; i < n; i++)
        simint_initialize_multi_shellpair(P + i);
}

void simint_free_multi_shellpair(struct simint_multi_shellpair * P)
{
    if(P->ptr != NULL)
        pair_free(P->ptr);
    simint_initialize_multi_shellpair(P);
}

void simint_free_multi_shellpairs(int n, struct simint_multi_shellpair * P)
{
    for(int i = 0; i < n; i++)
        simint_free_multi_shellpair(P + i);
}

} // extern "C"

// one block: 11 prim arrays (+screen) (+alpha2, beta2), AB x/y/z, nprim12
static void allocate_base(int npair, int nprim, struct simint_multi_shellpair * P, int screen_method)
{
    const size_t dprim = (size_t)nprim * sizeof(double);
    const size_t dpair = (size_t)npair * sizeof(double);
    const size_t ipair = (size_t)npair * sizeof(int);
    int narr = 11 + (screen_method ? 1 : 0) + 2;
    const size_t memsize = dprim * narr + dpair * 3 + ipair;
    if(P->memsize < memsize)
    {
        simint_free_multi_shellpair(P);
        P->ptr = pair_alloc(memsize);
        P->memsize = memsize;
    }
    char * base = (char *)P->ptr;
    int c = 0;
    P->x = (double *)(base + dprim * c++);
    P->y = (double *)(base + dprim * c++);
    P->z = (double *)(base + dprim * c++);
    P->PA_x = (double *)(base + dprim * c++);
    P->PA_y = (double *)(base + dprim * c++);
    P->PA_z = (double *)(base + dprim * c++);
    P->PB_x = (double *)(base + dprim * c++);
    P->PB_y = (double *)(base + dprim * c++);
    P->PB_z = (double *)(base + dprim * c++);
    P->alpha = (double *)(base + dprim * c++);
    P->prefac = (double *)(base + dprim * c++);
    P->screen = screen_method ? (double *)(base + dprim * c++) : NULL;
    P->alpha2 = (double *)(base + dprim * c++);
    P->beta2 = (double *)(base + dprim * c++);
    P->AB_x = (double *)(base + dprim * c);
    P->AB_y = (double *)(base + dprim * c + dpair);
    P->AB_z = (double *)(base + dprim * c + 2 * dpair);
    P->nprim12 = (int *)(base + dprim * c + 3 * dpair);
}

static int pair_nprim(const struct simint_shell * A, const struct simint_shell * B)
{
    return compare_shell(A, B) ? (A->nprim * (A->nprim + 1)) / 2 : A->nprim * B->nprim;
}

extern "C" {

void simint_allocate_multi_shellpair2(int npair, struct simint_shell const * AB,
                                      struct simint_multi_shellpair * P, int screen_method)
{
    int nprim = 0, batch = 0;
    for(int i = 0; i < npair; i++)
    {
        batch += pair_nprim(&AB[2 * i], &AB[2 * i + 1]);
        if(((i + 1) % SIMINT_NSHELL_SIMD) == 0 || i + 1 >= npair)
        {
            nprim += SIMINT_SIMD_ROUND(batch);
            batch = 0;
        }
    }
    allocate_base(npair, nprim, P, screen_method);
}

void simint_allocate_multi_shellpair(int na, struct simint_shell const * A,
                                     int nb, struct simint_shell const * B,
                                     struct simint_multi_shellpair * P, int screen_method)
{
    std::vector<simint_shell> AB(2 * (size_t)na * nb);
    size_t k = 0;
    for(int i = 0; i < na; ++i)
        for(int j = 0; j < nb; ++j)
        {
            AB[k++] = A[i];
            AB[k++] = B[j];
        }
    simint_allocate_multi_shellpair2(na * nb, AB.data(), P, screen_method);
}

} // extern "C"

namespace sb200 {
// Schwarz values of every primitive pair of a pair list, evaluated on the
// GPU in one launch (defined in batch.cu).  out follows the padded slot
// layout of the pair list; returns 0 on success.
int prim_schwarz_batch(int npair, const simint_shell * AB, double * out);
// The whole fill on the GPU (pairfill.cu); 0 on success.
int gpu_fill_multi_shellpair2(int npair, const simint_shell * AB, simint_multi_shellpair * P, int screen_method);
int pair_fill_mode();
int ensure_device();
}

// Whether a pair list's fill runs on the GPU: the mode set by
// simint_b200_set_pair_fill, in automatic mode lists of 4096 or more padded
// primitive pairs, and only with a device.
static bool fill_on_gpu(int npair, const simint_shell * AB)
{
    const int mode = sb200::pair_fill_mode();
    if(mode == SIMINT_B200_PAIR_FILL_HOST || npair <= 0)
        return false;
    if(mode == SIMINT_B200_PAIR_FILL_AUTO)
    {
        int npad = 0, batch = 0;
        for(int s = 0; s < npair; s++)
        {
            batch += pair_nprim(&AB[2 * s], &AB[2 * s + 1]);
            if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= npair)
            {
                npad += SIMINT_SIMD_ROUND(batch);
                batch = 0;
            }
        }
        if(npad < 4096)
            return false;
    }
    return sb200::ensure_device() == 0;
}

// descending screen order inside one shell pair (shell.c:37-128); a stable
// insertion sort is used, which keeps equal values in fill order
static void sort_pair(struct simint_multi_shellpair * P, int lo, int n)
{
    for(int a = lo + 1; a < lo + n; a++)
        for(int b = a; b > lo && P->screen[b - 1] < P->screen[b]; b--)
        {
            double * arr[14] = {P->x, P->y, P->z, P->PA_x, P->PA_y, P->PA_z, P->PB_x, P->PB_y,
                                P->PB_z, P->alpha, P->prefac, P->screen, P->alpha2, P->beta2};
            for(double * v : arr)
                std::swap(v[b - 1], v[b]);
        }
}

extern "C" {

void simint_fill_multi_shellpair2(int npair, struct simint_shell const * AB,
                                  struct simint_multi_shellpair * P, int screen_method)
{
    // pair sets are filled one at a time in the process (set-up work; the
    // Schwarz values of a screened fill create a pair set of their own, so
    // the lock is recursive)
    static std::recursive_mutex fill_mutex;
    std::lock_guard<std::recursive_mutex> fill_lock(fill_mutex);
    if(fill_on_gpu(npair, AB))
    {
        const int rc = sb200::gpu_fill_multi_shellpair2(npair, AB, P, screen_method);
        if(rc == 0)
            return;
        fprintf(stderr, "simint_b200: GPU pair fill failed (%s); filling on the host\n", simint_b200_last_error());
    }
    P->nshell12 = npair;
    P->nshell12_clip = npair;
    P->nprim = 0;
    P->screen_max = 1.e99;   // shell.c:434 (only ever raised)
    if(screen_method == SIMINT_SCREEN_SCHWARZ && npair > 0)
    {
        if(sb200::prim_schwarz_batch(npair, AB, P->screen) != 0)
        {
            // screening values could not be computed: keep every primitive
            fprintf(stderr, "simint_b200: Schwarz screening failed: %s\n", simint_b200_last_error());
            int npad = 0, batch = 0;
            for(int s = 0; s < npair; s++)
            {
                batch += pair_nprim(&AB[2 * s], &AB[2 * s + 1]);
                if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= npair)
                {
                    npad += SIMINT_SIMD_ROUND(batch);
                    batch = 0;
                }
            }
            for(int s = 0; s < npad; s++) P->screen[s] = INFINITY;
        }
    }
    int idx = 0;
    for(int s = 0; s < npair; s++)
    {
        const simint_shell * A = &AB[2 * s];
        const simint_shell * B = &AB[2 * s + 1];
        const int same = compare_shell(A, B);
        const int start = idx;
        if(screen_method == SIMINT_SCREEN_FASTSCHWARZ)
        {
            int k = idx;
            for(int i = 0; i < A->nprim; i++)
                for(int j = 0; j < (same ? i + 1 : B->nprim); j++)
                {
                    const double a = A->alpha[i], b = B->alpha[j];
                    const double p = a + b, oop = 1.0 / p, rho = (a * b) / p;
                    const double Rx = A->x - B->x, Ry = A->y - B->y, Rz = A->z - B->z;
                    const double R2 = Rx * Rx + Ry * Ry + Rz * Rz;
                    double g = SQRT_TWO_TIMES_PI_52 * std::pow(oop, 2.5) * std::exp(-2.0 * rho * R2);
                    g *= A->coef[i] * A->coef[i] * B->coef[j] * B->coef[j];
                    P->screen[k++] = g;
                }
        }
        if(screen_method)
        {
            double m = 0.0;
            for(int k = idx; k < idx + pair_nprim(A, B); k++)
                m = std::max(m, P->screen[k]);
            P->screen_max = std::max(m, P->screen_max);
        }
        P->am1 = A->am;
        P->am2 = B->am;
        const double Xab_x = A->x - B->x, Xab_y = A->y - B->y, Xab_z = A->z - B->z;
        const double Xab = Xab_x * Xab_x + Xab_y * Xab_y + Xab_z * Xab_z;
        for(int i = 0; i < A->nprim; ++i)
        {
            const double ai = A->alpha[i];
            const double AxAa = A->x * ai, AyAa = A->y * ai, AzAa = A->z * ai;
            const int jend = same ? i + 1 : B->nprim;
            for(int j = 0; j < jend; ++j)
            {
                const double aj = B->alpha[j];
                const double sum = ai + aj, mul = ai * aj;
                P->prefac[idx] = A->coef[i] * B->coef[j] * std::exp(-Xab * mul / sum) * SQRT_TWO_PI_52 / sum;
                if(same && i != j)
                    P->prefac[idx] *= 2.0;
                P->x[idx] = (AxAa + aj * B->x) / sum;
                P->y[idx] = (AyAa + aj * B->y) / sum;
                P->z[idx] = (AzAa + aj * B->z) / sum;
                P->PA_x[idx] = P->x[idx] - A->x;
                P->PA_y[idx] = P->y[idx] - A->y;
                P->PA_z[idx] = P->z[idx] - A->z;
                P->PB_x[idx] = P->x[idx] - B->x;
                P->PB_y[idx] = P->y[idx] - B->y;
                P->PB_z[idx] = P->z[idx] - B->z;
                P->alpha[idx] = sum;
                if(same && i != j)
                {
                    P->alpha2[idx] = sum;
                    P->beta2[idx] = sum;
                }
                else
                {
                    P->alpha2[idx] = 2.0 * ai;
                    P->beta2[idx] = 2.0 * aj;
                }
                ++idx;
            }
        }
        const int np = pair_nprim(A, B);
        P->AB_x[s] = Xab_x;
        P->AB_y[s] = Xab_y;
        P->AB_z[s] = Xab_z;
        if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= npair)
            while(idx < SIMINT_SIMD_ROUND(idx))
            {
                P->alpha[idx] = 1.0;
                P->prefac[idx] = 0.0;
                P->x[idx] = P->y[idx] = P->z[idx] = 0.0;
                P->PA_x[idx] = P->PA_y[idx] = P->PA_z[idx] = 0.0;
                P->PB_x[idx] = P->PB_y[idx] = P->PB_z[idx] = 0.0;
                if(P->screen)
                    P->screen[idx] = 0.0;
                P->alpha2[idx] = 1.0;
                P->beta2[idx] = 1.0;
                idx++;
            }
        P->nprim12[s] = np;
        P->nprim += np;
        if(screen_method && P->nprim > 1)
            sort_pair(P, start, np);
    }
}

void simint_fill_multi_shellpair(int na, struct simint_shell const * A,
                                 int nb, struct simint_shell const * B,
                                 struct simint_multi_shellpair * P, int screen_method)
{
    std::vector<simint_shell> AB(2 * (size_t)na * nb);
    size_t k = 0;
    for(int i = 0; i < na; ++i)
        for(int j = 0; j < nb; ++j)
        {
            AB[k++] = A[i];
            AB[k++] = B[j];
        }
    simint_fill_multi_shellpair2(na * nb, AB.data(), P, screen_method);
}

void simint_create_multi_shellpair(int na, struct simint_shell const * A,
                                   int nb, struct simint_shell const * B,
                                   struct simint_multi_shellpair * P, int screen_method)
{
    simint_allocate_multi_shellpair(na, A, nb, B, P, screen_method);
    simint_fill_multi_shellpair(na, A, nb, B, P, screen_method);
}

void simint_create_multi_shellpair2(int npair, struct simint_shell const * AB,
                                    struct simint_multi_shellpair * P, int screen_method)
{
    simint_allocate_multi_shellpair2(npair, AB, P, screen_method);
    simint_fill_multi_shellpair2(npair, AB, P, screen_method);
}

static void pad_tail(struct simint_multi_shellpair * P, int & idx)
{
    while(idx < SIMINT_SIMD_ROUND(idx))
    {
        P->alpha[idx] = 1.0;
        P->prefac[idx] = 0.0;
        P->x[idx] = P->y[idx] = P->z[idx] = 0.0;
        P->PA_x[idx] = P->PA_y[idx] = P->PA_z[idx] = 0.0;
        P->PB_x[idx] = P->PB_y[idx] = P->PB_z[idx] = 0.0;
        if(P->screen)
            P->screen[idx] = 0.0;
        P->alpha2[idx] = 1.0;
        P->beta2[idx] = 1.0;
        idx++;
    }
}

// shell.c:605-730.  The reference reads every input pair from index 0 of
// its arrays (Pin[i]->x[p]), i.e. it assumes each input holds one padded
// batch; we read each input shell pair from its own padded offset, which is
// the same thing for such inputs and correct for longer ones.
void simint_cat_multi_shellpair(int nmpair, struct simint_multi_shellpair const ** Pin,
                                struct simint_multi_shellpair * Pout, int screen_method)
{
    if(nmpair <= 0)
        return;
    int nshell12 = 0;
    for(int i = 0; i < nmpair; i++)
        nshell12 += Pin[i]->nshell12;
    int nprim = 0, batch = 0, ipair = 0;
    for(int i = 0; i < nmpair; i++)
        for(int j = 0; j < Pin[i]->nshell12; j++)
        {
            batch += Pin[i]->nprim12[j];
            if(((ipair + 1) % SIMINT_NSHELL_SIMD) == 0 || ipair + 1 >= nshell12)
            {
                nprim += SIMINT_SIMD_ROUND(batch);
                batch = 0;
            }
            ipair++;
        }
    allocate_base(nshell12, nprim, Pout, screen_method);
    Pout->am1 = Pin[0]->am1;
    Pout->am2 = Pin[0]->am2;
    Pout->screen_max = 0.0;
    Pout->nprim = 0;
    int idx = 0, s = 0;
    for(int i = 0; i < nmpair; i++)
    {
        const simint_multi_shellpair * Q = Pin[i];
        int src = 0;
        for(int j = 0; j < Q->nshell12; j++)
        {
            for(int p = 0; p < Q->nprim12[j]; p++, idx++)
            {
                const int k = src + p;
                Pout->x[idx] = Q->x[k]; Pout->y[idx] = Q->y[k]; Pout->z[idx] = Q->z[k];
                Pout->PA_x[idx] = Q->PA_x[k]; Pout->PA_y[idx] = Q->PA_y[k]; Pout->PA_z[idx] = Q->PA_z[k];
                Pout->PB_x[idx] = Q->PB_x[k]; Pout->PB_y[idx] = Q->PB_y[k]; Pout->PB_z[idx] = Q->PB_z[k];
                Pout->alpha[idx] = Q->alpha[k];
                Pout->prefac[idx] = Q->prefac[k];
                Pout->alpha2[idx] = Q->alpha2[k];
                Pout->beta2[idx] = Q->beta2[k];
                if(screen_method)
                    Pout->screen[idx] = Q->screen ? Q->screen[k] : 0.0;
            }
            Pout->screen_max = std::max(Pout->screen_max, Q->screen_max);
            Pout->AB_x[s] = Q->AB_x[j];
            Pout->AB_y[s] = Q->AB_y[j];
            Pout->AB_z[s] = Q->AB_z[j];
            Pout->nprim12[s] = Q->nprim12[j];
            src += Q->nprim12[j];
            if(((j + 1) % SIMINT_NSHELL_SIMD) == 0 || j + 1 >= Q->nshell12)
                src = SIMINT_SIMD_ROUND(src);
            if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= nshell12)
                pad_tail(Pout, idx);
            s++;
        }
        Pout->nprim += Q->nprim;
    }
    Pout->nshell12 = nshell12;
    Pout->nshell12_clip = nshell12;
}

} // extern "C"

namespace sb200 {
// dst = the shell pairs of src in the order order[0..nshell12), laid out as
// simint_create_multi_shellpair would lay them out for that pair list (the
// same padding rule, the same per-pair primitive order and values).
void permute_multi_shellpair(const simint_multi_shellpair * src, const int * order, simint_multi_shellpair * dst)
{
    const int n = src->nshell12;
    const int screen_method = src->screen ? SIMINT_SCREEN_SCHWARZ : 0;
    std::vector<int> start(n > 0 ? n : 1);
    int idx = 0;
    for(int p = 0; p < n; p++)
    {
        start[p] = idx;
        idx += src->nprim12[p];
        if(((p + 1) % SIMINT_NSHELL_SIMD) == 0 || p + 1 >= n)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    int nprim = 0, batch = 0;
    for(int s = 0; s < n; s++)
    {
        batch += src->nprim12[order[s]];
        if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= n)
        {
            nprim += SIMINT_SIMD_ROUND(batch);
            batch = 0;
        }
    }
    allocate_base(n, nprim, dst, screen_method);
    dst->am1 = src->am1;
    dst->am2 = src->am2;
    dst->nprim = src->nprim;
    dst->nshell12 = n;
    dst->nshell12_clip = n;
    dst->screen_max = src->screen_max;
    idx = 0;
    for(int s = 0; s < n; s++)
    {
        const int p = order[s];
        for(int k = start[p]; k < start[p] + src->nprim12[p]; k++, idx++)
        {
            dst->x[idx] = src->x[k]; dst->y[idx] = src->y[k]; dst->z[idx] = src->z[k];
            dst->PA_x[idx] = src->PA_x[k]; dst->PA_y[idx] = src->PA_y[k]; dst->PA_z[idx] = src->PA_z[k];
            dst->PB_x[idx] = src->PB_x[k]; dst->PB_y[idx] = src->PB_y[k]; dst->PB_z[idx] = src->PB_z[k];
            dst->alpha[idx] = src->alpha[k];
            dst->prefac[idx] = src->prefac[k];
            dst->alpha2[idx] = src->alpha2[k];
            dst->beta2[idx] = src->beta2[k];
            if(screen_method)
                dst->screen[idx] = src->screen[k];
        }
        dst->AB_x[s] = src->AB_x[p];
        dst->AB_y[s] = src->AB_y[p];
        dst->AB_z[s] = src->AB_z[p];
        dst->nprim12[s] = src->nprim12[p];
        if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= n)
            pad_tail(dst, idx);
    }
}
} // namespace sb200

extern "C" {

// shell.c:733-873: every input holds exactly one shell pair.
void simint_cat_shellpairs(int nmpair, struct simint_multi_shellpair const ** Pin,
                           struct simint_multi_shellpair * Pout, int screen_method)
{
    simint_cat_multi_shellpair(nmpair, Pin, Pout, screen_method);
}

// ---------------- screening ------------------------------------------------

double simint_primscreen_fastschwarz(struct simint_shell const * A, struct simint_shell const * B,
                                     double * out)
{
    const int same = compare_shell(A, B);
    double total_max = 0.0;
    int idx = 0;
    for(int i = 0; i < A->nprim; i++)
        for(int j = 0; j < (same ? i + 1 : B->nprim); j++)
        {
            const double a = A->alpha[i], b = B->alpha[j];
            const double p = a + b, oop = 1.0 / p, rho = (a * b) / p;
            const double Rx = A->x - B->x, Ry = A->y - B->y, Rz = A->z - B->z;
            const double R2 = Rx * Rx + Ry * Ry + Rz * Rz;
            double g = SQRT_TWO_TIMES_PI_52 * std::pow(oop, 2.5) * std::exp(-2.0 * rho * R2);
            g *= A->coef[i] * A->coef[i] * B->coef[j] * B->coef[j];
            if(out)
                out[idx] = g;
            total_max = std::max(total_max, g);
            idx++;
        }
    return total_max;
}

double simint_primscreen_schwarz(struct simint_shell const * A, struct simint_shell const * B,
                                 double * out)
{
    simint_shell AB[2] = {*A, *B};
    const int np = pair_nprim(A, B);
    std::vector<double> tmp(SIMINT_SIMD_ROUND(np) + 8, 0.0);
    if(sb200::prim_schwarz_batch(1, AB, tmp.data()) != 0)
        return INFINITY;
    double m = 0.0;
    for(int k = 0; k < np; k++)
        m = std::max(m, tmp[k]);
    if(out)
    {
        // padded like the pair arrays (a single pair: up to the next multiple of 8)
        for(int k = 0; k < SIMINT_SIMD_ROUND(np); k++)
            out[k] = tmp[k];
    }
    return m;
}

double simint_primscreen(struct simint_shell const * A, struct simint_shell const * B,
                         double * out, int screen_method)
{
    if(screen_method == SIMINT_SCREEN_FASTSCHWARZ)
        return simint_primscreen_fastschwarz(A, B, out);
    return simint_primscreen_schwarz(A, B, out);
}

double simint_shellscreen_fastschwarz(struct simint_shell const * A, struct simint_shell const * B)
{
    const int same = compare_shell(A, B);
    double val = 0.0;
    for(int i = 0; i < A->nprim; i++)
        for(int j = 0; j < (same ? i + 1 : B->nprim); j++)
        {
            const double a = A->alpha[i], b = B->alpha[j];
            const double p = a + b, oop = 1.0 / p, rho = (a * b) / p;
            const double Rx = A->x - B->x, Ry = A->y - B->y, Rz = A->z - B->z;
            const double R2 = Rx * Rx + Ry * Ry + Rz * Rz;
            double g = SQRT_TWO_TIMES_PI_52 * std::pow(oop, 2.5) * std::exp(-2.0 * rho * R2);
            g *= A->coef[i] * A->coef[i] * B->coef[j] * B->coef[j];
            val += g;
        }
    return val;
}

double simint_shellscreen_schwarz(struct simint_shell const * A, struct simint_shell const * B)
{
    struct simint_multi_shellpair P;
    simint_initialize_multi_shellpair(&P);
    simint_create_multi_shellpair(1, A, 1, B, &P, SIMINT_SCREEN_NONE);
    const int n12 = ((A->am + 1) * (A->am + 2) / 2) * ((B->am + 1) * (B->am + 2) / 2);
    std::vector<double> ints((size_t)n12 * n12);
    double m = 0.0;
    if(simint_compute_eri(&P, &P, 0.0, NULL, ints.data()) > 0)
        for(double v : ints)
            m = std::max(m, std::fabs(v));
    else
        m = INFINITY;
    simint_free_multi_shellpair(&P);
    return m;
}

double simint_shellscreen(struct simint_shell const * A, struct simint_shell const * B, int screen_method)
{
    if(screen_method == SIMINT_SCREEN_FASTSCHWARZ)
        return simint_shellscreen_fastschwarz(A, B);
    return simint_shellscreen_schwarz(A, B);
}

} // extern "C"
