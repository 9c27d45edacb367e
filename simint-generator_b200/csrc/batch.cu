// Batched device work: primitive Schwarz screening of whole pair lists.
//
// simint_primscreen_schwarz (skel/simint/shell/shell_screen.c:127-223)
// computes, for every primitive pair (i,j) of a shell pair, the integrals
// (ab|ab) of the two uncontracted primitives and keeps the largest diagonal
// element max_mn |(a_m b_n | a_m b_n)|.  The reference does this with one
// library call per primitive pair.  Here the primitive pairs of a whole pair
// list become one multi-shell-pair of single-primitive pairs and all their
// (ab|ab) run as one task list on the GPU, followed by a reduction kernel
// that keeps only the diagonal maxima.

#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "simint/simint.h"
#include "simint_b200.h"
#include "runtime.h"

__global__ void k_diag_max(const double * __restrict__ ints, int n1, int n2, long long ntask,
                           long long stride, double * __restrict__ out)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= ntask)
        return;
    const double * v = ints + t * stride;
    double m = 0.0;
    for(int a = 0; a < n1; a++)
        for(int b = 0; b < n2; b++)
        {
            const long long idx = (long long)a * n2 * n1 * n2 + (long long)a * n2 + (long long)b * n1 * n2 + b;
            m = fmax(m, fabs(v[idx]));
        }
    out[t] = m;
}

namespace sb200 {

// max over the diagonal Cartesians of (ab|ab) for every shell pair k < n of
// a packed pair set, written to dmax[k] (device).  Runs the class kernel on
// the task list (k, k) in chunks of at most 512 MiB of (ab|ab) blocks.
int pair_diag_max(const PairSetDev & dP, int am1, int am2, int n, double * dmax, cudaStream_t stream)
{
    Workspace & w = workspace();
    const int n1 = ncart_of(am1), n2 = ncart_of(am2);
    const long long nc = (long long)n1 * n2 * n1 * n2;
    const long long chunk = std::max<long long>(1, std::min<long long>(n, (512ll << 20) / (nc * 8)));
    std::vector<int2> ht(chunk);
    if(!w.dkord.reserve((size_t)chunk * sizeof(int2)) || !w.dout.reserve((size_t)chunk * nc * sizeof(double)))
    {
        set_error("out of device memory in pair_diag_max");
        return SIMINT_B200_ERR_CUDA;
    }
    int2 * dtask = (int2 *)w.dkord.ptr;
    for(long long c0 = 0; c0 < n; c0 += chunk)
    {
        const long long cn = std::min<long long>(chunk, n - c0);
        cudaStreamSynchronize(stream);       // host task staging is reused
        for(long long k = 0; k < cn; k++)
            ht[k] = make_int2((int)(c0 + k), (int)(c0 + k));
        cudaMemcpyAsync(dtask, ht.data(), cn * sizeof(int2), cudaMemcpyHostToDevice, stream);
        KernArgs a;
        memset(&a, 0, sizeof(a));
        a.P = dP; a.Q = dP;
        a.tasks = dtask;
        a.ntask = cn;
        a.out = (double *)w.dout.ptr;
        a.nout = (int)nc;
        const int req[4] = {am1, am2, am1, am2};
        // the diagonal does not depend on the Cartesian ordering
        int rc = launch_class(a, req, 0, 1, SIMINT_B200_PREC_FP64, stream);
        if(rc != 0)
            return rc;
        k_diag_max<<<(unsigned)((cn + 127) / 128), 128, 0, stream>>>(
            (double *)w.dout.ptr, n1, n2, cn, nc, dmax + c0);
        count_launch(1);
    }
    cudaStreamSynchronize(stream);
    return 0;
}

int prim_schwarz_batch(int npair, const simint_shell * AB, double * out)
{
    init_tables();
    if(ensure_device() < 0)
        return SIMINT_B200_ERR_NODEVICE;
    // enumerate primitive pairs and their padded slots in the caller's layout
    std::vector<int> slot;
    std::vector<double> store;            // alpha, coef of every single-primitive shell
    std::vector<std::array<int, 4>> pp;   // (pair, i, j, same)
    int idx = 0;
    for(int s = 0; s < npair; s++)
    {
        const simint_shell * A = &AB[2 * s];
        const simint_shell * B = &AB[2 * s + 1];
        const int same = compare_shell(A, B);
        for(int i = 0; i < A->nprim; i++)
            for(int j = 0; j < (same ? i + 1 : B->nprim); j++)
            {
                pp.push_back({s, i, j, same});
                slot.push_back(idx++);
            }
        if(((s + 1) % SIMINT_NSHELL_SIMD) == 0 || s + 1 >= npair)
            idx = SIMINT_SIMD_ROUND(idx);
    }
    const int npad = idx;
    for(int k = 0; k < npad; k++)
        out[k] = 0.0;
    const int n = (int)pp.size();
    if(n == 0)
        return 0;
    // one single-primitive shell pair per primitive pair; distinct storage
    // so that no pair counts as a shell with itself (shell_screen.c:160-175)
    store.resize(4 * (size_t)n);
    std::vector<simint_shell> sh(2 * (size_t)n);
    for(int k = 0; k < n; k++)
    {
        const simint_shell * A = &AB[2 * pp[k][0]];
        const simint_shell * B = &AB[2 * pp[k][0] + 1];
        double * st = &store[4 * (size_t)k];
        st[0] = A->alpha[pp[k][1]]; st[1] = A->coef[pp[k][1]];
        st[2] = B->alpha[pp[k][2]]; st[3] = B->coef[pp[k][2]];
        simint_shell & a = sh[2 * (size_t)k];
        simint_shell & b = sh[2 * (size_t)k + 1];
        a = *A; b = *B;
        a.nprim = b.nprim = 1;
        a.alpha = st; a.coef = st + 1; a.ptr = st; a.memsize = 0;
        b.alpha = st + 2; b.coef = st + 3; b.ptr = st + 2; b.memsize = 0;
    }
    simint_multi_shellpair PP;
    simint_initialize_multi_shellpair(&PP);
    simint_create_multi_shellpair2(n, sh.data(), &PP, SIMINT_SCREEN_NONE);

    Workspace & w = workspace();
    if(!w.stream && cudaStreamCreateWithFlags(&w.stream, cudaStreamNonBlocking) != cudaSuccess)
    {
        simint_free_multi_shellpair(&PP);
        set_error("cudaStreamCreate failed");
        return SIMINT_B200_ERR_CUDA;
    }
    PackedLayout LP;
    const size_t szP = (pack_pairs(&PP, nullptr, LP) + 255) & ~(size_t)255;
    const size_t szM = ((size_t)n * sizeof(double) + 255) & ~(size_t)255;
    if(!w.hstage.reserve(szP) || !w.dpair.reserve(szP + szM))
    {
        simint_free_multi_shellpair(&PP);
        set_error("out of memory in Schwarz screening");
        return SIMINT_B200_ERR_CUDA;
    }
    char * h = (char *)w.hstage.ptr;
    char * d = (char *)w.dpair.ptr;
    pack_pairs(&PP, h, LP);
    cudaMemcpyAsync(d, h, szP, cudaMemcpyHostToDevice, w.stream);
    const PairSetDev dP = device_view(d, LP, PP.screen_max);
    double * dmax = (double *)(d + szP);
    int rc = pair_diag_max(dP, AB[0].am, AB[1].am, n, dmax, w.stream);
    std::vector<double> mx(n);
    if(rc == 0)
    {
        cudaMemcpyAsync(mx.data(), dmax, n * sizeof(double), cudaMemcpyDeviceToHost, w.stream);
        cudaError_t e = cudaStreamSynchronize(w.stream);
        if(e == cudaSuccess)
            e = cudaGetLastError();
        if(e != cudaSuccess)
        {
            set_error(std::string("CUDA error in Schwarz screening: ") + cudaGetErrorString(e));
            rc = SIMINT_B200_ERR_CUDA;
        }
    }
    simint_free_multi_shellpair(&PP);
    if(rc != 0)
        return rc;
    for(int k = 0; k < n; k++)
        out[slot[k]] = mx[k];
    return 0;
}

} // namespace sb200
