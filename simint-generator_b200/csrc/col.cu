// Host side of the column kernel (colkern.cuh): the registry of the
// generated classes, the shared-memory layout of a launch and the launch.
#include <algorithm>
#include <array>
#include <map>
#include <mutex>

#include "runtime.h"
#include "colkern.cuh"

namespace sb200 {

static std::once_flag g_col_once;
static ColTable g_col_table;
static std::map<std::array<int, 4>, int> g_col_index;

static const ColKernels * col_find(const int am[4])
{
    std::call_once(g_col_once, [] {
        simint_b200_register_col(g_col_table);
        for(size_t k = 0; k < g_col_table.list.size(); k++)
        {
            const ColKernels & c = g_col_table.list[k];
            g_col_index[{c.am[0], c.am[1], c.am[2], c.am[3]}] = (int)k;
        }
    });
    auto it = g_col_index.find({am[0], am[1], am[2], am[3]});
    return it == g_col_index.end() ? nullptr : &g_col_table.list[it->second];
}

bool col_is_variant(int v) { return v >= 81 && v <= 80 + COL_NNP; }

struct ColLayout
{
    int npi, nt, vdoubles, fs, phd;       // nt: threads per CTA; phd: shared doubles per group
    size_t smem;
};

// Shared memory of a launch, per group of threads: the recursion area V
// (the bra block of FS primitive quartets and the stage areas of a batch of
// NP; also the slot-sum and HRR scratch), the coefficient records of a
// block, the accumulators of the HRR and the two survivor lists.  FS is the
// largest of 32, 16, 8, 4 (a multiple of NP) for which the H groups fit.
static bool col_layout(const ColKernels & k, const C2Params & p, int v, ColLayout & L)
{
    L.npi = v - 81;
    if(L.npi < 0 || L.npi >= COL_NNP || !k.fn[L.npi][0][0])
        return false;
    const int np = COL_NPS[L.npi], h = COL_HS[L.npi];
    const int nth = k.nt[L.npi];
    L.nt = h * nth;
    const int acc = (p.acc_size + 1) & ~1;
    for(int fs = 32; fs >= np; fs /= 2)
    {
        int vd = std::max(k.f0b * col_pitch(fs) + k.sab * np, k.red_per_np * np);
        vd = std::max(vd, p.hrr_need);
        vd = (vd + 1) & ~1;
        // survivors: 2 nth ints = nth doubles
        const int phd = (vd + k.ncoef * fs + acc + nth + 1) & ~1;
        const size_t smem = (size_t)h * phd * sizeof(double);
        if(smem <= 220 * 1024)
        {
            L.fs = fs;
            L.vdoubles = vd;
            L.phd = phd;
            L.smem = smem;
            return true;
        }
    }
    return false;
}

bool col_supported(const int req[4], int deriv, int v)
{
    if(deriv != 0 || !col_is_variant(v))
        return false;
    const UniqueMap u = unique_of(req);
    const ColKernels * k = col_find(u.am);
    if(!k)
        return false;
    C2Params p;
    if(!coop2_hrr_params(u.am, p))
        return false;
    ColLayout L;
    return col_layout(*k, p, v, L);
}

int launch_col(KernArgs & a, const int req[4], int mode, int prec, cudaStream_t stream, int v)
{
    const UniqueMap u = unique_of(req);
    const ColKernels * k = col_find(u.am);
    C2Params p;
    ColLayout L;
    if(!k || !coop2_hrr_params(u.am, p) || !col_layout(*k, p, v, L))
    {
        set_error("class outside the column kernel's range");
        return SIMINT_B200_ERR_CLASS;
    }
    a.swapB = u.swapB; a.swapK = u.swapK; a.pq = u.pq;
    a.oidx = oidx_table(req, u, ordering());
    if(!a.oidx)
    {
        set_error("cannot allocate output index table");
        return SIMINT_B200_ERR_CUDA;
    }
    const bool mixed = prec == SIMINT_B200_PREC_MIXED && a.gate > 0.0;
    ColFn fn = k->fn[L.npi][mode][mixed ? 1 : 0];
    static std::mutex m;
    static std::map<std::pair<int, ColFn>, int> per_sm_cache;    // (device, kernel) -> CTAs per SM
    int dev = 0, nsm = 148, per_sm = 1;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(m);
        auto it = per_sm_cache.find({dev, fn});
        if(it == per_sm_cache.end())
        {
            cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
            if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, L.nt, L.smem) != cudaSuccess)
            {
                cudaGetLastError();
                per_sm = 1;
            }
            it = per_sm_cache.emplace(std::make_pair(dev, fn), std::max(per_sm, 1)).first;
        }
        per_sm = it->second;
    }
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // each CTA runs H shell quartets at a time
    const int h = COL_HS[L.npi];
    long long grid = std::min<long long>((a.ntask + h - 1) / h, (long long)nsm * per_sm);
    grid = std::max<long long>(grid, 1);
    fn<<<(unsigned)grid, L.nt, L.smem, stream>>>(a, p, L.vdoubles, L.fs, L.phd);
    count_launch(1);
    return 0;
}

} // namespace sb200
