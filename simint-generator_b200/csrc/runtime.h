// Internal declarations shared by the host runtime files.
#pragma once

#include <array>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "simint/simint.h"
#include "ostei_device.cuh"
#include "kernels.h"

namespace sb200 {

struct UniqueMap
{
    int am[4];
    int swapB, swapK, pq;
};

struct DevBuf
{
    void * ptr = nullptr;
    size_t cap = 0;
    bool reserve(size_t n);
    void release();
};

struct HostBuf
{
    void * ptr = nullptr;
    size_t cap = 0;
    bool reserve(size_t n);
    void release();
};

struct Workspace
{
    cudaStream_t stream = nullptr;
    cudaStream_t dstream = nullptr;       // downloads of pipelined calls
    DevBuf dpair, dout, dkord, dscratch;
    DevBuf dsoa;                          // pair arrays copied from page-locked host memory
    HostBuf hstage, hout;
    ~Workspace();
};

struct PackedLayout
{
    int npad = 0, npair = 0;
    size_t off_rec = 0, off_start = 0, off_nprim = 0, off_AB = 0;
};

void set_error(const std::string & s);
void count_launch(long long n);
int ensure_device();
const double * boys_table();
void init_tables();
int ordering();
int precision();
double gate();
Workspace & workspace();
// Launches issued by this host thread use `w` (nullptr: the thread's own
// workspace) for their scratch: concurrent streams of one sweep each get one.
void set_workspace_override(Workspace * w);
UniqueMap unique_of(const int am[4]);
const ClassKernels * find_kernels(const UniqueMap & u);
int cart_index(int i, int j, int k, int ordering);
void carts(int l, std::vector<std::array<int, 3>> & out);
void pair_starts(const simint_multi_shellpair * P, std::vector<int> & start, int & npad);
size_t pack_pairs(const simint_multi_shellpair * P, char * dst, PackedLayout & L);
PairSetDev device_view(const char * base, const PackedLayout & L, double screen_max);
const unsigned short * oidx_table(const int req[4], const UniqueMap & u, int ord);

// The P x Q rectangle (nqc < 0), or its part P x (kets dkord[0..nqc)) with
// the rectangle's output layout.
int launch_rectangle(const simint_multi_shellpair * P, const PairSetDev & dP,
                     const simint_multi_shellpair * Q, const PairSetDev & dQ,
                     const int * dkord, double screen_tol, int deriv, int prec, double gatev,
                     double * dout, cudaStream_t stream, int nqc = -1);
void pack_records(const simint_multi_shellpair * P, int npad, int g0, int g1, double * rec);

int launch_class(KernArgs & a, const int req[4], int deriv, int mode, int prec,
                 cudaStream_t stream);
bool class_uses_queue(const int req[4], int deriv, int prec);
// Whether P's arrays live in page-locked host memory (large pair sets made
// by simint_create_multi_shellpair; shell.cpp).
bool pair_data_pinned(const simint_multi_shellpair * P);
void permute_multi_shellpair(const simint_multi_shellpair * src, const int * order, simint_multi_shellpair * dst);
void ssss_clip_vector(const simint_multi_shellpair * P, const simint_multi_shellpair * Q, int & v0, int & v1);

// Generic (table-driven, dense) kernel for classes without a straight-line
// kernel and for deriv=1.  Everything in a except the role swaps is filled.
int launch_generic(KernArgs & a, const int req[4], const UniqueMap & u, int deriv, int mode,
                   cudaStream_t stream);

int ncart_of(int l);
bool coop_supported(const int am[4], int deriv);
// Cooperative kernel v2; v = 0 for the default plan or a variant code
// (20 + B: 256 threads, 40 + B: 128 threads, 60 + B: 64 threads; B = 1, 2, 4).
bool coop2_supported(const int am[4], int deriv, int v = 0);
bool coop2_is_variant(int v);
int launch_coop2(KernArgs & a, const int req[4], int deriv, int mode, int prec, cudaStream_t stream,
                 int v = 0);
// Column kernel (colkern.cuh), deriv 0: variant codes 81 (4 primitive
// quartets per batch), 82 (8) and 83 (4, two groups of threads per CTA
// running separate shell quartets).
bool col_is_variant(int v);
bool col_supported(const int req[4], int deriv, int v);
int launch_col(KernArgs & a, const int req[4], int mode, int prec, cudaStream_t stream, int v);

// Kernel variant per (requested class, deriv, precision), chosen by the
// autotuner: 0 default rule, 1 straight-line, 3 cooperative v1, 4 generic,
// 5 straight-line in FP64 even in mixed mode, 6 (7) straight-line with a
// warp per shell quartet (in FP64 even in mixed mode), 20+B / 40+B / 60+B
// cooperative v2 with batch B and 256 / 128 / 64 threads, 81 / 82 / 83
// column kernel (4 / 8 primitive quartets per batch, 83: two groups per
// CTA); 100 + a cooperative or column code: that kernel in FP64 even in
// mixed mode.
enum { VAR_DEFAULT = 0, VAR_STRAIGHT = 1, VAR_COOP2 = 2, VAR_COOP1 = 3, VAR_GENERIC = 4, VAR_STRAIGHT64 = 5,
       VAR_WARP = 6, VAR_WARP64 = 7 };
int variant_of(const int req[4], int deriv, int prec);
void set_variant(const int req[4], int deriv, int prec, int v);
// Incremented whenever a setting that captured sweep graphs bake in changes
// (kernel variant, ordering, precision gate); graphs older than it are rebuilt.
long long settings_epoch();
void bump_settings_epoch();
bool has_straight(const int req[4]);
bool has_warp(const int req[4], int mode);
void save_tune_file();
int launch_coop(KernArgs & a, const int req[4], int deriv, int mode, cudaStream_t stream);
int pair_diag_max(const PairSetDev & dP, int am1, int am2, int n, double * dmax, cudaStream_t stream);

} // namespace sb200
