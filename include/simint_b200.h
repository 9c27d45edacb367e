#pragma once
/* Extensions of the B200 Simint engine beyond the reference's C API.
 *
 * None of these exist in the reference (skel/simint/ has no GPU code); they
 * are the non-breaking additions its drop-in replacement needs: choosing the
 * Cartesian ordering and arithmetic mode at run time, reading errors, and the
 * batched, device-resident sweep that the reference's callers (tests,
 * benchmark, QC codes) otherwise express as many simint_compute_eri calls
 * (skel/test/benchmark_eri.cpp:135-216). */
#include <stddef.h>
#include <stdint.h>
#include "simint/simint.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes returned (negative) by simint_compute_eri and the functions
 * below.  -1 keeps its reference meaning: everything was screened. */
#define SIMINT_B200_SCREENED      -1
#define SIMINT_B200_ERR_NODEVICE  -2   /* no CUDA device / driver */
#define SIMINT_B200_ERR_CLASS     -3   /* AM class or derivative not supported */
#define SIMINT_B200_ERR_CUDA      -4   /* a CUDA call failed (see last_error) */
#define SIMINT_B200_ERR_ARG       -5   /* bad argument */
#define SIMINT_B200_ERR_TIMEOUT   -6   /* a bounded device wait ran out */

#define SIMINT_B200_ORDERING_PSI4   0
#define SIMINT_B200_ORDERING_GAMESS 1

#define SIMINT_B200_PREC_FP64  0
#define SIMINT_B200_PREC_MIXED 1

/* Cartesian ordering of the output (reference: compile-time SIMINT_ORDERING,
 * generator/CMakeLists.txt:9-10; default Psi4).  Process-wide. */
int simint_b200_set_ordering(int ordering);
int simint_b200_get_ordering(void);

/* FP64 everywhere, or FP32 VRR for primitive quartets whose estimated FP32
 * error keeps every integral within `gate` (FP64 Boys, prefactors,
 * contraction and HRR in both modes).  The estimate of one primitive quartet
 * of a class with recursion depth L = la+lb+lc+ld is
 *     8 (L+1) 2^-24 |prefac| r^L (1 + |AB|)^min(la,lb) (1 + |CD|)^min(lc,ld),
 *     r = (g + sqrt(g^2 + 4h)) / 2,  g = 1 + max|X| + max|Y|,
 *     h = L (1/2p + 1/2q + 1/2(p+q))
 * (X: P-A, P-B, Q-C, Q-D components; Y: the rho/p, rho/q (P-Q) terms), a
 * bound on the absolute error its FP32 VRR adds to any integral of the
 * shell quartet.  An integral's error is at most the sum over its primitive
 * quartets, so a primitive quartet runs in FP32 only when its estimate is
 * below gate / (the shell quartet's primitive quartets): the gate bounds
 * the error of each integral.  Classes with L = 0 stay in FP64 (no VRR).
 * gate = 0 keeps FP64.  Process-wide. */
int simint_b200_set_precision(int mode, double gate);
int simint_b200_get_precision(void);

/* Pair data placement: simint_create_multi_shellpair(2) and
 * simint_cat_multi_shellpair allocate pair sets of 256 KB or more in
 * page-locked host memory when a CUDA device is present (environment
 * variable SIMINT_B200_PIN_PAIRS=0: never); simint_free_multi_shellpair
 * frees them.  simint_compute_eri(_deriv) copies such a set to the device
 * with one DMA of its allocation and builds the device records there;
 * arrays a caller pointed outside the allocation are packed on the host. */

/* Where simint_fill_multi_shellpair(2) and simint_create_multi_shellpair(2)
 * (shell.h:193-236, shell.c:425-582) compute the Gaussian-product fill.
 * SIMINT_B200_PAIR_FILL_AUTO (default): on the GPU for lists of 4096 or
 * more padded primitive pairs when a device is present, else on the host;
 * _HOST: always on the host (bit for bit the reference's shell.c);
 * _GPU: on the GPU whenever a device is present.  The GPU fill is one
 * thread per shell pair writing a device image of the allocation (one copy
 * back), the Schwarz values of all primitive pairs as one task list and the
 * reference's per-pair sort on the device: every array equals the host fill
 * bit for bit except the prefactors and screening values, which may differ
 * in the last bits (CUDA's exp against the host's).  A failed GPU fill
 * prints a message and fills on the host.  The environment variable
 * SIMINT_B200_PAIR_FILL=host|gpu sets the initial mode.  Process-wide;
 * returns 0 or SIMINT_B200_ERR_ARG. */
#define SIMINT_B200_PAIR_FILL_AUTO 0
#define SIMINT_B200_PAIR_FILL_HOST 1
#define SIMINT_B200_PAIR_FILL_GPU  2
int simint_b200_set_pair_fill(int mode);
int simint_b200_get_pair_fill(void);

/* Text of the last error seen by the calling thread. */
const char * simint_b200_last_error(void);

/* Number of kernels this library launched so far in the calling thread. */
long long simint_b200_launch_count(void);

/* ---------------------------------------------------------------------
 * Batched, device-resident sweeps.
 *
 * A basis is uploaded once; the caller then asks for every shell quartet of
 * the basis that survives shell-pair Schwarz screening (|(ab|cd)| bound
 * Q_ab*Q_cd >= tol), grouped by AM class.  Inputs, pair data and outputs
 * stay in device memory; the whole sweep is one CUDA graph.
 * ------------------------------------------------------------------- */
typedef struct simint_b200_basis simint_b200_basis;

/* Build pair data for all shell pairs (i >= j) of `shells` on the device,
 * with primitive Schwarz values, and the per-class quartet task lists for
 * screen_tol.  Returns NULL on error. */
simint_b200_basis * simint_b200_basis_create(int nshell, struct simint_shell const * shells,
                                             double screen_tol, int max_am);
void simint_b200_basis_free(simint_b200_basis * b);

/* Keep a deterministic stratified subsample of every class: bra-pair rows
 * are taken with a constant stride chosen so a class keeps about
 * max_quartets quartets (classes already smaller keep everything).  Used to
 * bound benchmark steps on very large sweeps; the full-sweep quartet counts
 * stay available through simint_b200_basis_class_full. */
int simint_b200_basis_subsample(simint_b200_basis * b, long long max_quartets);

/* Quartets of class k before subsampling. */
long long simint_b200_basis_class_full(simint_b200_basis const * b, int k);

/* Count the primitive quartets that survive primitive screening in the
 * current task lists (one device pass); returns the total. */
long long simint_b200_basis_count_primq(simint_b200_basis * b);

/* Quartet and primitive-quartet counts of the sweep (after screening). */
long long simint_b200_basis_nquartets(simint_b200_basis const * b);
long long simint_b200_basis_nprimquartets(simint_b200_basis const * b);
/* Number of doubles the full output of the sweep occupies. */
long long simint_b200_basis_output_size(simint_b200_basis const * b);

/* Run the sweep on `stream` (cudaStream_t, may be NULL).  Integrals are
 * written to device memory dev_out of dev_out_doubles doubles.  When that
 * holds the whole sweep (simint_b200_basis_output_size), class k starts at
 * its class offset and quartet q of the class at offset + q*nout; otherwise
 * the sweep is streamed through dev_out in chunks (each chunk overwrites the
 * previous one).  Either way per-class checksums are accumulated (see
 * simint_b200_basis_checksums).  prec selects FP64 or mixed.  The launches
 * are captured once into a CUDA graph per (prec, buffer) and replayed.
 * Returns the number of kernel launches of one sweep, or a negative code. */
int simint_b200_basis_compute(simint_b200_basis * b, int prec, double * dev_out,
                              long long dev_out_doubles, void * stream);

/* Number of AM classes in the sweep and their description: requested class
 * am[4], quartets, evaluated primitive quartets (after the reference's
 * primitive screening), doubles per quartet, offset of the class in a full
 * output buffer. */
int simint_b200_basis_nclass(simint_b200_basis const * b);
int simint_b200_basis_class_info(simint_b200_basis const * b, int k, int am[4],
                                 long long * nquart, long long * nprimq,
                                 int * nout, long long * offset);

/* The (bra pair, ket pair) shells of quartet q of class k:
 * shells[0..3] = indices into the shell array given to basis_create. */
int simint_b200_basis_quartet(simint_b200_basis const * b, int k, long long q, int shells[4]);

/* The same for every quartet of class k at once: shells[4q .. 4q+3] for
 * q < the class's quartet count (host array of 4 ints per quartet). */
int simint_b200_basis_class_quartets(simint_b200_basis const * b, int k, int * shells);

/* The ket pair list of class k in the order the sweep stores it (decreasing
 * Schwarz bound Q_cd): shells[2i], shells[2i+1] of pair i when shells is
 * not NULL.  Every row of the class takes a prefix of this list (a row is
 * simint_compute_eri(bra pair, this list with nshell12_clip = the row's ket
 * count)).  Returns the number of pairs or a negative code. */
int simint_b200_basis_class_kets(simint_b200_basis const * b, int k, int * shells);

/* Per-class checksums of the last compute: sums[2k] = sum of values,
 * sums[2k+1] = sum of absolute values.  Waits for the device.  Returns
 * SIMINT_B200_ERR_TIMEOUT when a bounded work-queue wait of the sweep ran
 * out (see simint_b200_basis_queue_probe). */
int simint_b200_basis_checksums(simint_b200_basis * b, double * sums);

/* Primitive quartets of the last compute that ran their VRR in FP32 (mixed
 * precision), per class: counts[k] for every class k (host array of
 * simint_b200_basis_nclass entries), counted by every kernel with an FP32
 * path (register, cooperative and column kernels).  Waits for the
 * device. */
int simint_b200_basis_fp32_counts(simint_b200_basis * b, long long * counts);

/* Work queue.  The cooperative and column kernels of a sweep take their
 * shell quartets from a device work queue, one atomic pull per CTA, in
 * order of decreasing primitive count (the longest quartets first, the
 * short ones fill the tail).  A CTA that finds no published task waits --
 * bounded, about one microsecond per poll -- until more are published or
 * the queue is closed; a wait that runs out marks the queue and the CTA
 * returns, so the launch always ends.  In a sweep every task is published
 * before the launch.
 *
 * simint_b200_basis_queue_probe runs class k (FP64, its current kernel,
 * which must be a queue kernel) with a queue whose first `published` tasks
 * are available and which is closed (closed != 0) or left open, each wait
 * limited to about wait_ms milliseconds, writing to dev_out (at least the
 * class's quartets x nout doubles; quartet q at q*nout).  Returns
 * `published` when every CTA finished normally, SIMINT_B200_ERR_TIMEOUT when
 * a wait ran out (an open queue), or another negative code.  The device
 * stays usable after a timeout. */
int simint_b200_basis_queue_probe(simint_b200_basis * b, int k, long long published, int closed,
                                  int wait_ms, double * dev_out, long long dev_out_doubles);

/* Autotuner: for every class of the sweep time each kernel variant (the
 * register kernel where one exists, thread- and warp-per-quartet; the
 * cooperative kernel with 256, 128 or 64 threads and 1, 2, 4 or 8
 * primitive quartets per wavefront pass; the column kernel with 4 or 8
 * primitive quartets per batch, or 4 in two thread groups per CTA; in mixed mode each also in FP64) on the
 * sweep's own tasks and keep the fastest for `prec`: one untimed run, then the best of two timed
 * runs, except for a candidate whose untimed run took over twice the best time so far plus a
 * millisecond.  Choices are process-wide and are written to the
 * JSON file $SIMINT_B200_TUNE_FILE when set (read back by simint_init). */
int simint_b200_basis_autotune(simint_b200_basis * b, int prec, double * dev_out,
                               long long dev_out_doubles, void * stream);

/* The kernel variant chosen for a requested class (0 = untuned default: the
 * register kernel while its contracted results fit registers, else the
 * cooperative kernel;
 * 1 = register kernel, 20+B / 40+B / 60+B = cooperative kernel with 256 /
 * 128 / 64 threads and batch B = 1, 2, 4, 8, 81 / 82 = column kernel with
 * 4 / 8 primitive quartets per batch, 83 = column kernel with 4 per batch
 * and two thread groups per CTA each running its own shell quartets,
 * deriv 0). */
int simint_b200_variant(const int am[4], int deriv, int prec);

/* Pin the kernel variant of a requested class (same codes, plus 3 = first
 * cooperative kernel, 4 = generic kernel, 5 = register kernel run in FP64
 * even in mixed mode, 6 = register kernel with one warp per shell quartet,
 * 7 = the same in FP64 even in mixed mode, and 100 + a cooperative or
 * column code = that kernel in FP64 even in mixed mode (prec must be
 * SIMINT_B200_PREC_MIXED); 0 restores the default rule).
 * Returns SIMINT_B200_ERR_ARG when the variant does not exist for the class.
 * Sweep graphs captured earlier are rebuilt on their next use. */
int simint_b200_set_variant(const int am[4], int deriv, int prec, int variant);

/* Device time of each class in one (non-graph) sweep, milliseconds. */
int simint_b200_basis_class_times(simint_b200_basis * b, int prec, double * dev_out,
                                  long long dev_out_doubles, void * stream, float * ms);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Keep bra-pair rows offset, offset+stride, ... of every class (a
 * proportional stratified subsample: the class mix of the full sweep is
 * preserved; disjoint offsets give disjoint shards). */
int simint_b200_basis_subsample_stride(simint_b200_basis * b, int stride, int offset);

/* Rows of class k (one bra pair each) and the task range of row r. */
int simint_b200_basis_nrows(simint_b200_basis const * b, int k);
int simint_b200_basis_row(simint_b200_basis const * b, int k, int r, long long * first, long long * n);

/* Primitive quartets simint_compute_eri(P, Q, screen_tol) evaluates: the
 * reference's bra-primitive and 8-wide ket-vector screening applied to the
 * host pair data (no device work). */
long long simint_b200_count_primq(struct simint_multi_shellpair const * P,
                                  struct simint_multi_shellpair const * Q, double screen_tol);

/* Measured FMA throughput of the current device in TFLOP/s: FP64 (fp32 = 0)
 * or FP32 (fp32 = 1).  Used as the roofline denominator. */
double simint_b200_fma_peak(int fp32);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------------
 * ERIs without any allocation (no counterpart in the reference).
 *
 * For callers that may not allocate device memory -- code inside a
 * framework that owns the device memory pool and only hands out buffers,
 * code that runs while such a pool is captured or frozen, or hot paths that
 * must never trigger the implicit synchronisation of cudaMalloc/cudaFree.
 *
 * simint_b200_packed_size / simint_b200_pack write the packed pair layout
 * of P into caller memory (host); the caller copies it to a device buffer it
 * owns.  simint_b200_compute_eri_noalloc then computes the same integrals
 * as simint_compute_eri_deriv(deriv, P, Q, ...) into the caller's device
 * buffer dev_integrals, on `stream` (cudaStream_t; NULL = legacy stream),
 * asynchronously, in FP64 whatever simint_b200_set_precision says.  It runs
 * the first cooperative kernel (classes whose shared-memory plan exceeds
 * 200 KB -- the largest g classes -- return SIMINT_B200_ERR_CLASS); its
 * working memory is a
 * file-scope static device array of simint_b200_noalloc_scratch_bytes()
 * (32 MiB) that every GPU which loads the library holds until exit, plus
 * static Boys tables and an identity ket order (at most 2^20 ket pairs).
 * It calls no cudaMalloc, cudaFree or other allocating routine.
 *
 * The first call on a device performs that device's set-up (resolves the
 * static arrays with cudaGetSymbolAddress, uploads tables, synchronises the
 * device), so make it before any stream capture.  All calls share the one
 * scratch array, which keeps the last call's contents: calls that overlap
 * on the GPU (different streams, threads or graphs) race and must be
 * serialised by the caller.  Returns nshell12_clip(P)*nshell12_clip(Q),
 * -1 when the pair-level test screens everything (nothing written), or a
 * negative SIMINT_B200_ERR_* code: ERR_ARG also when one CTA's scratch
 * would exceed the static array or Q has more than 2^20 pairs. */
size_t simint_b200_packed_size(struct simint_multi_shellpair const * P);
int simint_b200_pack(struct simint_multi_shellpair const * P, void * host_dst, size_t capacity);
long long simint_b200_noalloc_scratch_bytes(void);
int simint_b200_compute_eri_noalloc(int deriv,
                                    struct simint_multi_shellpair const * P, const void * dev_P,
                                    struct simint_multi_shellpair const * Q, const void * dev_Q,
                                    double screen_tol, double * dev_integrals, void * stream);

/* Device-resident form of simint_compute_eri_deriv (no reference
 * counterpart; its host form is simint_compute_eri_deriv,
 * skel/simint/ostei/ostei.c:10-41): dev_P and dev_Q hold the packed pair
 * layout of simint_b200_pack in device memory, dev_integrals receives the
 * same values simint_compute_eri_deriv(deriv, P, Q, ...) returns, on
 * `stream`, asynchronously, with the kernel variant, precision and ordering
 * in force.  Kets are processed in the order of Q.  Working memory is the
 * calling host thread's (allocated on first need, growth synchronises the
 * device): calls of one host thread must stay on one stream.  Returns the
 * shell-quartet count, -1 when the pair-level test screens everything, or a
 * negative SIMINT_B200_ERR_*. */
int simint_b200_compute_eri_device(int deriv,
                                   struct simint_multi_shellpair const * P, const void * dev_P,
                                   struct simint_multi_shellpair const * Q, const void * dev_Q,
                                   double screen_tol, double * dev_integrals, void * stream);

/* Fock-matrix digestion of a sweep (no counterpart in the reference, whose
 * callers -- Psi4, GTFock -- contract the integrals themselves): from the
 * full-layout output of simint_b200_basis_compute (dev_out of at least
 * simint_b200_basis_output_size doubles, every shell of the basis at most
 * the sweep's max_am), the Coulomb and exchange matrices
 *     J_pq = sum_rs (pq|rs) D_rs,   K_pq = sum_rs (pr|qs) D_rs
 * of a symmetric density D, all nbf x nbf row-major in device memory, basis
 * functions shell by shell in the order given to simint_b200_basis_create
 * and in the current Cartesian ordering inside a shell.  Quartets the sweep
 * screened out contribute nothing.  Classes whose integrals and six density
 * sub-blocks fit 227 KB of shared memory (about 28 000 integrals per shell
 * quartet: up to (gg|gd), (gf|gf), (gg|ff)); larger ones ((gg|gf), (gg|gg))
 * return SIMINT_B200_ERR_CLASS.
 * Asynchronous on `stream`; returns the number of kernel launches or a
 * negative SIMINT_B200_ERR_*. */
int simint_b200_basis_nbf(simint_b200_basis const * b);
int simint_b200_basis_jk(simint_b200_basis * b, const double * dev_out, long long dev_out_doubles,
                         const double * dev_D, double * dev_J, double * dev_K, void * stream);

/* The sweep and its J/K digestion in one pass, without the sweep's output
 * in HBM: the classes run on four streams at once (as a full-layout sweep
 * runs them), each stream streaming its classes in chunks through its
 * quarter of dev_scratch, and each chunk is contracted into J and K (as
 * simint_b200_basis_jk) right after it is computed, on the same stream,
 * while its integrals are still in the 126 MB L2 (a scratch buffer of a few
 * tens of MB keeps them there).  A scratch buffer whose quarter cannot hold
 * one quartet of every class is used by one stream; one that holds the
 * whole sweep is used as its full layout.  prec as for
 * simint_b200_basis_compute; the class checksums are accumulated as by a
 * streamed compute.  dev_scratch must hold one quartet of every class;
 * classes whose digestion does not fit shared memory return
 * SIMINT_B200_ERR_CLASS.  Issued eagerly on `stream`; returns the number of
 * kernel launches or a negative SIMINT_B200_ERR_*. */
int simint_b200_basis_compute_jk(simint_b200_basis * b, int prec, const double * dev_D, double * dev_J,
                                 double * dev_K, double * dev_scratch, long long scratch_doubles,
                                 void * stream);

/* One-electron matrices of a whole basis (the batched form of
 * simint_compute_overlap / simint_compute_ke / simint_compute_potential,
 * skel/simint/simint_oneelectron.h:12-27): kind SIMINT_B200_OEI_OVERLAP,
 * _KINETIC or _POTENTIAL (-sum_C Z_C 1/|r - C| over the ncenter point
 * charges Z, x, y, z, host arrays).  Writes the full symmetric nbf x nbf
 * matrix, row-major, into dev_out (device memory): basis functions shell by
 * shell in the given order, Cartesians inside a shell in the current ERI
 * ordering (simint_b200_set_ordering), so the matrix pairs with the
 * sweep's J and K.  Every shell at most am 4.  Asynchronous on `stream`
 * (the shells and centres are copied before the call returns); returns the
 * number of kernel launches or a negative SIMINT_B200_ERR_*. */
#define SIMINT_B200_OEI_OVERLAP   0
#define SIMINT_B200_OEI_KINETIC   1
#define SIMINT_B200_OEI_POTENTIAL 2
int simint_b200_oei_matrix(int kind, int nshell, struct simint_shell const * shells,
                           int ncenter, const double * Z, const double * x, const double * y,
                           const double * z, double * dev_out, void * stream);

#ifdef __cplusplus
}
#endif
