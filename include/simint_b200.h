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

/* FP64 everywhere, or FP32 VRR for primitive quartets whose Schwarz bound
 * sqrt(screen_ab * screen_cd) is below `gate` (FP64 Boys, prefactors,
 * contraction and HRR in both modes).  Applies to pairs built with Schwarz
 * screening; others always run in FP64.  Process-wide. */
int simint_b200_set_precision(int mode, double gate);
int simint_b200_get_precision(void);

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

/* Quartet and primitive-quartet counts of the sweep (after screening). */
long long simint_b200_basis_nquartets(simint_b200_basis const * b);
long long simint_b200_basis_nprimquartets(simint_b200_basis const * b);
/* Number of doubles the full output of the sweep occupies. */
long long simint_b200_basis_output_size(simint_b200_basis const * b);

/* Run the sweep on `stream` (cudaStream_t, may be NULL) writing all
 * integrals to device memory `dev_out` (simint_b200_basis_output_size
 * doubles), class after class, quartets in the order of
 * simint_b200_basis_tasks.  prec selects FP64 or mixed.  Returns the number
 * of kernel launches, or a negative error code. */
int simint_b200_basis_compute(simint_b200_basis * b, int prec, double * dev_out, void * stream);

#ifdef __cplusplus
}
#endif
