#pragma once
/* Build limits and host workspace sizes of the B200 Simint engine.
 *
 * SIMINT_OSTEI_MAXAM / MAXDER replace the CMake-substituted values of the
 * reference's skel/simint/ostei/ostei_config.h.in:5-7.
 *
 * simint_ostei_worksize / simint_ostei_workmem replace the functions that the
 * reference's create.py writes into that header (create.py:435-456).  The GPU
 * path needs no host workspace, but callers size their buffers with these
 * functions, so they return the reference's numbers.  The element counts
 * (batched contracted quartets, primitive VRR storage, HRR intermediates per
 * class, maximised over classes up to each AM) were computed by our own
 * recurrence planner (simint_b200/gen/plan.py, ClassPlan.reference_worksize),
 * which reproduces the reference generator's "WORK SIZE" log lines. */
#include <stddef.h>
#include "simint/vectorization/vectorization.h"

#define SIMINT_OSTEI_MAXAM 4
#define SIMINT_OSTEI_MAXDER 1
#define SIMINT_OSTEI_DERIV1_MAXAM (SIMINT_OSTEI_MAXDER > 0 ? 4 : -1)

#define SIMINT_B200_WS_(bcont, cont, prim) \
    (SIMINT_SIMD_ROUND(SIMINT_NSHELL_SIMD*(bcont)) + SIMINT_SIMD_ROUND(cont) + SIMINT_SIMD_LEN*(prim))

static inline size_t simint_ostei_worksize(int derorder, int maxam)
{
    static const size_t nelements[2][5] = {
        { SIMINT_B200_WS_(1, 0, 1),
          SIMINT_B200_WS_(81, 81, 149),
          SIMINT_B200_WS_(961, 4332, 2405),
          SIMINT_B200_WS_(5476, 57512, 17273),
          SIMINT_B200_WS_(21025, 418905, 79965) },
        { SIMINT_B200_WS_(10, 3, 8),
          SIMINT_B200_WS_(522, 1323, 495),
          SIMINT_B200_WS_(5386, 37116, 5801),
          SIMINT_B200_WS_(28520, 407144, 34759),
          SIMINT_B200_WS_(104550, 2694800, 142986) },
    };
    if(derorder < 0 || derorder > SIMINT_OSTEI_MAXDER || maxam < 0 || maxam > SIMINT_OSTEI_MAXAM)
        return 0;
    return nelements[derorder][maxam];
}

static inline size_t simint_ostei_workmem(int derorder, int maxam)
{
    return simint_ostei_worksize(derorder, maxam) * sizeof(double);
}
