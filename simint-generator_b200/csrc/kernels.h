// Registry of the generated per-class kernels.
#pragma once
#include <vector>
#include "ostei_device.cuh"

typedef void (*KernFn)(const KernArgs);

struct ClassKernels
{
    int am[4];           // unique class (a b | c d)
    int L;               // a+b+c+d
    int ntop;            // contracted top quartets
    int vrr_flops;       // per primitive quartet (minimal plan)
    int hrr_flops;       // per shell quartet
    KernFn fn[3][2];     // [mode: 0 rectangle, 1 task list, 2 screened sweep][prec: 0 FP64, 1 mixed]
    KernFn fnw[3][2];    // warp per shell quartet (modes 0 and 2)
};

struct KernelTable
{
    std::vector<ClassKernels> list;
    void add(const ClassKernels & k) { list.push_back(k); }
};

void simint_b200_register_generated(KernelTable & t);
