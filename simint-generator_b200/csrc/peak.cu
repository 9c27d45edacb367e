// FP64 / FP32 FMA throughput probe (the roofline denominators).
//
// Each thread runs 8 independent FMA chains for `iters` iterations; the
// result is written so nothing is optimised away.  Timed with CUDA events.
#include <cuda_runtime.h>
#include "simint_b200.h"

template<typename T>
__global__ void k_fma_chain(T * out, int iters, T a, T b)
{
    T x[8];
    for(int k = 0; k < 8; k++)
        x[k] = (T)(threadIdx.x + k);
    for(int i = 0; i < iters; i++)
    {
        #pragma unroll
        for(int k = 0; k < 8; k++)
            x[k] = fma(x[k], a, b);
    }
    T s = 0;
    for(int k = 0; k < 8; k++)
        s += x[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// Returns the measured FMA rate in TFLOP/s (2 flops per FMA) for FP64
// (fp32 = 0) or FP32 (fp32 = 1), or a negative error code.
extern "C" double simint_b200_fma_peak(int fp32)
{
    int dev = 0, nsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256, blocks = nsm * 8, iters = 1 << 14;
    void * out = nullptr;
    if(cudaMalloc(&out, (size_t)threads * blocks * 8) != cudaSuccess)
        return SIMINT_B200_ERR_CUDA;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for(int rep = 0; rep < 5; rep++)
    {
        cudaEventRecord(e0);
        if(fp32)
            k_fma_chain<float><<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
        else
            k_fma_chain<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if(rep > 0 && ms < best)
            best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
    return flops / (best * 1e-3) / 1e12;
}
