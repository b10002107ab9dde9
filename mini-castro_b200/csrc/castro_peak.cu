// castro_peak.cu -- FP64 FMA throughput probe (roofline denominator).
//
// Every thread runs eight independent dependent chains of DFMA; the grid
// covers every SM several times over.  No reference counterpart.
#include <cuda_runtime.h>

#include "../../include/castro_b200.h"

namespace {

__global__ void k_dfma(double* out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) x[c] = threadIdx.x * 1e-9 + c;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < 8; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += x[c];
    if (s == 1.2345) out[0] = s;   // keeps the chains live
}

}  // namespace

extern "C" double castro_measure_fp64_tflops(void)
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0.0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    double* out = nullptr;
    if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return 0.0;
    const int threads = 256, blocks = sms * 8, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_dfma<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);   // warm-up
    double best = 0.0;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        k_dfma<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        double flops = 2.0 * 8.0 * iters * (double)threads * blocks;
        double tf = flops / (ms * 1e-3) / 1e12;
        if (tf > best) best = tf;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    return best;
}
