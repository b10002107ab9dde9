// castro_common.cuh -- host/device plumbing shared by the CUDA translation
// units: FAB views, box launches, error state, species dispatch.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "castro_device.cuh"

// NVTX ranges around the host routines (the counterpart of the reference's
// BL_PROFILE regions, e.g. Source/Castro_advance.cpp:28,
// Source/Castro_hydro.cpp:10); header-only NVTX v3, inert unless a profiler
// attaches.  -DCASTRO_NVTX=0 compiles them out.
#ifndef CASTRO_NVTX
#define CASTRO_NVTX 1
#endif
#if CASTRO_NVTX
#include <nvtx3/nvToolsExt.h>
#endif

namespace castro {

struct NvtxRange {
#if CASTRO_NVTX
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
#else
    explicit NvtxRange(const char*) {}
#endif
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// A FAB view in BL_FORT_FAB_ARG_3D form: Fortran order, component slowest.
struct Fab {
    double* p;
    int lx, ly, lz;
    int nx, ny, nz;
    __host__ __device__ __forceinline__ double& operator()(int i, int j, int k, int n) const
    {
        return p[(long long)(i - lx) + (long long)nx * ((long long)(j - ly) + (long long)ny * ((long long)(k - lz) + (long long)nz * n))];
    }
};

inline Fab make_fab(const double* p, const int* lo, const int* hi)
{
    Fab f;
    f.p = const_cast<double*>(p);
    f.lx = lo[0]; f.ly = lo[1]; f.lz = lo[2];
    f.nx = hi[0] - lo[0] + 1; f.ny = hi[1] - lo[1] + 1; f.nz = hi[2] - lo[2] + 1;
    return f;
}

struct BoxRange {
    int lx, ly, lz, nx, ny, nz;
    long long n;
};

inline BoxRange make_range(const int* lo, const int* hi)
{
    BoxRange r;
    r.lx = lo[0]; r.ly = lo[1]; r.lz = lo[2];
    r.nx = hi[0] - lo[0] + 1; r.ny = hi[1] - lo[1] + 1; r.nz = hi[2] - lo[2] + 1;
    if (r.nx <= 0 || r.ny <= 0 || r.nz <= 0) r.n = 0;
    else r.n = (long long)r.nx * r.ny * r.nz;
    return r;
}

template <class F>
__global__ void k_box(BoxRange r, F f)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= r.n) return;
    int i = r.lx + (int)(t % r.nx);
    long long t2 = t / r.nx;
    int j = r.ly + (int)(t2 % r.ny);
    int k = r.lz + (int)(t2 / r.ny);
    f(i, j, k);
}

// error state and stream, defined in castro_host.cu
void set_error(int code, const char* what);
cudaStream_t stream();
bool table_ready();
int nspec();

inline bool check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
        set_error(1, buf);
        return false;
    }
    return true;
}

template <int BLOCK = 128, class F>
inline void launch_box(const char* what, const int* lo, const int* hi, F f)
{
    BoxRange r = make_range(lo, hi);
    if (r.n == 0) return;
    long long nb = (r.n + BLOCK - 1) / BLOCK;
    k_box<<<(unsigned)nb, BLOCK, 0, stream()>>>(r, f);
    check_launch(what);
}

// run-time nspec -> template dispatch
#define CASTRO_DISPATCH_NS(FN, ...)                                            \
    do {                                                                       \
        if (!::castro::table_ready()) { ::castro::set_error(2, #FN ": eos_init has not run"); break; } \
        int ns_ = ::castro::nspec();                                           \
        if (ns_ == 2) FN<2>(__VA_ARGS__);                                      \
        else if (ns_ == 13) FN<13>(__VA_ARGS__);                               \
        else ::castro::set_error(4, #FN ": nspec must be 2 or 13");            \
    } while (0)

}  // namespace castro
