// castro_adjoint.cu -- the reverse (adjoint) step of the CTU hydro advance.
//
// Two layers:
//  * <routine>_adj entry points: the adjoint of each Source/Castro_F.H routine
//    over [lo,hi], same FAB conventions as the forward entry point, adjoints of
//    the routine's inputs ACCUMULATED into caller arrays (x_b += J^T y_b);
//  * castro_adj_*: a checkpointed reverse sweep of a whole Sedov run on one
//    GPU.  Forward: initdata, then per step computeNewDt + Castro::advance +
//    post_timestep exactly as the plain path.  Reverse: for each checkpoint
//    segment (from the last), the segment's states are recomputed from its
//    checkpoint, then each step is recomputed with every intermediate kept and
//    reversed stage by stage; the time step's dependence on the state (the CFL
//    reduction at its arg-min zone, the 1.1x growth limit and the stop-time
//    clamp) is reversed as well.  Finally the initial data are reversed to the
//    gradient with respect to the blast energy, the ambient density and the
//    per-zone density perturbation field.
//
// Scatter-adds into shared adjoint arrays use FP64 atomics, so the last bits
// of a gradient may differ from run to run.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "castro_adjoint.cuh"
#include "castro_common.cuh"
#include "../../include/castro_b200.h"

using namespace castro;

namespace castro {
void upload_constants_adj(const EosTableDev& e, const NetworkDev& n)
{
    cudaMemcpyToSymbol(c_eos, &e, sizeof e);
    cudaMemcpyToSymbol(c_net, &n, sizeof n);
}
const castro_problem& problem();
const NetworkDev& network_host();
}  // namespace castro

namespace {

constexpr int NG = 4;

struct SpeciesXAdj { double x[MAX_SPEC]; };

// ---- device helpers ----------------------------------------------------------
__device__ __forceinline__ void aadd(double* p, double v)
{
    if (v != 0.0) atomicAdd(p, v);
}

// stencil sink of the trace / flatten adjoints: atomic adds into FABs
struct AtomicSink {
    Fab qb, qab;
    CASTRO_HD void q(int i, int j, int k, int n, double v) const
    {
#ifdef __CUDA_ARCH__
        aadd(&qb(i, j, k, n), v);
#else
        qb(i, j, k, n) += v;
#endif
    }
    CASTRO_HD void gamc(int i, int j, int k, double v) const
    {
#ifdef __CUDA_ARCH__
        aadd(&qab(i, j, k, QGAMC), v);
#else
        qab(i, j, k, QGAMC) += v;
#endif
    }
    CASTRO_HD void c(int i, int j, int k, double v) const
    {
#ifdef __CUDA_ARCH__
        aadd(&qab(i, j, k, QC), v);
#else
        qab(i, j, k, QC) += v;
#endif
    }
};

struct QLoad {
    Fab qf, qaf;
    CASTRO_HD double q(int i, int j, int k, int n) const { return qf(i, j, k, n); }
    CASTRO_HD double gamc(int i, int j, int k) const { return qaf(i, j, k, QGAMC); }
    CASTRO_HD double c(int i, int j, int k) const { return qaf(i, j, k, QC); }
};

// compact face state <-> full QVAR record (QGAME/QTEMP have no adjoint)
template <int NS>
__device__ __forceinline__ void ld_state(const Fab& f, int i, int j, int k, double* s)
{
    s[SRHO] = f(i, j, k, QRHO);
    s[SU] = f(i, j, k, QU);
    s[SV] = f(i, j, k, QV);
    s[SW] = f(i, j, k, QW);
    s[SPRES] = f(i, j, k, QPRES);
    s[SREI] = f(i, j, k, QREINT);
#pragma unroll
    for (int n = 0; n < NS; ++n) s[SX + n] = f(i, j, k, QFS + n);
}

template <int NS>
__device__ __forceinline__ void add_state(const Fab& f, int i, int j, int k, const double* s)
{
    f(i, j, k, QRHO) += s[SRHO];
    f(i, j, k, QU) += s[SU];
    f(i, j, k, QV) += s[SV];
    f(i, j, k, QW) += s[SW];
    f(i, j, k, QPRES) += s[SPRES];
    f(i, j, k, QREINT) += s[SREI];
#pragma unroll
    for (int n = 0; n < NS; ++n) f(i, j, k, QFS + n) += s[SX + n];
}

template <int NS>
__device__ __forceinline__ void ld_tflux(const Fab& f, const Fab& qg, int i, int j, int k, int normal, double* r)
{
    using R = TF<NS>;
    r[R::RHO] = f(i, j, k, URHO);
    r[R::MX] = f(i, j, k, UMX);
    r[R::MY] = f(i, j, k, UMY);
    r[R::MZ] = f(i, j, k, UMZ);
    r[R::ED] = f(i, j, k, UEDEN);
#pragma unroll
    for (int n = 0; n < NS; ++n) r[R::X + n] = f(i, j, k, UFS + n);
    r[R::PG] = qg(i, j, k, GDPRES);
    r[R::UG] = qg(i, j, k, GDU + normal);
}

template <int NS>
__device__ __forceinline__ void aadd_tflux(const Fab& f, const Fab& qg, int i, int j, int k, int normal, const double* r)
{
    using R = TF<NS>;
    aadd(&f(i, j, k, URHO), r[R::RHO]);
    aadd(&f(i, j, k, UMX), r[R::MX]);
    aadd(&f(i, j, k, UMY), r[R::MY]);
    aadd(&f(i, j, k, UMZ), r[R::MZ]);
    aadd(&f(i, j, k, UEDEN), r[R::ED]);
#pragma unroll
    for (int n = 0; n < NS; ++n) aadd(&f(i, j, k, UFS + n), r[R::X + n]);
    aadd(&qg(i, j, k, GDPRES), r[R::PG]);
    aadd(&qg(i, j, k, GDU + normal), r[R::UG]);
}

// box launch whose body returns a double; the block sums are added to *out
// Per-block partials of the scalar reductions go to a device buffer (no
// same-address atomics from thousands of blocks); a one-block kernel then adds
// their sum to the output scalar(s).
constexpr int PART_MAX = 1 << 20;
// PART_MAX x 2 doubles per device, allocated on first use on that device;
// shared by every reduction of this library on the device, which are issued on
// the library stream one after another
constexpr int MAX_DEVICES = 64;
double* g_part_dev[MAX_DEVICES] = {};
double* g_part = nullptr;   // the current device's buffer (set by part_buffer)

__global__ void k_finish_sum(const double* part, int nb, double* out0, double* out1)
{
    __shared__ double red[2][32];
    double s0 = 0.0, s1 = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) { s0 += part[2 * b]; s1 += part[2 * b + 1]; }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = s0; red[1][threadIdx.x >> 5] = s1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += red[0][w]; b += red[1][w]; }
        if (out0) *out0 += a;
        if (out1) *out1 += b;
    }
}

bool part_buffer()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
        set_error(CASTRO_ERR_CUDA, "adjoint: current device");
        return false;
    }
    if (!g_part_dev[dev] && cudaMalloc(&g_part_dev[dev], sizeof(double) * 2 * PART_MAX) != cudaSuccess) {
        g_part_dev[dev] = nullptr;
        set_error(CASTRO_ERR_CUDA, "adjoint: partial-sum buffer");
        return false;
    }
    g_part = g_part_dev[dev];
    return true;
}

template <class F>
__global__ void k_box_sum(BoxRange r, F f, double* out)
{
    __shared__ double red[32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (t < r.n) {
        int i = r.lx + (int)(t % r.nx);
        long long t2 = t / r.nx;
        int j = r.ly + (int)(t2 % r.ny);
        int k = r.lz + (int)(t2 / r.ny);
        v = f(i, j, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        out[2 * blockIdx.x] = s;
        out[2 * blockIdx.x + 1] = 0.0;
    }
}

// same with two sums: the body returns a double2
template <int MINB, class F>
__global__ void __launch_bounds__(128, MINB) k_box_sum2_lb(BoxRange r, F f, double* out0);

template <class F>
__global__ void k_box_sum2(BoxRange r, F f, double* out0)
{
    __shared__ double red[2][32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double2 v = make_double2(0.0, 0.0);
    if (t < r.n) {
        int i = r.lx + (int)(t % r.nx);
        long long t2 = t / r.nx;
        int j = r.ly + (int)(t2 % r.ny);
        int k = r.lz + (int)(t2 / r.ny);
        v = f(i, j, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = v.x; red[1][threadIdx.x >> 5] = v.y; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s0 += red[0][w]; s1 += red[1][w]; }
        out0[2 * blockIdx.x] = s0;
        out0[2 * blockIdx.x + 1] = s1;
    }
}

template <int MINB, class F>
__global__ void __launch_bounds__(128, MINB) k_box_sum2_lb(BoxRange r, F f, double* out0)
{
    __shared__ double red[2][32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double2 v = make_double2(0.0, 0.0);
    if (t < r.n) {
        int i = r.lx + (int)(t % r.nx);
        long long t2 = t / r.nx;
        int j = r.ly + (int)(t2 % r.ny);
        int k = r.lz + (int)(t2 / r.ny);
        v = f(i, j, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = v.x; red[1][threadIdx.x >> 5] = v.y; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { s0 += red[0][w]; s1 += red[1][w]; }
        out0[2 * blockIdx.x] = s0;
        out0[2 * blockIdx.x + 1] = s1;
    }
}

// Register budgets (minimum resident blocks of 128 per SM) of the three
// heaviest reverse kernels, chosen by timing the reverse sweep on B200
#ifndef CASTRO_ADJ_MINB_TRACE
#define CASTRO_ADJ_MINB_TRACE 4
#endif
#ifndef CASTRO_ADJ_MINB_TRANS1
#define CASTRO_ADJ_MINB_TRANS1 4
#endif
#ifndef CASTRO_ADJ_MINB_TRANS2
#define CASTRO_ADJ_MINB_TRANS2 3
#endif

// MINB = 0: no register budget
template <int MINB = 0, class F>
void launch_sum2(const char* what, const int* lo, const int* hi, F f, double* out0, double* out1)
{
    BoxRange r = make_range(lo, hi);
    if (r.n == 0) return;
    const int B = 128;
    const long long nb = (r.n + B - 1) / B;
    if (nb > PART_MAX || !part_buffer()) { set_error(CASTRO_ERR_ARG, "adjoint: box too large for the partial sums"); return; }
    if (MINB == 0) k_box_sum2<<<(unsigned)nb, B, 0, stream()>>>(r, f, g_part);
    else k_box_sum2_lb<(MINB > 0 ? MINB : 1)><<<(unsigned)nb, B, 0, stream()>>>(r, f, g_part);
    if (out0 || out1) k_finish_sum<<<1, 256, 0, stream()>>>(g_part, (int)nb, out0, out1);
    check_launch(what);
}

// k_box_sum with a register budget for MINB resident blocks of 128 threads
template <int MINB, class F>
__global__ void __launch_bounds__(128, MINB) k_box_sum_lb(BoxRange r, F f, double* out)
{
    __shared__ double red[32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (t < r.n) {
        int i = r.lx + (int)(t % r.nx);
        long long t2 = t / r.nx;
        int j = r.ly + (int)(t2 % r.ny);
        int k = r.lz + (int)(t2 / r.ny);
        v = f(i, j, k);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        out[2 * blockIdx.x] = s;
        out[2 * blockIdx.x + 1] = 0.0;
    }
}

// MINB = 0: no register budget (the compiler's choice)
template <int MINB = 0, class F>
void launch_sum(const char* what, const int* lo, const int* hi, F f, double* out)
{
    BoxRange r = make_range(lo, hi);
    if (r.n == 0) return;
    const int B = 128;
    const long long nb = (r.n + B - 1) / B;
    if (nb > PART_MAX || !part_buffer()) { set_error(CASTRO_ERR_ARG, "adjoint: box too large for the partial sums"); return; }
    if (MINB == 0) k_box_sum<<<(unsigned)nb, B, 0, stream()>>>(r, f, g_part);
    else k_box_sum_lb<(MINB > 0 ? MINB : 1)><<<(unsigned)nb, B, 0, stream()>>>(r, f, g_part);
    if (out) k_finish_sum<<<1, 256, 0, stream()>>>(g_part, (int)nb, out, nullptr);
    check_launch(what);
}

// ============================================================================
// Per-routine adjoints
// ============================================================================
template <int NS>
void ctoprim_adj_impl(const int* lo, const int* hi, Fab U, Fab QB, Fab QAB, Fab UB)
{
    launch_box("ctoprim_adj", lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NV = Dims<NS>::NVAR, QV = Dims<NS>::QVAR;
        double u[NV], qb[QV], qab[NQAUX], ub[NV];
#pragma unroll
        for (int n = 0; n < NV; ++n) { u[n] = U(i, j, k, n); ub[n] = 0.0; }
#pragma unroll
        for (int n = 0; n < QV; ++n) qb[n] = QB(i, j, k, n);
#pragma unroll
        for (int n = 0; n < NQAUX; ++n) qab[n] = QAB(i, j, k, n);
        ctoprim_pt_adj<NS>(c_eos, c_net, u, qb, qab, ub);
#pragma unroll
        for (int n = 0; n < NV; ++n) UB(i, j, k, n) += ub[n];
    });
}

template <int NS>
void clean_state_adj_impl(const int* lo, const int* hi, Fab U, Fab UB, bool frozen = false)
{
    launch_box("clean_state_adj", lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NV = Dims<NS>::NVAR;
        double u[NV], ub[NV];
#pragma unroll
        for (int n = 0; n < NV; ++n) { u[n] = U(i, j, k, n); ub[n] = UB(i, j, k, n); }
        clean_state_pt_adj<NS>(c_eos, c_net, u, ub, frozen);
#pragma unroll
        for (int n = 0; n < NV; ++n) UB(i, j, k, n) = ub[n];
    });
}

template <int NS>
void divu_adj_impl(const int* lo, const int* hi, Fab DIVB, Fab QB, double dx0, double dx1, double dx2)
{
    launch_box("divu_adj", lo, hi, [=] __device__(int i, int j, int k) {
        const double d = DIVB(i, j, k, 0);
        if (d == 0.0) return;
        const double ax = 0.25 * d / dx0, ay = 0.25 * d / dx1, az = 0.25 * d / dx2;
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                aadd(&QB(i, j - b, k - c, QU), ax);
                aadd(&QB(i - 1, j - b, k - c, QU), -ax);
                aadd(&QB(i - b, j, k - c, QV), ay);
                aadd(&QB(i - b, j - 1, k - c, QV), -ay);
                aadd(&QB(i - b, j - c, k, QW), az);
                aadd(&QB(i - b, j - c, k - 1, QW), -az);
            }
    });
}

// FLB: when given, the adjoint of the zone's flattening coefficient is left in
// FLB (stored by direction 0, added by the others) for one uflatten reverse
// after the three directions (uflatten_adj_zones); else it is reversed here
template <int NS, int D>
void trace_adj_dir(const int* lo, const int* hi, int vl, int vh, Fab Q, Fab QA, Fab QMB, Fab QPB, Fab QB, Fab QAB,
                   double dtdx, double* dtdxb, Fab FLB)
{
    launch_sum<CASTRO_ADJ_MINB_TRACE>("trace_ppm_adj", lo, hi, [=] __device__(int i, int j, int k) -> double {
        constexpr int NQS = Dims<NS>::NQS;
        QLoad ld{Q, QA};
        AtomicSink sk{QB, QAB};
        const int idx = D == 0 ? i : D == 1 ? j : k;
        double qpb[NQS], qmb[NQS];
        const bool hp = idx >= vl, hm = idx <= vh;
        if (hp) ld_state<NS>(QPB, i, j, k, qpb);
        if (hm) ld_state<NS>(QMB, i + (D == 0), j + (D == 1), k + (D == 2), qmb);
        double flatn = uflatten(ld, i, j, k);
        double dtdxb_l = 0.0;
        double fb = trace_zone_adj<NS, D>(ld, sk, i, j, k, dtdx, flatn, hp ? qpb : nullptr, hm ? qmb : nullptr, dtdxb_l);
        if (FLB.p) {
            if (D == 0) FLB(i, j, k, 0) = fb;
            else FLB(i, j, k, 0) += fb;
        } else {
            uflatten_adj(ld, sk, i, j, k, fb);
        }
        return dtdxb_l;
    }, dtdxb);
}

// the flattening reverse of every zone with the adjoint summed over the three
// trace directions (uflatten_adj is linear in that adjoint)
template <int NS>
void uflatten_adj_zones(const int* lo, const int* hi, Fab Q, Fab QA, Fab QB, Fab QAB, Fab FLB)
{
    launch_box("uflatten_adj zones", lo, hi, [=] __device__(int i, int j, int k) {
        QLoad ld{Q, QA};
        AtomicSink sk{QB, QAB};
        uflatten_adj(ld, sk, i, j, k, FLB(i, j, k, 0));
    });
}

template <int NS>
void trace_adj_impl(const int* lo, const int* hi, const int* vlo, const int* vhi, int idir, Fab Q, Fab QA, Fab QMB,
                    Fab QPB, Fab QB, Fab QAB, double dtdx, double* dtdxb, Fab FLB = Fab{})
{
    if (idir == 0) trace_adj_dir<NS, 0>(lo, hi, vlo[0], vhi[0], Q, QA, QMB, QPB, QB, QAB, dtdx, dtdxb, FLB);
    else if (idir == 1) trace_adj_dir<NS, 1>(lo, hi, vlo[1], vhi[1], Q, QA, QMB, QPB, QB, QAB, dtdx, dtdxb, FLB);
    else trace_adj_dir<NS, 2>(lo, hi, vlo[2], vhi[2], Q, QA, QMB, QPB, QB, QAB, dtdx, dtdxb, FLB);
}

template <int NS>
__device__ __forceinline__ void put_state(const Fab& f, int i, int j, int k, const double* s)
{
    f(i, j, k, QRHO) = s[SRHO];
    f(i, j, k, QU) = s[SU];
    f(i, j, k, QV) = s[SV];
    f(i, j, k, QW) = s[SW];
    f(i, j, k, QPRES) = s[SPRES];
    f(i, j, k, QREINT) = s[SREI];
#pragma unroll
    for (int n = 0; n < NS; ++n) f(i, j, k, QFS + n) = s[SX + n];
}

// STORE: the face-state adjoints are written instead of accumulated (the
// caller's first writer of those faces, so they need no zeroing)
template <int NS, int D, bool STORE = false>
void compute_flux_adj_dir(const int* lo, const int* hi, Fab QL, Fab QR, Fab QA, Fab FXB, Fab QGB, Fab QLB, Fab QRB,
                          Fab QAB)
{
    launch_box("compute_flux_adj", lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NQS = Dims<NS>::NQS, NV = Dims<NS>::NVAR;
        constexpr int ex = D == 0, ey = D == 1, ez = D == 2;
        double ql[NQS], qr[NQS], flxb[NV], qgb[NGDNV], qlb[NQS], qrb[NQS];
        ld_state<NS>(QL, i, j, k, ql);
        ld_state<NS>(QR, i, j, k, qr);
#pragma unroll
        for (int n = 0; n < NV; ++n) flxb[n] = FXB(i, j, k, n);
        flxb[UTEMP] = 0.0;
#pragma unroll
        for (int n = 0; n < NGDNV; ++n) qgb[n] = QGB(i, j, k, n);
#pragma unroll
        for (int n = 0; n < NQS; ++n) { qlb[n] = 0.0; qrb[n] = 0.0; }
        double gl = 0.0, gr = 0.0, cl = 0.0, cr = 0.0;
        riemann_cgf_adj<NS, D>(ql, qr, QA(i - ex, j - ey, k - ez, QGAMC), QA(i, j, k, QGAMC), QA(i - ex, j - ey, k - ez, QC),
                               QA(i, j, k, QC), flxb, qgb, qlb, qrb, gl, gr, cl, cr);
        if (STORE) {
            put_state<NS>(QLB, i, j, k, qlb);
            put_state<NS>(QRB, i, j, k, qrb);
        } else {
            add_state<NS>(QLB, i, j, k, qlb);
            add_state<NS>(QRB, i, j, k, qrb);
        }
        aadd(&QAB(i - ex, j - ey, k - ez, QGAMC), gl);
        aadd(&QAB(i, j, k, QGAMC), gr);
        aadd(&QAB(i - ex, j - ey, k - ez, QC), cl);
        aadd(&QAB(i, j, k, QC), cr);
    });
}

template <int NS>
void compute_flux_adj_impl(const int* lo, const int* hi, Fab QL, Fab QR, Fab QA, Fab FXB, Fab QGB, Fab QLB, Fab QRB,
                           Fab QAB, int idir, bool store = false)
{
    if (store) {
        if (idir == 0) compute_flux_adj_dir<NS, 0, true>(lo, hi, QL, QR, QA, FXB, QGB, QLB, QRB, QAB);
        else if (idir == 1) compute_flux_adj_dir<NS, 1, true>(lo, hi, QL, QR, QA, FXB, QGB, QLB, QRB, QAB);
        else compute_flux_adj_dir<NS, 2, true>(lo, hi, QL, QR, QA, FXB, QGB, QLB, QRB, QAB);
        return;
    }
    if (idir == 0) compute_flux_adj_dir<NS, 0>(lo, hi, QL, QR, QA, FXB, QGB, QLB, QRB, QAB);
    else if (idir == 1) compute_flux_adj_dir<NS, 1>(lo, hi, QL, QR, QA, FXB, QGB, QLB, QRB, QAB);
    else compute_flux_adj_dir<NS, 2>(lo, hi, QL, QR, QA, FXB, QGB, QLB, QRB, QAB);
}

template <int NS>
void trans1_adj_impl(const int* lo, const int* hi, int idir1, int idir2, Fab Q2M, Fab Q2P, Fab QA, Fab F1, Fab Q1,
                     double cdtdx, Fab Q2MOB, Fab Q2POB, Fab Q2MB, Fab Q2PB, Fab QAB, Fab F1B, Fab Q1B, double* cdtdxb)
{
    launch_sum("trans1_adj", lo, hi, [=] __device__(int i, int j, int k) -> double {
        constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF;
        const int e1x = idir1 == 0, e1y = idir1 == 1, e1z = idir1 == 2;
        const int e2x = idir2 == 0, e2y = idir2 == 1, e2z = idir2 == 2;
        double cb = 0.0;
#pragma unroll
        for (int d = -1; d <= 0; ++d) {
            int il = i + d * e2x, jl = j + d * e2y, kl = k + d * e2z;
            int ir = il + e1x, jr = jl + e1y, kr = kl + e1z;
            double lq[NQS], lqob[NQS], lqb[NQS], fr[NTF], fl[NTF], frb[NTF], flb[NTF];
            ld_state<NS>(d == -1 ? Q2M : Q2P, i, j, k, lq);
            ld_state<NS>(d == -1 ? Q2MOB : Q2POB, i, j, k, lqob);
            ld_tflux<NS>(F1, Q1, ir, jr, kr, idir1, fr);
            ld_tflux<NS>(F1, Q1, il, jl, kl, idir1, fl);
#pragma unroll
            for (int n = 0; n < NQS; ++n) lqb[n] = 0.0;
#pragma unroll
            for (int n = 0; n < NTF; ++n) { frb[n] = 0.0; flb[n] = 0.0; }
            double gb = 0.0;
            trans1_state_adj<NS>(lq, fr, fl, QA(il, jl, kl, QGAMC), cdtdx, lqob, lqb, frb, flb, gb, cb);
            add_state<NS>(d == -1 ? Q2MB : Q2PB, i, j, k, lqb);
            aadd_tflux<NS>(F1B, Q1B, ir, jr, kr, idir1, frb);
            aadd_tflux<NS>(F1B, Q1B, il, jl, kl, idir1, flb);
            aadd(&QAB(il, jl, kl, QGAMC), gb);
        }
        return cb;
    }, cdtdxb);
}

template <int NS>
void trans2_adj_impl(const int* lo, const int* hi, int idir1, int idir2, int idir3, Fab QM, Fab QP, Fab QA, Fab F2,
                     Fab F3, Fab G2, Fab G3, double cdtdx2, double cdtdx3, Fab QMOB, Fab QPOB, Fab QMB, Fab QPB, Fab QAB,
                     Fab F2B, Fab F3B, Fab G2B, Fab G3B, double* cdtdx2b, double* cdtdx3b)
{
    launch_sum2("trans2_adj", lo, hi, [=] __device__(int i, int j, int k) -> double2 {
        constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF;
        const int e1x = idir1 == 0, e1y = idir1 == 1, e1z = idir1 == 2;
        const int e2x = idir2 == 0, e2y = idir2 == 1, e2z = idir2 == 2;
        const int e3x = idir3 == 0, e3y = idir3 == 1, e3z = idir3 == 2;
        double c2 = 0.0, c3 = 0.0;
#pragma unroll
        for (int d = -1; d <= 0; ++d) {
            int il = i + d * e1x, jl = j + d * e1y, kl = k + d * e1z;
            double lq[NQS], lqob[NQS], lqb[NQS], f2r[NTF], f2l[NTF], f3r[NTF], f3l[NTF];
            double f2rb[NTF], f2lb[NTF], f3rb[NTF], f3lb[NTF];
            ld_state<NS>(d == -1 ? QM : QP, i, j, k, lq);
            ld_state<NS>(d == -1 ? QMOB : QPOB, i, j, k, lqob);
            ld_tflux<NS>(F2, G2, il + e2x, jl + e2y, kl + e2z, idir2, f2r);
            ld_tflux<NS>(F2, G2, il, jl, kl, idir2, f2l);
            ld_tflux<NS>(F3, G3, il + e3x, jl + e3y, kl + e3z, idir3, f3r);
            ld_tflux<NS>(F3, G3, il, jl, kl, idir3, f3l);
#pragma unroll
            for (int n = 0; n < NQS; ++n) lqb[n] = 0.0;
#pragma unroll
            for (int n = 0; n < NTF; ++n) { f2rb[n] = 0.0; f2lb[n] = 0.0; f3rb[n] = 0.0; f3lb[n] = 0.0; }
            double gb = 0.0;
            trans2_state_adj<NS>(lq, f2r, f2l, f3r, f3l, QA(il, jl, kl, QGAMC), cdtdx2, cdtdx3, lqob, lqb, f2rb, f2lb,
                                 f3rb, f3lb, gb, c2, c3);
            add_state<NS>(d == -1 ? QMB : QPB, i, j, k, lqb);
            aadd_tflux<NS>(F2B, G2B, il + e2x, jl + e2y, kl + e2z, idir2, f2rb);
            aadd_tflux<NS>(F2B, G2B, il, jl, kl, idir2, f2lb);
            aadd_tflux<NS>(F3B, G3B, il + e3x, jl + e3y, kl + e3z, idir3, f3rb);
            aadd_tflux<NS>(F3B, G3B, il, jl, kl, idir3, f3lb);
            aadd(&QAB(il, jl, kl, QGAMC), gb);
        }
        return make_double2(c2, c3);
    }, cdtdx2b, cdtdx3b);
}

template <int NS>
void apply_av_adj_impl(const int* lo, const int* hi, int idir, double dxd, Fab DIV, Fab U, Fab FXB, Fab DIVB, Fab UB)
{
    launch_box("apply_av_adj", lo, hi, [=] __device__(int i, int j, int k) {
        double ds;
        if (idir == 0) ds = DIV(i, j, k, 0) + DIV(i, j + 1, k, 0) + DIV(i, j, k + 1, 0) + DIV(i, j + 1, k, 0);
        else if (idir == 1) ds = DIV(i, j, k, 0) + DIV(i + 1, j, k, 0) + DIV(i, j, k + 1, 0) + DIV(i + 1, j, k, 0);
        else ds = DIV(i, j, k, 0) + DIV(i + 1, j, k, 0) + DIV(i, j + 1, k, 0) + DIV(i + 1, j + 1, k, 0);
        const int ex = idir == 0, ey = idir == 1, ez = idir == 2;
        const double d1 = 0.25 * ds;
        const double div1 = 0.1 * DMIN(0.0, d1);
        double div1b = 0.0;
#pragma unroll
        for (int n = 0; n < Dims<NS>::NVAR; ++n) {
            if (n == UTEMP) continue;
            const double g = FXB(i, j, k, n) * dxd;
            if (g == 0.0) continue;
            const double du = U(i, j, k, n) - U(i - ex, j - ey, k - ez, n);
            aadd(&UB(i, j, k, n), g * div1);
            aadd(&UB(i - ex, j - ey, k - ez, n), -g * div1);
            div1b += g * du;
        }
        if (!(0.0 < d1) && div1b != 0.0) {
            const double dsb = 0.1 * 0.25 * div1b;
            if (idir == 0) {
                aadd(&DIVB(i, j, k, 0), dsb); aadd(&DIVB(i, j + 1, k, 0), 2.0 * dsb); aadd(&DIVB(i, j, k + 1, 0), dsb);
            } else if (idir == 1) {
                aadd(&DIVB(i, j, k, 0), dsb); aadd(&DIVB(i + 1, j, k, 0), 2.0 * dsb); aadd(&DIVB(i, j, k + 1, 0), dsb);
            } else {
                aadd(&DIVB(i, j, k, 0), dsb); aadd(&DIVB(i + 1, j, k, 0), dsb); aadd(&DIVB(i, j + 1, k, 0), dsb);
                aadd(&DIVB(i + 1, j + 1, k, 0), dsb);
            }
        }
    });
}

template <int NS>
void normalize_species_fluxes_adj_impl(const int* lo, const int* hi, Fab FX, Fab FXB)
{
    launch_box("normalize_species_fluxes_adj", lo, hi, [=] __device__(int i, int j, int k) {
        double sum = 0.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) sum = sum + FX(i, j, k, UFS + n);
        if (sum == 0.0) return;
        const double fr = FX(i, j, k, URHO);
        const double fac = fr / sum;
        double facb = 0.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) facb += FXB(i, j, k, UFS + n) * FX(i, j, k, UFS + n);
        const double sumb = -(facb / sum) * fac;
        FXB(i, j, k, URHO) += facb / sum;
#pragma unroll
        for (int n = 0; n < NS; ++n) FXB(i, j, k, UFS + n) = FXB(i, j, k, UFS + n) * fac + sumb;
    });
}

template <int NS>
void fill_hydro_source_adj_impl(const int* lo, const int* hi, Fab SRCB, Fab Q0, Fab Q1, Fab Q2, Fab A0, Fab A1, Fab A2,
                                Fab V, double dx0, double dx1, double dx2, Fab F0B, Fab F1B, Fab F2B, Fab Q0B, Fab Q1B,
                                Fab Q2B)
{
    launch_box("fill_hydro_source_adj", lo, hi, [=] __device__(int i, int j, int k) {
        const double volinv = 1.0 / V(i, j, k, 0);
        for (int n = 0; n < Dims<NS>::NVAR; ++n) {
            const double sb = SRCB(i, j, k, n);
            if (sb == 0.0) continue;
            const double t = sb * volinv;
            aadd(&F0B(i, j, k, n), t * A0(i, j, k, 0));
            aadd(&F0B(i + 1, j, k, n), -t * A0(i + 1, j, k, 0));
            aadd(&F1B(i, j, k, n), t * A1(i, j, k, 0));
            aadd(&F1B(i, j + 1, k, n), -t * A1(i, j + 1, k, 0));
            aadd(&F2B(i, j, k, n), t * A2(i, j, k, 0));
            aadd(&F2B(i, j, k + 1, n), -t * A2(i, j, k + 1, 0));
            if (n == UEINT) {
                const double pb = -sb;   // source -= pdivu
                {
                    const double P = 0.5 * (Q0(i + 1, j, k, GDPRES) + Q0(i, j, k, GDPRES));
                    const double Du = Q0(i + 1, j, k, GDU) - Q0(i, j, k, GDU);
                    const double Pb = pb * Du / dx0, Dub = pb * P / dx0;
                    aadd(&Q0B(i + 1, j, k, GDPRES), 0.5 * Pb); aadd(&Q0B(i, j, k, GDPRES), 0.5 * Pb);
                    aadd(&Q0B(i + 1, j, k, GDU), Dub); aadd(&Q0B(i, j, k, GDU), -Dub);
                }
                {
                    const double P = 0.5 * (Q1(i, j + 1, k, GDPRES) + Q1(i, j, k, GDPRES));
                    const double Du = Q1(i, j + 1, k, GDV) - Q1(i, j, k, GDV);
                    const double Pb = pb * Du / dx1, Dub = pb * P / dx1;
                    aadd(&Q1B(i, j + 1, k, GDPRES), 0.5 * Pb); aadd(&Q1B(i, j, k, GDPRES), 0.5 * Pb);
                    aadd(&Q1B(i, j + 1, k, GDV), Dub); aadd(&Q1B(i, j, k, GDV), -Dub);
                }
                {
                    const double P = 0.5 * (Q2(i, j, k + 1, GDPRES) + Q2(i, j, k, GDPRES));
                    const double Du = Q2(i, j, k + 1, GDW) - Q2(i, j, k, GDW);
                    const double Pb = pb * Du / dx2, Dub = pb * P / dx2;
                    aadd(&Q2B(i, j, k + 1, GDPRES), 0.5 * Pb); aadd(&Q2B(i, j, k, GDPRES), 0.5 * Pb);
                    aadd(&Q2B(i, j, k + 1, GDW), Dub); aadd(&Q2B(i, j, k, GDW), -Dub);
                }
            }
        }
    });
}

// The reverse EOS has no Coulomb corrections: with them switched on, every
// entry point that would differentiate an EOS call refuses (CASTRO_ERR_ARG).
bool coulomb_refused(const char* who)
{
    if (!network_host().coulomb) return false;
    set_error(CASTRO_ERR_ARG, (std::string(who) + ": the adjoint EOS has no Coulomb corrections").c_str());
    return true;
}

}  // namespace

// ============================================================================
// extern "C" per-routine adjoints
// ============================================================================
extern "C" {

void ctoprim_adj(const int* lo, const int* hi, const double* u, const int* u_lo, const int* u_hi,
                 const double* qb, const int* qb_lo, const int* qb_hi, const double* qab, const int* qab_lo,
                 const int* qab_hi, double* ub, const int* ub_lo, const int* ub_hi)
{
    if (coulomb_refused("ctoprim_adj")) return;
    CASTRO_DISPATCH_NS(ctoprim_adj_impl, lo, hi, make_fab(u, u_lo, u_hi), make_fab(qb, qb_lo, qb_hi),
                       make_fab(qab, qab_lo, qab_hi), make_fab(ub, ub_lo, ub_hi));
}

void clean_state_adj(const int* lo, const int* hi, const double* u, const int* u_lo, const int* u_hi, double* ub,
                     const int* ub_lo, const int* ub_hi)
{
    if (coulomb_refused("clean_state_adj")) return;
    CASTRO_DISPATCH_NS(clean_state_adj_impl, lo, hi, make_fab(u, u_lo, u_hi), make_fab(ub, ub_lo, ub_hi));
}

void divu_adj(const int* lo, const int* hi, const double* dx, const double* divb, const int* d_lo, const int* d_hi,
              double* qb, const int* q_lo, const int* q_hi)
{
    CASTRO_DISPATCH_NS(divu_adj_impl, lo, hi, make_fab(divb, d_lo, d_hi), make_fab(qb, q_lo, q_hi), dx[0], dx[1], dx[2]);
}

void trace_ppm_adj(const int* lo, const int* hi, const int* vlo, const int* vhi, const int idir,
                   const double* q, const int* q_lo, const int* q_hi, const double* qaux, const int* qa_lo,
                   const int* qa_hi, const double* qmb, const int* qm_lo, const int* qm_hi, const double* qpb,
                   const int* qp_lo, const int* qp_hi, double* qb, const int* qb_lo, const int* qb_hi, double* qab,
                   const int* qab_lo, const int* qab_hi, const double* dx, const double dt, double* dtb)
{
    if (idir < 1 || idir > 3) { set_error(CASTRO_ERR_ARG, "trace_ppm_adj: idir"); return; }
    // the kernel accumulates the adjoint of dtdx = dt/dx; dtb receives d/d(dt)
    double* tmp = nullptr;
    if (dtb && cudaMallocAsync(&tmp, sizeof(double), stream()) != cudaSuccess) { set_error(CASTRO_ERR_CUDA, "trace_ppm_adj: alloc"); return; }
    if (tmp) cudaMemsetAsync(tmp, 0, sizeof(double), stream());
    CASTRO_DISPATCH_NS(trace_adj_impl, lo, hi, vlo, vhi, idir - 1, make_fab(q, q_lo, q_hi), make_fab(qaux, qa_lo, qa_hi),
                       make_fab(qmb, qm_lo, qm_hi), make_fab(qpb, qp_lo, qp_hi), make_fab(qb, qb_lo, qb_hi),
                       make_fab(qab, qab_lo, qab_hi), dt / dx[idir - 1], tmp);
    if (tmp) {
        const double inv = 1.0 / dx[idir - 1];
        double* out = dtb;
        launch_box<32>("trace_ppm_adj(dt)", lo, lo, [=] __device__(int, int, int) { *out += *tmp * inv; });
        cudaFreeAsync(tmp, stream());
    }
}

void compute_flux_adj(const int* lo, const int* hi, const double* ql, const int* ql_lo, const int* ql_hi,
                      const double* qr, const int* qr_lo, const int* qr_hi, const double* qaux, const int* qa_lo,
                      const int* qa_hi, const double* fluxb, const int* fx_lo, const int* fx_hi, const double* qeb,
                      const int* qe_lo, const int* qe_hi, double* qlb, const int* qlb_lo, const int* qlb_hi,
                      double* qrb, const int* qrb_lo, const int* qrb_hi, double* qab, const int* qab_lo,
                      const int* qab_hi, const int idir)
{
    if (idir < 1 || idir > 3) { set_error(CASTRO_ERR_ARG, "compute_flux_adj: idir"); return; }
    CASTRO_DISPATCH_NS(compute_flux_adj_impl, lo, hi, make_fab(ql, ql_lo, ql_hi), make_fab(qr, qr_lo, qr_hi),
                       make_fab(qaux, qa_lo, qa_hi), make_fab(fluxb, fx_lo, fx_hi), make_fab(qeb, qe_lo, qe_hi),
                       make_fab(qlb, qlb_lo, qlb_hi), make_fab(qrb, qrb_lo, qrb_hi), make_fab(qab, qab_lo, qab_hi),
                       idir - 1);
}

void trans1_adj(const int* lo, const int* hi, const int idir1, const int idir2,
                const double* q2m, const int* q2m_lo, const int* q2m_hi, const double* q2p, const int* q2p_lo,
                const int* q2p_hi, const double* qaux, const int* qa_lo, const int* qa_hi, const double* f1,
                const int* f1_lo, const int* f1_hi, const double* q1, const int* q1_lo, const int* q1_hi,
                const double cdtdx, const double* q2mob, const int* q2mob_lo, const int* q2mob_hi,
                const double* q2pob, const int* q2pob_lo, const int* q2pob_hi, double* q2mb, const int* q2mb_lo,
                const int* q2mb_hi, double* q2pb, const int* q2pb_lo, const int* q2pb_hi, double* qab,
                const int* qab_lo, const int* qab_hi, double* f1b, const int* f1b_lo, const int* f1b_hi, double* q1b,
                const int* q1b_lo, const int* q1b_hi, double* cdtdxb)
{
    if (idir1 < 1 || idir1 > 3 || idir2 < 1 || idir2 > 3 || idir1 == idir2) { set_error(CASTRO_ERR_ARG, "trans1_adj: idir"); return; }
    CASTRO_DISPATCH_NS(trans1_adj_impl, lo, hi, idir1 - 1, idir2 - 1, make_fab(q2m, q2m_lo, q2m_hi),
                       make_fab(q2p, q2p_lo, q2p_hi), make_fab(qaux, qa_lo, qa_hi), make_fab(f1, f1_lo, f1_hi),
                       make_fab(q1, q1_lo, q1_hi), cdtdx, make_fab(q2mob, q2mob_lo, q2mob_hi),
                       make_fab(q2pob, q2pob_lo, q2pob_hi), make_fab(q2mb, q2mb_lo, q2mb_hi),
                       make_fab(q2pb, q2pb_lo, q2pb_hi), make_fab(qab, qab_lo, qab_hi), make_fab(f1b, f1b_lo, f1b_hi),
                       make_fab(q1b, q1b_lo, q1b_hi), cdtdxb);
}

void trans2_adj(const int* lo, const int* hi, const int idir1, const int idir2, const int idir3,
                const double* qm, const int* qm_lo, const int* qm_hi, const double* qp, const int* qp_lo,
                const int* qp_hi, const double* qaux, const int* qa_lo, const int* qa_hi, const double* fyz,
                const int* fyz_lo, const int* fyz_hi, const double* fzy, const int* fzy_lo, const int* fzy_hi,
                const double* qy, const int* qy_lo, const int* qy_hi, const double* qz, const int* qz_lo,
                const int* qz_hi, const double cdtdy, const double cdtdz, const double* qmob, const int* qmob_lo,
                const int* qmob_hi, const double* qpob, const int* qpob_lo, const int* qpob_hi, double* qmb,
                const int* qmb_lo, const int* qmb_hi, double* qpb, const int* qpb_lo, const int* qpb_hi, double* qab,
                const int* qab_lo, const int* qab_hi, double* fyzb, const int* fyzb_lo, const int* fyzb_hi,
                double* fzyb, const int* fzyb_lo, const int* fzyb_hi, double* qyb, const int* qyb_lo,
                const int* qyb_hi, double* qzb, const int* qzb_lo, const int* qzb_hi, double* cdtdyb, double* cdtdzb)
{
    if (idir1 < 1 || idir1 > 3 || idir2 < 1 || idir2 > 3 || idir3 < 1 || idir3 > 3) { set_error(CASTRO_ERR_ARG, "trans2_adj: idir"); return; }
    CASTRO_DISPATCH_NS(trans2_adj_impl, lo, hi, idir1 - 1, idir2 - 1, idir3 - 1, make_fab(qm, qm_lo, qm_hi),
                       make_fab(qp, qp_lo, qp_hi), make_fab(qaux, qa_lo, qa_hi), make_fab(fyz, fyz_lo, fyz_hi),
                       make_fab(fzy, fzy_lo, fzy_hi), make_fab(qy, qy_lo, qy_hi), make_fab(qz, qz_lo, qz_hi), cdtdy,
                       cdtdz, make_fab(qmob, qmob_lo, qmob_hi), make_fab(qpob, qpob_lo, qpob_hi),
                       make_fab(qmb, qmb_lo, qmb_hi), make_fab(qpb, qpb_lo, qpb_hi), make_fab(qab, qab_lo, qab_hi),
                       make_fab(fyzb, fyzb_lo, fyzb_hi), make_fab(fzyb, fzyb_lo, fzyb_hi), make_fab(qyb, qyb_lo, qyb_hi),
                       make_fab(qzb, qzb_lo, qzb_hi), cdtdyb, cdtdzb);
}

void apply_av_adj(const int* lo, const int* hi, const int idir, const double* dx, const double* div, const int* d_lo,
                  const int* d_hi, const double* sb, const int* s_lo, const int* s_hi, const double* fluxb,
                  const int* f_lo, const int* f_hi, double* divb, const int* db_lo, const int* db_hi, double* sbb,
                  const int* sbb_lo, const int* sbb_hi)
{
    if (idir < 1 || idir > 3) { set_error(CASTRO_ERR_ARG, "apply_av_adj: idir"); return; }
    CASTRO_DISPATCH_NS(apply_av_adj_impl, lo, hi, idir - 1, dx[idir - 1], make_fab(div, d_lo, d_hi),
                       make_fab(sb, s_lo, s_hi), make_fab(fluxb, f_lo, f_hi), make_fab(divb, db_lo, db_hi),
                       make_fab(sbb, sbb_lo, sbb_hi));
}

void normalize_species_fluxes_adj(const int* lo, const int* hi, const double* flux, const int* f_lo, const int* f_hi,
                                  double* fluxb, const int* fb_lo, const int* fb_hi)
{
    CASTRO_DISPATCH_NS(normalize_species_fluxes_adj_impl, lo, hi, make_fab(flux, f_lo, f_hi),
                       make_fab(fluxb, fb_lo, fb_hi));
}

void fill_hydro_source_adj(const int* lo, const int* hi, const double* sourceb, const int* sr_lo, const int* sr_hi,
                           const double* qe0, const int* qe0_lo, const int* qe0_hi,
                           const double* qe1, const int* qe1_lo, const int* qe1_hi,
                           const double* qe2, const int* qe2_lo, const int* qe2_hi,
                           const double* area0, const int* a0_lo, const int* a0_hi,
                           const double* area1, const int* a1_lo, const int* a1_hi,
                           const double* area2, const int* a2_lo, const int* a2_hi,
                           const double* volume, const int* v_lo, const int* v_hi, const double* dx,
                           double* flux0b, const int* f0_lo, const int* f0_hi,
                           double* flux1b, const int* f1_lo, const int* f1_hi,
                           double* flux2b, const int* f2_lo, const int* f2_hi,
                           double* qe0b, const int* qe0b_lo, const int* qe0b_hi,
                           double* qe1b, const int* qe1b_lo, const int* qe1b_hi,
                           double* qe2b, const int* qe2b_lo, const int* qe2b_hi)
{
    CASTRO_DISPATCH_NS(fill_hydro_source_adj_impl, lo, hi, make_fab(sourceb, sr_lo, sr_hi),
                       make_fab(qe0, qe0_lo, qe0_hi), make_fab(qe1, qe1_lo, qe1_hi), make_fab(qe2, qe2_lo, qe2_hi),
                       make_fab(area0, a0_lo, a0_hi), make_fab(area1, a1_lo, a1_hi), make_fab(area2, a2_lo, a2_hi),
                       make_fab(volume, v_lo, v_hi), dx[0], dx[1], dx[2], make_fab(flux0b, f0_lo, f0_hi),
                       make_fab(flux1b, f1_lo, f1_hi), make_fab(flux2b, f2_lo, f2_hi),
                       make_fab(qe0b, qe0b_lo, qe0b_hi), make_fab(qe1b, qe1b_lo, qe1b_hi),
                       make_fab(qe2b, qe2b_lo, qe2b_hi));
}

}  // extern "C"

// ============================================================================
// Checkpointed reverse sweep of a Sedov run
// ============================================================================
namespace {

struct IBx { int lo[3], hi[3]; };
IBx growb(IBx b, int gx, int gy, int gz)
{
    b.lo[0] -= gx; b.lo[1] -= gy; b.lo[2] -= gz;
    b.hi[0] += gx; b.hi[1] += gy; b.hi[2] += gz;
    return b;
}
long long nptsb(const IBx& b) { return (long long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1); }

struct Arr {
    double* p = nullptr;
    IBx b{};
    int nc = 0;
    Fab fab() const { return make_fab(p, b.lo, b.hi); }
    long long n() const { return nptsb(b) * nc; }
};

__device__ __forceinline__ int map_bc_adj(int i, int lo, int hi, int bc)
{
    if (bc == CASTRO_BC_PERIODIC) {
        int n = hi - lo + 1;
        int r = (i - lo) % n;
        if (r < 0) r += n;
        return lo + r;
    }
    return i < lo ? lo : (i > hi ? hi : i);
}

}  // namespace

struct Prim {
    Arr A, Bs, Cs, Sb, q, qaux, div, qint, qm[3][3], qp[3][3], F1[3], G1[3], F2[3][3], G2[3][3], ql[3], qr[3];
    Arr Fav[3], flux[3], qe[3], src;
};

struct castro_adj {
    int ns = 2, nv = 9, qv = 10;
    // dom: the instance's domain, held as one box.  bx and its grown boxes are
    // the working box: the domain itself, or one z-slab of it when the step is
    // reversed slab by slab (the per-step arrays are then slab-sized and move
    // from slab to slab; the states and their adjoints stay domain-sized)
    IBx dom{};
    std::vector<IBx> slabs;
    std::vector<Arr*> slab_arrs;
    int n_start = 0;   // first step of the differentiated window (0: from initdata)
    IBx bx{}, obx{}, qbx{}, ebx[3], gebx[3], tbx[3][3];
    int bc = CASTRO_BC_OUTFLOW;
    double dx[3] = {0, 0, 0}, problo[3] = {0, 0, 0}, probhi[3] = {0, 0, 0};
    castro_problem prob{};
    double stop_time = -1.0;
    int nsteps = 0, ckpt = 5;
    double shell_r0 = 0.3, shell_r1 = 0.4;
    cudaStream_t st = nullptr;
    std::vector<char*> blocks;
    std::vector<Arr> all;   // every allocation (size accounting)
    // primal
    std::vector<Arr> ckpts;   // V at steps 0, ckpt, 2 ckpt, ...
    std::vector<Arr> seg;     // V_n of the segment being reversed
    // forward intermediates of one step; one set per step of a checkpoint
    // segment when device memory allows (the reverse then reads the set the
    // segment recomputation filled), else one set recomputed per step
    std::vector<Prim> sets;
    Prim* P = nullptr;
    Arr V, area[3], vol, Vfinal;
    // adjoint
    Arr flb;   // adjoint of the flattening coefficient, summed over the trace directions
    Arr Vb, Ab, Sbb, qb, qab, divb, qmb[3][3], qpb[3][3], F1b[3], G1b[3], F2b[3][3], G2b[3][3], qlb[3], qrb[3];
    Arr fluxb[3], qeb[3], srcb;
    // per-zone flux-record adjoints of the zone-based transverse reverses:
    // T1L/T1R[d][t] for trans1 (flux d correcting states normal to t),
    // T2L/T2R[d][0|1] for trans2 of direction d (fluxes t1|t2 and t2|t1)
    Arr T1L[3][3], T1R[3][3], T2L[3][2], T2R[3][2];
    double* d_scal = nullptr;   // [32] scalar accumulators
    int* d_idx = nullptr;
    double* d_est = nullptr;
    double* d_chain = nullptr;  // time-step adjoint chain of the reverse sweep
    std::vector<double> dts, times, ests, estmin;
    std::vector<char> limited, clamped;
    double J = 0.0;
    bool fwd_done = false;
    bool last_seg_ready = false;   // the forward left the last segment's states and intermediates
    float ms_forward = 0.0f, ms_backward = 0.0f;
};

namespace {

struct StreamScope {
    cudaStream_t saved;
    explicit StreamScope(cudaStream_t s) : saved(stream()) { castro_set_stream(s); }
    ~StreamScope() { castro_set_stream(saved); }
};

// the working box and its grown boxes (Source/Castro_hydro.cpp:81-101)
void set_geometry(castro_adj* a, const IBx& b)
{
    a->bx = b;
    a->obx = growb(b, 1, 1, 1);
    a->qbx = growb(b, NG, NG, NG);
    for (int d = 0; d < 3; ++d) {
        a->ebx[d] = b;
        a->ebx[d].hi[d] += 1;
        a->gebx[d] = growb(a->ebx[d], 1, 1, 1);
    }
    a->tbx[0][0] = growb(a->ebx[0], 0, 1, 1); a->tbx[0][1] = growb(a->ebx[0], 0, 0, 1); a->tbx[0][2] = growb(a->ebx[0], 0, 1, 0);
    a->tbx[1][0] = growb(a->ebx[1], 0, 0, 1); a->tbx[1][1] = growb(a->ebx[1], 1, 0, 1); a->tbx[1][2] = growb(a->ebx[1], 1, 0, 0);
    a->tbx[2][0] = growb(a->ebx[2], 0, 1, 0); a->tbx[2][1] = growb(a->ebx[2], 1, 0, 0); a->tbx[2][2] = growb(a->ebx[2], 1, 1, 0);
}

// make slab s the working box: the slab-sized arrays (every slab has the same
// shape) are re-labelled with the slab's z position
void use_slab(castro_adj* a, int s)
{
    const int shift = a->slabs[s].lo[2] - a->bx.lo[2];
    if (shift == 0) return;
    set_geometry(a, a->slabs[s]);
    for (Arr* r : a->slab_arrs) {
        r->b.lo[2] += shift;
        r->b.hi[2] += shift;
    }
}

bool alloc_arr(castro_adj* a, Arr& r, const IBx& b, int nc)
{
    r.b = b;
    r.nc = nc;
    size_t bytes = (size_t)r.n() * sizeof(double);
    char* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return false;
    a->blocks.push_back(p);
    r.p = (double*)p;
    a->all.push_back(r);
    return true;
}

void zero(const Arr& r, cudaStream_t s) { cudaMemsetAsync(r.p, 0, (size_t)r.n() * sizeof(double), s); }
void copy(const Arr& d, const Arr& s, cudaStream_t st)
{
    cudaMemcpyAsync(d.p, s.p, (size_t)s.n() * sizeof(double), cudaMemcpyDeviceToDevice, st);
}

__global__ void k_fill_const(double* p, long long n, double v)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) p[t] = v;
}

void fill_const(const Arr& r, double v, cudaStream_t s)
{
    long long n = r.n();
    k_fill_const<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(r.p, n, v);
}

void clean(const IBx& b, const Arr& u)
{
    enforce_minimum_density(b.lo, b.hi, u.p, u.b.lo, u.b.hi);
    normalize_species(b.lo, b.hi, u.p, u.b.lo, u.b.hi);
    reset_internal_e(b.lo, b.hi, u.p, u.b.lo, u.b.hi);
    compute_temp(b.lo, b.hi, u.p, u.b.lo, u.b.hi);
}

// Sborder fill: every zone of qbx from A under the boundary condition
template <int NS>
void fill_sborder(castro_adj* a)
{
    Fab S = a->P->Sb.fab(), A = a->P->A.fab();     // A: the domain's cleaned S_old
    const int bc = a->bc;
    const IBx bx = a->dom;
    launch_box("adj fill", a->qbx.lo, a->qbx.hi, [=] __device__(int i, int j, int k) {
        int ii = map_bc_adj(i, bx.lo[0], bx.hi[0], bc);
        int jj = map_bc_adj(j, bx.lo[1], bx.hi[1], bc);
        int kk = map_bc_adj(k, bx.lo[2], bx.hi[2], bc);
#pragma unroll
        for (int n = 0; n < Dims<NS>::NVAR; ++n) S(i, j, k, n) = A(ii, jj, kk, n);
    });
}

// adjoint of "Sb = clean(fill(A))" on qbx: accumulates into Ab
template <int NS>
void fill_clean_adj(castro_adj* a)
{
    Fab SB = a->Sbb.fab(), A = a->P->A.fab(), AB = a->Ab.fab();   // A, AB: domain-sized
    const int bc = a->bc;
    const IBx bx = a->dom;
    launch_box("adj fill_clean", a->qbx.lo, a->qbx.hi, [=] __device__(int i, int j, int k) {
        constexpr int NV = Dims<NS>::NVAR;
        int ii = map_bc_adj(i, bx.lo[0], bx.hi[0], bc);
        int jj = map_bc_adj(j, bx.lo[1], bx.hi[1], bc);
        int kk = map_bc_adj(k, bx.lo[2], bx.hi[2], bc);
        double u[NV], ub[NV];
        bool any = false;
#pragma unroll
        for (int n = 0; n < NV; ++n) { u[n] = A(ii, jj, kk, n); ub[n] = SB(i, j, k, n); any |= ub[n] != 0.0; }
        if (!any) return;
        clean_state_pt_adj<NS>(c_eos, c_net, u, ub, true);
#pragma unroll
        for (int n = 0; n < NV; ++n) aadd(&AB(ii, jj, kk, n), ub[n]);
    });
}

// diagnostics: with CASTRO_ADJ_CHECK set, every adjoint array is scanned after
// each reverse stage and the first stage that leaves a non-finite value is
// reported through castro_last_error
__global__ void k_nonfinite(const double* p, long long n, int* flag, double* amax)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        if (!isfinite(p[t])) atomicExch(flag, 1);
        else if (amax) {
            double a = fabs(p[t]);
            if (a > 0.0) atomicMax((unsigned long long*)amax, (unsigned long long)__double_as_longlong(a));
        }
    }
}

int adj_check_level()
{
    static int on = -1;
    if (on < 0) {
        const char* e = getenv("CASTRO_ADJ_CHECK");
        on = e ? atoi(e) : 0;
        if (e && on == 0) on = 1;
    }
    return on;
}
bool adj_check_enabled() { return adj_check_level() > 0; }

void adj_check(castro_adj* a, const char* stage);
void adj_mark(castro_adj* a, const char* name);
inline void adj_stage(castro_adj* a, const char* stage)
{
    adj_check(a, stage);
    adj_mark(a, stage);
}

void adj_check(castro_adj* a, const char* stage)
{
    if (!adj_check_enabled()) return;
    std::vector<std::pair<const char*, const Arr*>> arrs = {
        {"Vb", &a->Vb}, {"Ab", &a->Ab}, {"Sbb", &a->Sbb}, {"qb", &a->qb}, {"qab", &a->qab}, {"divb", &a->divb},
        {"srcb", &a->srcb}, {"flb", &a->flb}};
    for (int d = 0; d < 3; ++d) {
        arrs.push_back({"F1b", &a->F1b[d]}); arrs.push_back({"G1b", &a->G1b[d]});
        arrs.push_back({"qlb", &a->qlb[d]}); arrs.push_back({"qrb", &a->qrb[d]});
        arrs.push_back({"fluxb", &a->fluxb[d]}); arrs.push_back({"qeb", &a->qeb[d]});
        for (int e = 0; e < 3; ++e) {
            arrs.push_back({"qmb", &a->qmb[d][e]}); arrs.push_back({"qpb", &a->qpb[d][e]});
            arrs.push_back({"F2b", &a->F2b[d][e]}); arrs.push_back({"G2b", &a->G2b[d][e]});
        }
    }
    const bool mags = adj_check_level() >= 2;
    std::string line;
    for (auto& pr : arrs) {
        cudaMemsetAsync(a->d_idx, 0, sizeof(int), a->st);
        cudaMemsetAsync(a->d_scal + 31, 0, sizeof(double), a->st);
        long long n = pr.second->n();
        k_nonfinite<<<(unsigned)((n + 255) / 256), 256, 0, a->st>>>(pr.second->p, n, a->d_idx,
                                                                     mags ? a->d_scal + 31 : nullptr);
        int f = 0;
        double mx = 0.0;
        cudaMemcpyAsync(&f, a->d_idx, sizeof f, cudaMemcpyDeviceToHost, a->st);
        cudaMemcpyAsync(&mx, a->d_scal + 31, sizeof mx, cudaMemcpyDeviceToHost, a->st);
        cudaStreamSynchronize(a->st);
        if (mags && mx > 0.0) {
            char b[64];
            snprintf(b, sizeof b, " %s=%.1e", pr.first, mx);
            line += b;
        }
        if (f) {
            char buf[160];
            snprintf(buf, sizeof buf, "adjoint check: non-finite %s after %s", pr.first, stage);
            fprintf(stderr, "%s\n", buf);
            set_error(CASTRO_ERR_EOS, buf);
            return;
        }
    }
    if (mags) fprintf(stderr, "[%s]%s\n", stage, line.c_str());
}

// stage timing: with CASTRO_ADJ_PROFILE set, CUDA events between the stages of
// the reverse sweep; castro_adj_backward prints the accumulated table
struct AdjProf {
    std::vector<std::pair<std::string, cudaEvent_t>> marks;
    std::vector<std::pair<std::string, double>> total;
};
AdjProf g_prof;
bool adj_prof_enabled()
{
    static int on = -1;
    if (on < 0) on = getenv("CASTRO_ADJ_PROFILE") ? 1 : 0;
    return on == 1;
}
void adj_mark(castro_adj* a, const char* name)
{
    if (!adj_prof_enabled()) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, a->st);
    g_prof.marks.push_back({name, e});
}
void adj_prof_flush()
{
    if (!adj_prof_enabled() || g_prof.marks.empty()) return;
    cudaEventSynchronize(g_prof.marks.back().second);
    for (size_t i = 1; i < g_prof.marks.size(); ++i) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, g_prof.marks[i - 1].second, g_prof.marks[i].second);
        const std::string& nm = g_prof.marks[i].first;
        bool found = false;
        for (auto& t : g_prof.total)
            if (t.first == nm) { t.second += ms; found = true; break; }
        if (!found) g_prof.total.push_back({nm, ms});
    }
    for (auto& m : g_prof.marks) cudaEventDestroy(m.second);
    g_prof.marks.clear();
}
void adj_prof_report()
{
    if (!adj_prof_enabled()) return;
    adj_prof_flush();
    double sum = 0.0;
    for (auto& t : g_prof.total) sum += t.second;
    fprintf(stderr, "adjoint stage times (ms, summed over the sweep):\n");
    for (auto& t : g_prof.total) fprintf(stderr, "  %-28s %9.3f  %5.1f%%\n", t.first.c_str(), t.second, 100.0 * t.second / sum);
    g_prof.total.clear();
}

// B = A + dt*src (valid box); Saxpy of Source/Castro_advance.cpp:74
// clean_state(S_old) of the whole domain, Castro_advance.cpp:51: the step's
// every working box (the domain, or each slab in turn) fills its Sborder from it
void begin_step(castro_adj* a, const Arr& Vin)
{
    copy(a->P->A, Vin, a->st);
    clean(a->dom, a->P->A);
}

__global__ void k_saxpy_box(BoxRange r, Fab A, Fab S, Fab B, int nv, double dt)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= r.n) return;
    const int i = r.lx + (int)(t % r.nx);
    const long long t2 = t / r.nx;
    const int j = r.ly + (int)(t2 % r.ny);
    const int k = r.lz + (int)(t2 / r.ny);
    for (int n = 0; n < nv; ++n) B(i, j, k, n) = A(i, j, k, n) + dt * S(i, j, k, n);
}

// the forward of one step on the working box from the domain's cleaned S_old
// (begin_step), with every intermediate kept
template <int NS>
void forward_step(castro_adj* a, double dt)
{
    cudaStream_t st = a->st;
    fill_sborder<NS>(a);
    clean(a->qbx, a->P->Sb);                                      // clean_state(Sborder)
    const IBx &bx = a->bx, &obx = a->obx, &qbx = a->qbx;
    ctoprim(qbx.lo, qbx.hi, a->P->Sb.p, qbx.lo, qbx.hi, a->P->q.p, qbx.lo, qbx.hi, a->P->qaux.p, qbx.lo, qbx.hi);
    divu(obx.lo, obx.hi, a->P->q.p, qbx.lo, qbx.hi, a->dx, a->P->div.p, obx.lo, obx.hi);
    double hdtdx[3], cdtdx[3];
    for (int d = 0; d < 3; ++d) { hdtdx[d] = 0.5 * dt / a->dx[d]; cdtdx[d] = dt / a->dx[d] / 3.0; }
    for (int d = 0; d < 3; ++d)
        trace_ppm(obx.lo, obx.hi, bx.lo, bx.hi, d + 1, a->P->q.p, qbx.lo, qbx.hi, a->P->qaux.p, qbx.lo, qbx.hi,
                  a->P->qm[d][d].p, a->P->qm[d][d].b.lo, a->P->qm[d][d].b.hi, a->P->qp[d][d].p, a->P->qp[d][d].b.lo,
                  a->P->qp[d][d].b.hi, bx.lo, bx.hi, a->dx, dt);
    for (int d = 0; d < 3; ++d) {
        const IBx& b = a->tbx[d][d];
        compute_flux(b.lo, b.hi, a->P->qm[d][d].p, a->P->qm[d][d].b.lo, a->P->qm[d][d].b.hi, a->P->qp[d][d].p, a->P->qp[d][d].b.lo,
                     a->P->qp[d][d].b.hi, a->P->F1[d].p, obx.lo, obx.hi, a->P->qint.p, obx.lo, obx.hi, a->P->G1[d].p, obx.lo,
                     obx.hi, a->P->qaux.p, qbx.lo, qbx.hi, d + 1);
        for (int tt = 0; tt < 2; ++tt) {
            int t = (tt == 0) ? (d == 0 ? 1 : 0) : (d == 2 ? 1 : 2);
            const IBx& tb = a->tbx[t][d];
            trans1(tb.lo, tb.hi, d + 1, t + 1, a->P->qm[t][t].p, a->P->qm[t][t].b.lo, a->P->qm[t][t].b.hi, a->P->qm[t][d].p,
                   a->P->qm[t][d].b.lo, a->P->qm[t][d].b.hi, a->P->qp[t][t].p, a->P->qp[t][t].b.lo, a->P->qp[t][t].b.hi,
                   a->P->qp[t][d].p, a->P->qp[t][d].b.lo, a->P->qp[t][d].b.hi, a->P->qaux.p, qbx.lo, qbx.hi, a->P->F1[d].p, obx.lo,
                   obx.hi, a->P->G1[d].p, obx.lo, obx.hi, cdtdx[d]);
        }
    }
    for (int d = 0; d < 3; ++d) {
        int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
        for (int pp = 0; pp < 2; ++pp) {
            int x = pp == 0 ? t1 : t2, y = pp == 0 ? t2 : t1;
            const IBx& b = a->tbx[x][y];
            compute_flux(b.lo, b.hi, a->P->qm[x][y].p, a->P->qm[x][y].b.lo, a->P->qm[x][y].b.hi, a->P->qp[x][y].p,
                         a->P->qp[x][y].b.lo, a->P->qp[x][y].b.hi, a->P->F2[x][y].p, obx.lo, obx.hi, a->P->qint.p, obx.lo, obx.hi,
                         a->P->G2[x][y].p, obx.lo, obx.hi, a->P->qaux.p, qbx.lo, qbx.hi, x + 1);
        }
        trans2(a->ebx[d].lo, a->ebx[d].hi, d + 1, t1 + 1, t2 + 1, a->P->qm[d][d].p, a->P->qm[d][d].b.lo, a->P->qm[d][d].b.hi,
               a->P->ql[d].p, obx.lo, obx.hi, a->P->qp[d][d].p, a->P->qp[d][d].b.lo, a->P->qp[d][d].b.hi, a->P->qr[d].p, obx.lo,
               obx.hi, a->P->qaux.p, qbx.lo, qbx.hi, a->P->F2[t1][t2].p, obx.lo, obx.hi, a->P->F2[t2][t1].p, obx.lo, obx.hi,
               a->P->G2[t1][t2].p, obx.lo, obx.hi, a->P->G2[t2][t1].p, obx.lo, obx.hi, hdtdx[d], hdtdx[t1], hdtdx[t2]);
        compute_flux(a->ebx[d].lo, a->ebx[d].hi, a->P->ql[d].p, obx.lo, obx.hi, a->P->qr[d].p, obx.lo, obx.hi,
                     a->P->flux[d].p, a->gebx[d].lo, a->gebx[d].hi, a->P->qint.p, obx.lo, obx.hi, a->P->qe[d].p,
                     a->gebx[d].lo, a->gebx[d].hi, a->P->qaux.p, qbx.lo, qbx.hi, d + 1);
    }
    for (int d = 0; d < 3; ++d) {
        apply_av(a->ebx[d].lo, a->ebx[d].hi, d + 1, a->dx, a->P->div.p, obx.lo, obx.hi, a->P->Sb.p, qbx.lo, qbx.hi,
                 a->P->flux[d].p, a->gebx[d].lo, a->gebx[d].hi);
        copy(a->P->Fav[d], a->P->flux[d], st);
        normalize_species_fluxes(a->ebx[d].lo, a->ebx[d].hi, a->P->flux[d].p, a->gebx[d].lo, a->gebx[d].hi);
    }
    zero(a->P->src, st);                                          // hydro_source.setVal(0)
    fill_hydro_source(bx.lo, bx.hi, a->P->Sb.p, qbx.lo, qbx.hi, a->P->q.p, qbx.lo, qbx.hi, a->P->src.p, bx.lo, bx.hi,
                      a->P->flux[0].p, a->gebx[0].lo, a->gebx[0].hi, a->P->flux[1].p, a->gebx[1].lo, a->gebx[1].hi,
                      a->P->flux[2].p, a->gebx[2].lo, a->gebx[2].hi, a->P->qe[0].p, a->gebx[0].lo, a->gebx[0].hi,
                      a->P->qe[1].p, a->gebx[1].lo, a->gebx[1].hi, a->P->qe[2].p, a->gebx[2].lo, a->gebx[2].hi,
                      a->area[0].p, a->gebx[0].lo, a->gebx[0].hi, a->area[1].p, a->gebx[1].lo, a->gebx[1].hi,
                      a->area[2].p, a->gebx[2].lo, a->gebx[2].hi, a->vol.p, bx.lo, bx.hi, a->dx, dt);
    {
        BoxRange r = make_range(bx.lo, bx.hi);                      // B = A + dt * src on the working box
        k_saxpy_box<<<(unsigned)((r.n + 255) / 256), 256, 0, st>>>(r, a->P->A.fab(), a->P->src.fab(), a->P->Bs.fab(),
                                                                     Dims<NS>::NVAR, dt);
    }
    copy(a->P->Cs, a->P->Bs, st);
    clean(bx, a->P->Cs);                                          // clean_state(S_new), Castro_advance.cpp
}

__global__ void k_copy_box(BoxRange r, Fab D, Fab S, int nv)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= r.n) return;
    const int i = r.lx + (int)(t % r.nx);
    const long long t2 = t / r.nx;
    const int j = r.ly + (int)(t2 % r.ny);
    const int k = r.lz + (int)(t2 / r.ny);
    for (int n = 0; n < nv; ++n) D(i, j, k, n) = S(i, j, k, n);
}

// V_{n+1} = clean(C) on the working box of the domain-sized Vout
void finish_step(castro_adj* a, const Arr& Vout)
{
    BoxRange r = make_range(a->bx.lo, a->bx.hi);
    k_copy_box<<<(unsigned)((r.n + 255) / 256), 256, 0, a->st>>>(r, Vout.fab(), a->P->Cs.fab(), a->nv);
    clean(a->bx, Vout);                                        // post_timestep clean_state, Castro.cpp:369
}

// estTimeStep on V: returns min over zones of estdt (before the CFL factor)
double est_min(castro_adj* a, const Arr& V)
{
    double big = 1.79769313486231570e+308;
    cudaMemcpyAsync(a->d_est, &big, sizeof big, cudaMemcpyHostToDevice, a->st);
    estdt(a->dom.lo, a->dom.hi, V.p, V.b.lo, V.b.hi, a->dx, a->d_est);
    double v;
    cudaMemcpyAsync(&v, a->d_est, sizeof v, cudaMemcpyDeviceToHost, a->st);
    cudaStreamSynchronize(a->st);
    return v;
}

// objective: kinetic energy in the shell r0 <= r/L <= r1 about the domain centre
template <int NS>
double objective(castro_adj* a, const Arr& V, bool grad, const Arr& Vb)
{
    cudaMemsetAsync(a->d_scal, 0, sizeof(double), a->st);
    Fab U = V.fab(), UB = Vb.fab();
    const double pl0 = a->problo[0], pl1 = a->problo[1], pl2 = a->problo[2];
    const double dx0 = a->dx[0], dx1 = a->dx[1], dx2 = a->dx[2];
    const double c0 = 0.5 * (a->problo[0] + a->probhi[0]), c1 = 0.5 * (a->problo[1] + a->probhi[1]),
                 c2 = 0.5 * (a->problo[2] + a->probhi[2]);
    const double L = a->probhi[0] - a->problo[0];
    const double r0 = a->shell_r0 * L, r1 = a->shell_r1 * L, dV = dx0 * dx1 * dx2;
    launch_sum("adj objective", a->dom.lo, a->dom.hi, [=] __device__(int i, int j, int k) -> double {
        const double x = pl0 + (i + 0.5) * dx0 - c0, y = pl1 + (j + 0.5) * dx1 - c1, z = pl2 + (k + 0.5) * dx2 - c2;
        const double r = sqrt(x * x + y * y + z * z);
        if (r < r0 || r > r1) return 0.0;
        const double rho = U(i, j, k, URHO), mx = U(i, j, k, UMX), my = U(i, j, k, UMY), mz = U(i, j, k, UMZ);
        const double m2 = mx * mx + my * my + mz * mz;
        if (grad) {
            UB(i, j, k, URHO) += -0.5 * m2 / (rho * rho) * dV;
            UB(i, j, k, UMX) += mx / rho * dV;
            UB(i, j, k, UMY) += my / rho * dV;
            UB(i, j, k, UMZ) += mz / rho * dV;
        }
        return 0.5 * m2 / rho * dV;
    }, a->d_scal);
    double J;
    cudaMemcpyAsync(&J, a->d_scal, sizeof J, cudaMemcpyDeviceToHost, a->st);
    cudaStreamSynchronize(a->st);
    return J;
}

// adjoint of the CFL estimate at its arg-min zone: Vb(m) += scale * d(estdt_m)/dV
template <int NS>
void estdt_adj(castro_adj* a, const Arr& V, double minval, const double* scale, const Arr& Vb)
{
    int big = 0x7fffffff;
    cudaMemcpyAsync(a->d_idx, &big, sizeof big, cudaMemcpyHostToDevice, a->st);
    Fab U = V.fab();
    const IBx bx = a->dom;
    const double dx0 = a->dx[0], dx1 = a->dx[1], dx2 = a->dx[2];
    int* idx = a->d_idx;
    const int nx = bx.hi[0] - bx.lo[0] + 1, ny = bx.hi[1] - bx.lo[1] + 1;
    launch_box("adj estdt argmin", bx.lo, bx.hi, [=] __device__(int i, int j, int k) {
        double u[Dims<NS>::NVAR];
#pragma unroll
        for (int n = 0; n < Dims<NS>::NVAR; ++n) u[n] = U(i, j, k, n);
        if (estdt_pt<NS, false>(u, dx0, dx1, dx2) == minval)   // (the adjoint runs without Coulomb corrections)
            atomicMin(idx, (i - bx.lo[0]) + nx * ((j - bx.lo[1]) + ny * (k - bx.lo[2])));
    });
    Fab UB = Vb.fab();
    const int one[3] = {0, 0, 0};
    launch_box<32>("adj estdt", one, one, [=] __device__(int, int, int) {
        int m = *idx;
        const double sc_ = *scale;
        if (m == 0x7fffffff || sc_ == 0.0) return;
        int i = bx.lo[0] + m % nx, j = bx.lo[1] + (m / nx) % ny, k = bx.lo[2] + m / (nx * ny);
        double u[Dims<NS>::NVAR], ub[Dims<NS>::NVAR];
        for (int n = 0; n < Dims<NS>::NVAR; ++n) { u[n] = U(i, j, k, n); ub[n] = 0.0; }
        const double dxs[3] = {dx0, dx1, dx2};
        estdt_pt_adj<NS>(c_eos, c_net, u, dxs, sc_, ub);
        for (int n = 0; n < Dims<NS>::NVAR; ++n) UB(i, j, k, n) += ub[n];
    });
}

// ---- zone-based transverse reverses (no atomics on flux records) -----------
__host__ __device__ inline bool in_box(const IBx& b, int i, int j, int k)
{
    return i >= b.lo[0] && i <= b.hi[0] && j >= b.lo[1] && j <= b.hi[1] && k >= b.lo[2] && k <= b.hi[2];
}

template <int NS>
__device__ __forceinline__ void st_rec(const Fab& F, int i, int j, int k, const double* r)
{
#pragma unroll
    for (int n = 0; n < Dims<NS>::NTF; ++n) F(i, j, k, n) = r[n];
}

// trans1 (flux direction d corrects the states normal to t) over the zones
// that feed its face box fb = tbx[t][d]: zone z owns the minus state of face
// z+e_t and the plus state of face z, and both use the flux records of faces
// z and z+e_d; their adjoints go to L[z] and R[z]
template <int NS>
void trans1_adj_zones(castro_adj* a, int d, int t, double cdtdx, double* cdtdxb)
{
    const Prim& P = *a->P;
    const IBx fb = a->tbx[t][d];
    IBx zb = fb;
    zb.lo[t] -= 1;
    Fab Q2M = P.qm[t][t].fab(), Q2P = P.qp[t][t].fab(), QA = P.qaux.fab(), F1 = P.F1[d].fab(), Q1 = P.G1[d].fab();
    Fab MOB = a->qmb[t][d].fab(), POB = a->qpb[t][d].fab(), MB = a->qmb[t][t].fab(), PB = a->qpb[t][t].fab();
    Fab QAB = a->qab.fab(), LF = a->T1L[d][t].fab(), RF = a->T1R[d][t].fab();
    launch_sum<CASTRO_ADJ_MINB_TRANS1>("trans1_adj zones", zb.lo, zb.hi, [=] __device__(int i, int j, int k) -> double {
        constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF;
        const int etx = t == 0, ety = t == 1, etz = t == 2;
        const int edx = d == 0, edy = d == 1, edz = d == 2;
        double fr[NTF], fl[NTF], frb[NTF], flb[NTF];
        ld_tflux<NS>(F1, Q1, i + edx, j + edy, k + edz, d, fr);
        ld_tflux<NS>(F1, Q1, i, j, k, d, fl);
#pragma unroll
        for (int n = 0; n < NTF; ++n) { frb[n] = 0.0; flb[n] = 0.0; }
        const double gamc = QA(i, j, k, QGAMC);
        double gb = 0.0, cb = 0.0;
        double lq[NQS], lqob[NQS], lqb[NQS];
        if (in_box(fb, i + etx, j + ety, k + etz)) {   // minus state of face z+e_t
            ld_state<NS>(Q2M, i + etx, j + ety, k + etz, lq);
            ld_state<NS>(MOB, i + etx, j + ety, k + etz, lqob);
#pragma unroll
            for (int n = 0; n < NQS; ++n) lqb[n] = 0.0;
            trans1_state_adj<NS>(lq, fr, fl, gamc, cdtdx, lqob, lqb, frb, flb, gb, cb);
            add_state<NS>(MB, i + etx, j + ety, k + etz, lqb);
        }
        if (in_box(fb, i, j, k)) {                       // plus state of face z
            ld_state<NS>(Q2P, i, j, k, lq);
            ld_state<NS>(POB, i, j, k, lqob);
#pragma unroll
            for (int n = 0; n < NQS; ++n) lqb[n] = 0.0;
            trans1_state_adj<NS>(lq, fr, fl, gamc, cdtdx, lqob, lqb, frb, flb, gb, cb);
            add_state<NS>(PB, i, j, k, lqb);
        }
        st_rec<NS>(RF, i, j, k, frb);
        st_rec<NS>(LF, i, j, k, flb);
        QAB(i, j, k, QGAMC) += gb;
        return cb;
    }, cdtdxb);
}

// trans2 of direction d over the zones feeding ebx[d]: zone z owns the minus
// state of face z+e_d and the plus state of face z; records of the t1 fluxes
// (faces z, z+e_t1) go to T2L/T2R[d][0], of the t2 fluxes to [d][1]
template <int NS>
void trans2_adj_zones(castro_adj* a, int d, double c2, double c3, double* c2b, double* c3b)
{
    const Prim& P = *a->P;
    const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
    const IBx fb = a->ebx[d];
    IBx zb = fb;
    zb.lo[d] -= 1;
    Fab QM = P.qm[d][d].fab(), QP = P.qp[d][d].fab(), QA = P.qaux.fab();
    Fab F2 = P.F2[t1][t2].fab(), G2 = P.G2[t1][t2].fab(), F3 = P.F2[t2][t1].fab(), G3 = P.G2[t2][t1].fab();
    Fab MOB = a->qlb[d].fab(), POB = a->qrb[d].fab(), MB = a->qmb[d][d].fab(), PB = a->qpb[d][d].fab();
    Fab QAB = a->qab.fab(), L2 = a->T2L[d][0].fab(), R2 = a->T2R[d][0].fab(), L3 = a->T2L[d][1].fab(),
        R3 = a->T2R[d][1].fab();
    launch_sum2<CASTRO_ADJ_MINB_TRANS2>("trans2_adj zones", zb.lo, zb.hi, [=] __device__(int i, int j, int k) -> double2 {
        constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF;
        const int e1x = d == 0, e1y = d == 1, e1z = d == 2;
        const int e2x = t1 == 0, e2y = t1 == 1, e2z = t1 == 2;
        const int e3x = t2 == 0, e3y = t2 == 1, e3z = t2 == 2;
        double f2r[NTF], f2l[NTF], f3r[NTF], f3l[NTF], f2rb[NTF], f2lb[NTF], f3rb[NTF], f3lb[NTF];
        ld_tflux<NS>(F2, G2, i + e2x, j + e2y, k + e2z, t1, f2r);
        ld_tflux<NS>(F2, G2, i, j, k, t1, f2l);
        ld_tflux<NS>(F3, G3, i + e3x, j + e3y, k + e3z, t2, f3r);
        ld_tflux<NS>(F3, G3, i, j, k, t2, f3l);
#pragma unroll
        for (int n = 0; n < NTF; ++n) { f2rb[n] = 0.0; f2lb[n] = 0.0; f3rb[n] = 0.0; f3lb[n] = 0.0; }
        const double gamc = QA(i, j, k, QGAMC);
        double gb = 0.0, cb2 = 0.0, cb3 = 0.0;
        double lq[NQS], lqob[NQS], lqb[NQS];
        if (in_box(fb, i + e1x, j + e1y, k + e1z)) {     // minus state of face z+e_d
            ld_state<NS>(QM, i + e1x, j + e1y, k + e1z, lq);
            ld_state<NS>(MOB, i + e1x, j + e1y, k + e1z, lqob);
#pragma unroll
            for (int n = 0; n < NQS; ++n) lqb[n] = 0.0;
            trans2_state_adj<NS>(lq, f2r, f2l, f3r, f3l, gamc, c2, c3, lqob, lqb, f2rb, f2lb, f3rb, f3lb, gb, cb2, cb3);
            add_state<NS>(MB, i + e1x, j + e1y, k + e1z, lqb);
        }
        if (in_box(fb, i, j, k)) {                       // plus state of face z
            ld_state<NS>(QP, i, j, k, lq);
            ld_state<NS>(POB, i, j, k, lqob);
#pragma unroll
            for (int n = 0; n < NQS; ++n) lqb[n] = 0.0;
            trans2_state_adj<NS>(lq, f2r, f2l, f3r, f3l, gamc, c2, c3, lqob, lqb, f2rb, f2lb, f3rb, f3lb, gb, cb2, cb3);
            add_state<NS>(PB, i, j, k, lqb);
        }
        st_rec<NS>(R2, i, j, k, f2rb);
        st_rec<NS>(L2, i, j, k, f2lb);
        st_rec<NS>(R3, i, j, k, f3rb);
        st_rec<NS>(L3, i, j, k, f3lb);
        QAB(i, j, k, QGAMC) += gb;
        return make_double2(cb2, cb3);
    }, c2b, c3b);
}

// flux / qgdnv adjoints of the faces fb of direction n from up to two pairs of
// zone records: sum over pairs of L[g] + R[g - e_n] (zones inside zb)
template <int NS>
void gather_records(const IBx& fb, int n, const IBx& zb0, Fab L0, Fab R0, bool two, const IBx& zb1, Fab L1, Fab R1,
                    Fab FB, Fab GB)
{
    launch_box("adjoint record gather", fb.lo, fb.hi, [=] __device__(int i, int j, int k) {
        using R = TF<NS>;
        constexpr int NTF = Dims<NS>::NTF;
        const int ex = n == 0, ey = n == 1, ez = n == 2;
        double r[NTF];
#pragma unroll
        for (int m = 0; m < NTF; ++m) r[m] = 0.0;
        if (in_box(zb0, i, j, k))
#pragma unroll
            for (int m = 0; m < NTF; ++m) r[m] += L0(i, j, k, m);
        if (in_box(zb0, i - ex, j - ey, k - ez))
#pragma unroll
            for (int m = 0; m < NTF; ++m) r[m] += R0(i - ex, j - ey, k - ez, m);
        if (two) {
            if (in_box(zb1, i, j, k))
#pragma unroll
                for (int m = 0; m < NTF; ++m) r[m] += L1(i, j, k, m);
            if (in_box(zb1, i - ex, j - ey, k - ez))
#pragma unroll
                for (int m = 0; m < NTF; ++m) r[m] += R1(i - ex, j - ey, k - ez, m);
        }
        FB(i, j, k, URHO) = r[R::RHO];
        FB(i, j, k, UMX) = r[R::MX];
        FB(i, j, k, UMY) = r[R::MY];
        FB(i, j, k, UMZ) = r[R::MZ];
        FB(i, j, k, UEDEN) = r[R::ED];
#pragma unroll
        for (int m = 0; m < NS; ++m) FB(i, j, k, UFS + m) = r[R::X + m];
        GB(i, j, k, GDPRES) = r[R::PG];
        GB(i, j, k, GDU + n) = r[R::UG];
    });
}

// reverse of one step: a->Vb holds the adjoint of V_{n+1} on entry and of V_n
// on exit; slots 0..9 of a->d_scal receive the adjoint of dt_n from this
// step's uses of it
// the reverse of one step begins: the domain's S_old adjoint and the scalar
// accumulators (every working box adds to them)
void reverse_begin(castro_adj* a)
{
    zero(a->Ab, a->st);
    cudaMemsetAsync(a->d_scal, 0, 32 * sizeof(double), a->st);
}

// the reverse of one step on the working box, seeded by the adjoint of
// V_{n+1} on that box (Vb), with the forward intermediates of the same box
template <int NS>
void reverse_step(castro_adj* a, double dt)
{
    cudaStream_t st = a->st;
    const IBx &bx = a->bx, &obx = a->obx, &qbx = a->qbx;
    for (Arr* r : {&a->Sbb, &a->qb, &a->qab, &a->divb, &a->srcb}) zero(*r, st);
    for (int d = 0; d < 3; ++d) {
        // F1b/G1b/F2b/G2b need no zeroing: the record gathers write every face
        // the Riemann adjoints read (the other components stay zero from creation)
        // qlb/qrb and the cross face states qmb/qpb[a][b] (a != b) are stored, not
        // accumulated, by their first writer (the riemann3 / riemann2 adjoints)
        // on exactly the faces their readers use
        for (Arr* r : {&a->fluxb[d], &a->qeb[d]}) zero(*r, st);
        zero(a->qmb[d][d], st);
        zero(a->qpb[d][d], st);
    }
    double* sc = a->d_scal;
    adj_mark(a, "zero adjoint arrays");
    // V_{n+1} = clean(C), C = clean(B)
    clean_state_adj_impl<NS>(bx.lo, bx.hi, a->P->Cs.fab(), a->Vb.fab(), true);
    clean_state_adj_impl<NS>(bx.lo, bx.hi, a->P->Bs.fab(), a->Vb.fab(), true);
    adj_stage(a, "end cleans");
    // B = A + dt*src: Ab += Bb (other working boxes' Sborder adjoints may be
    // there already), srcb = dt*Bb, dtb += sum(src*Bb)
    {
        Fab BB = a->Vb.fab(), AB = a->Ab.fab(), SB = a->srcb.fab(), S = a->P->src.fab();
        launch_sum("adj saxpy", bx.lo, bx.hi, [=] __device__(int i, int j, int k) -> double {
            double s = 0.0;
#pragma unroll
            for (int n = 0; n < Dims<NS>::NVAR; ++n) {
                double b = BB(i, j, k, n);
                AB(i, j, k, n) += b;
                SB(i, j, k, n) = dt * b;
                s += S(i, j, k, n) * b;
            }
            return s;
        }, sc + 9);
    }
    adj_stage(a, "saxpy");
    fill_hydro_source_adj_impl<NS>(bx.lo, bx.hi, a->srcb.fab(), a->P->qe[0].fab(), a->P->qe[1].fab(), a->P->qe[2].fab(),
                                   a->area[0].fab(), a->area[1].fab(), a->area[2].fab(), a->vol.fab(), a->dx[0],
                                   a->dx[1], a->dx[2], a->fluxb[0].fab(), a->fluxb[1].fab(), a->fluxb[2].fab(),
                                   a->qeb[0].fab(), a->qeb[1].fab(), a->qeb[2].fab());
    adj_stage(a, "fill_hydro_source");
    for (int d = 0; d < 3; ++d) {
        normalize_species_fluxes_adj_impl<NS>(a->ebx[d].lo, a->ebx[d].hi, a->P->Fav[d].fab(), a->fluxb[d].fab());
        apply_av_adj_impl<NS>(a->ebx[d].lo, a->ebx[d].hi, d, a->dx[d], a->P->div.fab(), a->P->Sb.fab(), a->fluxb[d].fab(),
                              a->divb.fab(), a->Sbb.fab());
        compute_flux_adj_impl<NS>(a->ebx[d].lo, a->ebx[d].hi, a->P->ql[d].fab(), a->P->qr[d].fab(), a->P->qaux.fab(),
                                  a->fluxb[d].fab(), a->qeb[d].fab(), a->qlb[d].fab(), a->qrb[d].fab(), a->qab.fab(), d,
                                  true);
    }
    adj_stage(a, "normalize/av/riemann3");
    double hdtdx[3], cdtdx[3];
    for (int d = 0; d < 3; ++d) { hdtdx[d] = 0.5 * dt / a->dx[d]; cdtdx[d] = dt / a->dx[d] / 3.0; }
    for (int d = 0; d < 3; ++d) {
        int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
        trans2_adj_zones<NS>(a, d, hdtdx[t1], hdtdx[t2], sc + 6 + t1, sc + 6 + t2);
        IBx zb = a->ebx[d];
        zb.lo[d] -= 1;
        gather_records<NS>(a->tbx[t1][t2], t1, zb, a->T2L[d][0].fab(), a->T2R[d][0].fab(), false, zb,
                           a->T2L[d][0].fab(), a->T2R[d][0].fab(), a->F2b[t1][t2].fab(), a->G2b[t1][t2].fab());
        gather_records<NS>(a->tbx[t2][t1], t2, zb, a->T2L[d][1].fab(), a->T2R[d][1].fab(), false, zb,
                           a->T2L[d][1].fab(), a->T2R[d][1].fab(), a->F2b[t2][t1].fab(), a->G2b[t2][t1].fab());
    }
    adj_stage(a, "trans2");
    for (int x = 0; x < 3; ++x)
        for (int y = 0; y < 3; ++y) {
            if (x == y) continue;
            compute_flux_adj_impl<NS>(a->tbx[x][y].lo, a->tbx[x][y].hi, a->P->qm[x][y].fab(), a->P->qp[x][y].fab(),
                                      a->P->qaux.fab(), a->F2b[x][y].fab(), a->G2b[x][y].fab(), a->qmb[x][y].fab(),
                                      a->qpb[x][y].fab(), a->qab.fab(), x, true);
        }
    adj_stage(a, "riemann2");
    for (int d = 0; d < 3; ++d) {
        const int ta = d == 0 ? 1 : 0, tb = d == 2 ? 1 : 2;
        trans1_adj_zones<NS>(a, d, ta, cdtdx[d], sc + 3 + d);
        trans1_adj_zones<NS>(a, d, tb, cdtdx[d], sc + 3 + d);
        IBx za = a->tbx[ta][d], zbb = a->tbx[tb][d];
        za.lo[ta] -= 1;
        zbb.lo[tb] -= 1;
        gather_records<NS>(a->tbx[d][d], d, za, a->T1L[d][ta].fab(), a->T1R[d][ta].fab(), true, zbb,
                           a->T1L[d][tb].fab(), a->T1R[d][tb].fab(), a->F1b[d].fab(), a->G1b[d].fab());
    }
    adj_stage(a, "trans1");
    for (int d = 0; d < 3; ++d)
        compute_flux_adj_impl<NS>(a->tbx[d][d].lo, a->tbx[d][d].hi, a->P->qm[d][d].fab(), a->P->qp[d][d].fab(),
                                  a->P->qaux.fab(), a->F1b[d].fab(), a->G1b[d].fab(), a->qmb[d][d].fab(),
                                  a->qpb[d][d].fab(), a->qab.fab(), d);
    adj_stage(a, "riemann1");
    for (int d = 0; d < 3; ++d)
        trace_adj_impl<NS>(obx.lo, obx.hi, bx.lo, bx.hi, d, a->P->q.fab(), a->P->qaux.fab(), a->qmb[d][d].fab(),
                           a->qpb[d][d].fab(), a->qb.fab(), a->qab.fab(), dt / a->dx[d], sc + d, a->flb.fab());
    uflatten_adj_zones<NS>(obx.lo, obx.hi, a->P->q.fab(), a->P->qaux.fab(), a->qb.fab(), a->qab.fab(), a->flb.fab());
    adj_stage(a, "trace");
    divu_adj_impl<NS>(obx.lo, obx.hi, a->divb.fab(), a->qb.fab(), a->dx[0], a->dx[1], a->dx[2]);
    adj_stage(a, "divu");
    ctoprim_adj_impl<NS>(qbx.lo, qbx.hi, a->P->Sb.fab(), a->qb.fab(), a->qab.fab(), a->Sbb.fab());
    adj_stage(a, "ctoprim");
    fill_clean_adj<NS>(a);
    adj_stage(a, "sborder fill+clean");
}

// the reverse of one step ends: clean_state(S_old) of the domain reversed, and
// the adjoint of V_n replaces that of V_{n+1}
template <int NS>
void reverse_end(castro_adj* a, const Arr& Vn)
{
    clean_state_adj_impl<NS>(a->dom.lo, a->dom.hi, Vn.fab(), a->Ab.fab(), true);
    adj_stage(a, "start clean");
    copy(a->Vb, a->Ab, a->st);
}

// adjoint of dt_n: its uses in step n (slots 0..9 of sc), the growth-limit
// chain from later steps (chain[n]) and the time adjoint (chain[N]); then the
// rule that made dt_n: stop-time clamp (branch 1), 1.1x growth limit (2), or
// the CFL estimate (0: chain[N+1] = scale handed to estdt_adj)
__global__ void k_dt_chain(const double* sc, double dx0, double dx1, double dx2, double* chain, int n, int N,
                           int branch, double fac)
{
    const double dx[3] = {dx0, dx1, dx2};
    double dtb = sc[9];
    for (int d = 0; d < 3; ++d) dtb += sc[d] / dx[d] + sc[3 + d] / dx[d] / 3.0 + sc[6 + d] * 0.5 / dx[d];
    dtb += chain[n] + chain[N];
    chain[N + 1] = 0.0;
    if (branch == 1) chain[N] -= dtb;
    else if (branch == 2) chain[n - 1] += 1.1e0 * dtb;
    else chain[N + 1] = fac * dtb;
}

template <int NS>
int adj_forward(castro_adj* a)
{
    StreamScope ss(a->st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, a->st);
    a->P = &a->sets[0];
    castro_problem saved = castro::problem();
    castro_set_problem(&a->prob);
    initdata(a->dom.lo, a->dom.hi, a->V.p, a->dom.lo, a->dom.hi, a->dx, a->problo, a->probhi);
    castro_set_problem(&saved);
    const int N = a->nsteps;
    a->dts.assign(N, 0.0); a->times.assign(N + 1, 0.0); a->ests.assign(N, 0.0); a->estmin.assign(N, 0.0);
    a->limited.assign(N, 0); a->clamped.assign(N, 0);
    double time = 0.0, dt_prev = 0.0;
    // checkpoints from the window's first step on; the last checkpoint segment
    // keeps its states and intermediates, so the reverse sweep starts without
    // recomputing it
    const int K = a->ckpt, S0 = a->n_start;
    const int n0_last = S0 + ((N - 1 - S0) / K) * K;
    const bool keep_last = (int)a->sets.size() >= K;
    for (int n = 0; n < N; ++n) {
        if (n >= S0 && (n - S0) % K == 0) copy(a->ckpts[(n - S0) / K], a->V, a->st);
        if (keep_last && n >= n0_last) {
            a->P = &a->sets[n - n0_last];
            copy(a->seg[n - n0_last], a->V, a->st);
        }
        // computeNewDt / computeInitialDt, Source/Castro.cpp:162-341
        double m = est_min(a, a->V);
        double est = m * cfl;
        double dt;
        if (n == 0) dt = std::min(1.0e+100, 0.01 * est);
        else {
            double dt_min = std::min(est, 1.1e0 * dt_prev);
            a->limited[n] = (1.1e0 * dt_prev < est) ? 1 : 0;
            dt = std::min(1.0e+100, dt_min);
        }
        double eps = 0.001 * dt;
        if (a->stop_time >= 0.0 && (time + dt) > (a->stop_time - eps)) {
            dt = a->stop_time - time;
            a->clamped[n] = 1;
        }
        a->estmin[n] = m;
        a->ests[n] = est;
        a->dts[n] = dt;
        a->times[n] = time;
        begin_step(a, a->V);
        for (int sl = 0; sl < (int)a->slabs.size(); ++sl) {   // V is rewritten box by box; the boxes read P->A
            use_slab(a, sl);
            forward_step<NS>(a, dt);
            finish_step(a, a->V);
        }
        time += dt;
        dt_prev = dt;
    }
    a->times[N] = time;
    a->last_seg_ready = keep_last;
    copy(a->Vfinal, a->V, a->st);
    a->J = objective<NS>(a, a->V, false, a->Vb);
    cudaEventRecord(e1, a->st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&a->ms_forward, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    a->fwd_done = true;
    return check_launch("castro_adj_forward") ? CASTRO_OK : CASTRO_ERR_CUDA;
}

// reverse of initdata (Source/Prob.F90:19-129) for the configs' ambient-from-T
// setup: dJ/dE, dJ/drho_ambient and (into pertb, if given) dJ/dpert
template <int NS>
void initdata_adj(castro_adj* a, double* dE, double* drho, double* pertb)
{
    const castro_problem P = a->prob;
    cudaMemsetAsync(a->d_scal, 0, 32 * sizeof(double), a->st);
    double* sc = a->d_scal;
    // ambient e and its density derivative
    SpeciesXAdj xs;
    for (int n = 0; n < MAX_SPEC; ++n) xs.x[n] = P.X[n];
    const int from_T = P.ambient_from_T;
    const double rho_a = P.dens_ambient, p_a = P.p_ambient, T_a = P.T_ambient;
    const int one[3] = {0, 0, 0};
    launch_box<32>("initdata_adj(ambient)", one, one, [=] __device__(int, int, int) {
        EosOutT<double> r;
        double e, de_drho;
        if (from_T) {
            double s1 = 0.0, s2 = 0.0;
            for (int n = 0; n < NS; ++n) s1 = s1 + xs.x[n] * c_net.aion_inv[n];
            for (int n = 0; n < NS; ++n) s2 = s2 + xs.x[n] * c_net.zion[n] * c_net.aion_inv[n];
            double abar = 1.0 / s1, zbar = abar * s2;
            eos_solve_t<EOS_RT>(c_eos, rho_a, T_a, 0.0, abar, zbar, r);
            e = r.e;
            EosBar ob{0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0};
            double rb = 0.0, Tb = 0.0, ab = 0.0, zb = 0.0;
            eos_vjp<EOS_RT>(c_eos, rho_a, T_a, abar, zbar, ob, rb, Tb, ab, zb);
            de_drho = rb;
        } else {
            // T from p(rho, T) = p_a; e(rho, T(rho))
            double abar = c_net.aion[0], zbar = c_net.zion[0];
            double T = eos_solve_t<EOS_RP>(c_eos, rho_a, 1.e4, p_a, abar, zbar, r);
            e = r.e;
            EosOutT<D4> o;
            eos_eval_t<D4>(c_eos, d4seed(T, 1), d4seed(rho_a, 0), D4(1.0 / abar), D4(zbar / abar), o);
            de_drho = o.e.d[0] - o.e.d[1] * o.p.d[0] / o.p.d[1];
        }
        sc[20] = e;
        sc[21] = de_drho;
    });
    const double r_init = P.r_init;
    const double vctr = (4.0 / 3.0) * 3.14159265358979323846 * (r_init * r_init * r_init);
    const double e_exp = P.exp_energy / vctr / P.dens_ambient;
    const double c0 = (a->problo[0] + a->probhi[0]) / 2.e0, c1 = (a->problo[1] + a->probhi[1]) / 2.e0,
                 c2 = (a->problo[2] + a->probhi[2]) / 2.e0;
    const double pl0 = a->problo[0], pl1 = a->problo[1], pl2 = a->problo[2];
    const double dx0 = a->dx[0], dx1 = a->dx[1], dx2 = a->dx[2];
    const int nsub = P.nsub;
    const double pert_amp = P.pert_amp;
    Fab PERT{}, PB{};
    const bool has_pert = P.pert != nullptr;
    if (has_pert) {
        PERT = make_fab(P.pert, P.pert_lo, P.pert_hi);
        if (pertb) PB = make_fab(pertb, P.pert_lo, P.pert_hi);
    }
    const bool want_pb = has_pert && pertb;
    Fab UB = a->Vb.fab();
    launch_box("initdata_adj", a->dom.lo, a->dom.hi, [=] __device__(int i, int j, int k) {
        const double e_ambient = sc[20];
        double xmin = pl0 + dx0 * (double)i, ymin = pl1 + dx1 * (double)j, zmin = pl2 + dx2 * (double)k;
        int npert = 0, nambient = 0;
        for (int kk = 0; kk < nsub; ++kk) {
            double zz = zmin + (dx2 / (double)nsub) * (kk + 0.5e0);
            for (int jj = 0; jj < nsub; ++jj) {
                double yy = ymin + (dx1 / (double)nsub) * (jj + 0.5e0);
                for (int ii = 0; ii < nsub; ++ii) {
                    double xx = xmin + (dx0 / (double)nsub) * (ii + 0.5e0);
                    double dist = (c0 - xx) * (c0 - xx) + (c1 - yy) * (c1 - yy) + (c2 - zz) * (c2 - zz);
                    if (dist <= r_init * r_init) npert = npert + 1;
                    else nambient = nambient + 1;
                }
            }
        }
        const double nsub3 = (double)(nsub * nsub * nsub);
        const double eint = ((double)npert * e_exp + (double)nambient * e_ambient) / nsub3;
        const double g = has_pert ? (1.0 + pert_amp * PERT(i, j, k, 0)) : 1.0;
        const double rho = rho_a * g;
        double rhob = UB(i, j, k, URHO) + (UB(i, j, k, UEDEN) + UB(i, j, k, UEINT)) * eint;
        for (int n = 0; n < NS; ++n) rhob += UB(i, j, k, UFS + n) * xs.x[n];
        const double eintb = (UB(i, j, k, UEDEN) + UB(i, j, k, UEINT)) * rho;
        if (want_pb) PB(i, j, k, 0) += rhob * rho_a * pert_amp;
        aadd(&sc[0], eintb * (double)npert / nsub3);     // d/d e_exp
        aadd(&sc[1], eintb * (double)nambient / nsub3);  // d/d e_ambient
        aadd(&sc[2], rhob * g);                          // d/d rho_a through rho
    });
    double h[32];
    cudaMemcpyAsync(h, sc, 32 * sizeof(double), cudaMemcpyDeviceToHost, a->st);
    cudaStreamSynchronize(a->st);
    // e_exp = E / vctr / rho_a
    *dE = h[0] / vctr / P.dens_ambient;
    *drho = h[2] - h[0] * e_exp / P.dens_ambient + h[1] * h[21];
}

template <int NS>
int adj_backward(castro_adj* a, double* dE, double* drho, double* pertb)
{
    if (!a->fwd_done) { set_error(CASTRO_ERR_ARG, "castro_adj_backward: run castro_adj_forward first"); return CASTRO_ERR_ARG; }
    StreamScope ss(a->st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, a->st);
    const int N = a->nsteps, K = a->ckpt, S0 = a->n_start;
    const int nsl = (int)a->slabs.size();
    zero(a->Vb, a->st);
    objective<NS>(a, a->Vfinal, true, a->Vb);
    // chain[0..N-1]: adjoint of dt_n from the growth limit of later steps;
    // chain[N]: adjoint of the running time (stop-time clamp); chain[N+1]: scale
    cudaMemsetAsync(a->d_chain, 0, (N + 2) * sizeof(double), a->st);
    const int nseg = (N - S0 + K - 1) / K;
    for (int sgi = nseg - 1; sgi >= 0; --sgi) {
        const int n0 = S0 + sgi * K, n1 = std::min(N, n0 + K);
        adj_mark(a, "(segment start)");
        const bool keep = (int)a->sets.size() >= K;
        const bool ready = keep && a->last_seg_ready && sgi == nseg - 1;
        if (!ready) copy(a->seg[0], a->ckpts[sgi], a->st);
        for (int n = n0; n < (ready ? n0 : n1 - (keep ? 0 : 1)); ++n) {
            a->P = &a->sets[keep ? n - n0 : 0];
            begin_step(a, a->seg[n - n0]);
            for (int sl = 0; sl < nsl; ++sl) {
                use_slab(a, sl);
                forward_step<NS>(a, a->dts[n]);
                if (n < n1 - 1) finish_step(a, a->seg[n - n0 + 1]);
            }
        }
        adj_mark(a, "segment recompute");
        for (int n = n1 - 1; n >= n0; --n) {
            if (keep) {
                // the whole domain is the working box and the set holds its intermediates
                a->P = &a->sets[n - n0];
                reverse_begin(a);
                reverse_step<NS>(a, a->dts[n]);
            } else {
                // every working box: its intermediates recomputed, then reversed
                a->P = &a->sets[0];
                begin_step(a, a->seg[n - n0]);
                reverse_begin(a);
                for (int sl = 0; sl < nsl; ++sl) {
                    use_slab(a, sl);
                    forward_step<NS>(a, a->dts[n]);
                    adj_mark(a, "step recompute");
                    reverse_step<NS>(a, a->dts[n]);
                }
            }
            reverse_end<NS>(a, a->seg[n - n0]);
            // dt_n = rule(V_n, dt_{n-1}, time_n), reversed on the device
            const int branch = a->clamped[n] ? 1 : (n > 0 && a->limited[n]) ? 2 : 0;
            k_dt_chain<<<1, 1, 0, a->st>>>(a->d_scal, a->dx[0], a->dx[1], a->dx[2], a->d_chain, n, N, branch,
                                           cfl * (n == 0 ? 0.01 : 1.0));
            if (branch == 0) estdt_adj<NS>(a, a->seg[n - n0], a->estmin[n], a->d_chain + N + 1, a->Vb);
            adj_mark(a, "dt adjoint");
        }
        adj_prof_flush();
    }
    // earlier segments reused the sets: a second reverse sweep recomputes
    a->last_seg_ready = a->last_seg_ready && nseg == 1;
    if (S0 == 0) {
        adj_mark(a, "(init start)");
        initdata_adj<NS>(a, dE, drho, pertb);
        adj_mark(a, "initdata adjoint");
    } else {
        // the window starts at a state, not at initdata: its adjoint is Vb
        // (castro_adj_initial_adjoint); the problem parameters get none
        *dE = 0.0;
        *drho = 0.0;
    }
    adj_prof_report();
    cudaEventRecord(e1, a->st);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&a->ms_backward, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return check_launch("castro_adj_backward") ? CASTRO_OK : CASTRO_ERR_CUDA;
}

}  // namespace

extern "C" {

castro_adj* castro_adj_create_window(const castro_instance_desc* desc, int nsteps, int checkpoint_interval,
                                     int slab_nz, int first_step)
{
    if (!desc || nsteps < 1 || checkpoint_interval < 1 || first_step < 0 || first_step >= nsteps || slab_nz < 0) {
        set_error(CASTRO_ERR_ARG, "castro_adj_create: arguments");
        return nullptr;
    }
    if (!table_ready()) { set_error(CASTRO_ERR_NO_TABLE, "castro_adj_create: eos_init has not run"); return nullptr; }
    if (coulomb_refused("castro_adj_create")) return nullptr;
    const int nz = desc->dom_hi[2] - desc->dom_lo[2] + 1;
    if (slab_nz > 0 && slab_nz < nz && nz % slab_nz != 0) {
        set_error(CASTRO_ERR_ARG, "castro_adj_create: the slab thickness must divide the domain's z extent");
        return nullptr;
    }
    castro_adj* a = new castro_adj();
    a->ns = nspec();
    a->nv = 7 + a->ns;
    a->qv = 8 + a->ns;
    for (int d = 0; d < 3; ++d) {
        a->dom.lo[d] = desc->dom_lo[d];
        a->dom.hi[d] = desc->dom_hi[d];
        a->problo[d] = desc->problo[d];
        a->probhi[d] = desc->probhi[d];
        a->dx[d] = (desc->probhi[d] - desc->problo[d]) / (double)(desc->dom_hi[d] - desc->dom_lo[d] + 1);
    }
    a->bc = desc->bc;
    a->prob = desc->prob;
    a->stop_time = desc->stop_time;
    a->nsteps = nsteps;
    a->ckpt = checkpoint_interval;
    a->n_start = first_step;
    const int tz = (slab_nz > 0 && slab_nz < nz) ? slab_nz : nz;
    for (int z0 = a->dom.lo[2]; z0 <= a->dom.hi[2]; z0 += tz) {
        IBx b = a->dom;
        b.lo[2] = z0;
        b.hi[2] = z0 + tz - 1;
        a->slabs.push_back(b);
    }
    set_geometry(a, a->slabs[0]);
    if (cudaStreamCreateWithFlags(&a->st, cudaStreamNonBlocking) != cudaSuccess) {
        set_error(CASTRO_ERR_CUDA, "castro_adj_create: stream");
        delete a;
        return nullptr;
    }
    const int NV = a->nv, QV = a->qv;
    bool ok = true;
    // slab-sized arrays move with the working box (use_slab)
    auto sa = [&](Arr& r, const IBx& b, int nc) {
        if (!ok) return false;
        ok = alloc_arr(a, r, b, nc);
        if (ok) a->slab_arrs.push_back(&r);
        return ok;
    };
    const int nck = (nsteps - first_step + checkpoint_interval - 1) / checkpoint_interval;
    a->ckpts.resize(nck);
    a->seg.resize(checkpoint_interval);
    for (auto& r : a->ckpts) ok = ok && alloc_arr(a, r, a->dom, NV);
    for (auto& r : a->seg) ok = ok && alloc_arr(a, r, a->dom, NV);
    for (Arr* r : {&a->V, &a->Vfinal, &a->Vb, &a->Ab}) ok = ok && alloc_arr(a, *r, a->dom, NV);
    sa(a->srcb, a->bx, NV);
    sa(a->vol, a->bx, 1);
    sa(a->Sbb, a->qbx, NV) && sa(a->qb, a->qbx, QV) && sa(a->qab, a->qbx, NQAUX);
    sa(a->divb, a->obx, 1) && sa(a->flb, a->obx, 1);
    for (int d = 0; d < 3 && ok; ++d) {
        for (int e = 0; e < 3 && ok; ++e) {
            sa(a->qmb[d][e], a->obx, QV) && sa(a->qpb[d][e], a->obx, QV);
            if (d != e) sa(a->F2b[d][e], a->obx, NV) && sa(a->G2b[d][e], a->obx, NGDNV);
        }
        sa(a->F1b[d], a->obx, NV) && sa(a->G1b[d], a->obx, NGDNV);
        sa(a->qlb[d], a->obx, QV) && sa(a->qrb[d], a->obx, QV);
        sa(a->fluxb[d], a->gebx[d], NV) && sa(a->qeb[d], a->gebx[d], NGDNV);
        sa(a->area[d], a->gebx[d], 1);
        for (int e = 0; e < 3 && ok; ++e)
            if (e != d) sa(a->T1L[d][e], a->obx, a->nv) && sa(a->T1R[d][e], a->obx, a->nv);
        for (int e = 0; e < 2 && ok; ++e)
            sa(a->T2L[d][e], a->obx, a->nv) && sa(a->T2R[d][e], a->obx, a->nv);
    }
    // per-step forward intermediates: a set per segment step when they fit in
    // 70% of the free device memory (the whole domain as one working box only),
    // else one set recomputed per step
    auto set_bytes = [&]() {
        long long n = 4 * nptsb(a->bx) * NV + nptsb(a->qbx) * (NV + QV + NQAUX) + nptsb(a->obx) * (1 + QV);
        n += nptsb(a->obx) * (18LL * QV + 3LL * (NV + NGDNV) + 6LL * (NV + NGDNV) + 6LL * QV);
        for (int d = 0; d < 3; ++d) n += nptsb(a->gebx[d]) * (2LL * NV + NGDNV);
        return (size_t)n * sizeof(double);
    };
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    int nsets = (ok && a->slabs.size() == 1 && (size_t)checkpoint_interval * set_bytes() < (size_t)(0.7 * (double)fr))
                    ? checkpoint_interval : 1;
    a->sets.resize(nsets);
    for (Prim& P : a->sets) {
        ok = ok && alloc_arr(a, P.A, a->dom, NV);     // the domain's cleaned S_old
        for (Arr* r : {&P.Bs, &P.Cs, &P.src}) sa(*r, a->bx, NV);
        sa(P.Sb, a->qbx, NV) && sa(P.q, a->qbx, QV) && sa(P.qaux, a->qbx, NQAUX);
        sa(P.div, a->obx, 1) && sa(P.qint, a->obx, QV);
        for (int d = 0; d < 3 && ok; ++d) {
            for (int e = 0; e < 3 && ok; ++e) {
                sa(P.qm[d][e], a->obx, QV) && sa(P.qp[d][e], a->obx, QV);
                if (d != e) sa(P.F2[d][e], a->obx, NV) && sa(P.G2[d][e], a->obx, NGDNV);
            }
            sa(P.F1[d], a->obx, NV) && sa(P.G1[d], a->obx, NGDNV);
            sa(P.ql[d], a->obx, QV) && sa(P.qr[d], a->obx, QV);
            sa(P.Fav[d], a->gebx[d], NV) && sa(P.flux[d], a->gebx[d], NV);
            sa(P.qe[d], a->gebx[d], NGDNV);
        }
    }
    a->P = &a->sets[0];
    ok = ok && cudaMalloc(&a->d_scal, 32 * sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&a->d_idx, sizeof(int)) == cudaSuccess;
    ok = ok && cudaMalloc(&a->d_est, sizeof(double)) == cudaSuccess;
    ok = ok && cudaMalloc(&a->d_chain, (nsteps + 2) * sizeof(double)) == cudaSuccess;
    if (!ok) {
        set_error(CASTRO_ERR_CUDA, "castro_adj_create: device allocation failed");
        castro_adj_destroy(a);
        return nullptr;
    }
    // components of the record-gather targets that no gather writes stay zero
    for (int d = 0; d < 3; ++d) {
        zero(a->F1b[d], a->st);
        zero(a->G1b[d], a->st);
        for (int e = 0; e < 3; ++e)
            if (e != d) { zero(a->F2b[d][e], a->st); zero(a->G2b[d][e], a->st); }
    }
    // zero every face array once: entries outside the forward's face boxes are never written
    for (Prim& P : a->sets) {
        for (int d = 0; d < 3; ++d) {
            for (int e = 0; e < 3; ++e) {
                zero(P.qm[d][e], a->st);
                zero(P.qp[d][e], a->st);
                if (d != e) { zero(P.F2[d][e], a->st); zero(P.G2[d][e], a->st); }
            }
            for (Arr* r : {&P.F1[d], &P.G1[d], &P.ql[d], &P.qr[d], &P.Fav[d], &P.flux[d], &P.qe[d]}) zero(*r, a->st);
        }
        zero(P.qint, a->st);
    }
    const double ar[3] = {a->dx[1] * a->dx[2], a->dx[0] * a->dx[2], a->dx[0] * a->dx[1]};
    for (int d = 0; d < 3; ++d) fill_const(a->area[d], ar[d], a->st);
    fill_const(a->vol, a->dx[0] * a->dx[1] * a->dx[2], a->st);
    cudaStreamSynchronize(a->st);
    if (!check_launch("castro_adj_create")) {
        castro_adj_destroy(a);
        return nullptr;
    }
    return a;
}

castro_adj* castro_adj_create(const castro_instance_desc* desc, int nsteps, int checkpoint_interval)
{
    return castro_adj_create_window(desc, nsteps, checkpoint_interval, 0, 0);
}

void castro_adj_destroy(castro_adj* a)
{
    if (!a) return;
    if (a->st) cudaStreamSynchronize(a->st);
    for (char* p : a->blocks) cudaFree(p);
    if (a->d_scal) cudaFree(a->d_scal);
    if (a->d_idx) cudaFree(a->d_idx);
    if (a->d_est) cudaFree(a->d_est);
    if (a->d_chain) cudaFree(a->d_chain);
    if (a->st) cudaStreamDestroy(a->st);
    delete a;
}

int castro_adj_set_problem(castro_adj* a, const castro_problem* p)
{
    if (!a || !p || p->nsub < 1 || !(p->dens_ambient > 0.0)) { set_error(CASTRO_ERR_ARG, "castro_adj_set_problem: arguments"); return CASTRO_ERR_ARG; }
    a->prob = *p;
    a->fwd_done = false;
    return CASTRO_OK;
}

int castro_adj_set_shell(castro_adj* a, double r0, double r1)
{
    if (!a || !(r0 >= 0.0) || !(r1 > r0)) { set_error(CASTRO_ERR_ARG, "castro_adj_set_shell: arguments"); return CASTRO_ERR_ARG; }
    a->shell_r0 = r0;
    a->shell_r1 = r1;
    return CASTRO_OK;
}

int castro_adj_forward(castro_adj* a, double* J)
{
    NvtxRange r("castro_adj_forward");
    if (!a) { set_error(CASTRO_ERR_ARG, "castro_adj_forward: null"); return CASTRO_ERR_ARG; }
    if (coulomb_refused("castro_adj_forward")) return CASTRO_ERR_ARG;
    int rc = CASTRO_ERR_NSPEC;
    if (a->ns == 2) rc = adj_forward<2>(a);
    else if (a->ns == 13) rc = adj_forward<13>(a);
    if (J) *J = a->J;
    return rc;
}

int castro_adj_backward(castro_adj* a, double* dJ_dE, double* dJ_drho, double* dJ_dpert)
{
    NvtxRange r("castro_adj_backward");
    if (!a || !dJ_dE || !dJ_drho) { set_error(CASTRO_ERR_ARG, "castro_adj_backward: arguments"); return CASTRO_ERR_ARG; }
    if (coulomb_refused("castro_adj_backward")) return CASTRO_ERR_ARG;
    if (a->ns == 2) return adj_backward<2>(a, dJ_dE, dJ_drho, dJ_dpert);
    if (a->ns == 13) return adj_backward<13>(a, dJ_dE, dJ_drho, dJ_dpert);
    return CASTRO_ERR_NSPEC;
}

double castro_adj_dt(const castro_adj* a, int step)
{
    if (!a || step < 0 || step >= (int)a->dts.size()) return -1.0;
    return a->dts[step];
}

int castro_adj_final_state(const castro_adj* a, double* dst)
{
    if (!a || !dst || !a->fwd_done) { set_error(CASTRO_ERR_ARG, "castro_adj_final_state: arguments"); return CASTRO_ERR_ARG; }
    cudaMemcpyAsync(dst, a->Vfinal.p, (size_t)a->Vfinal.n() * sizeof(double), cudaMemcpyDeviceToDevice, a->st);
    cudaStreamSynchronize(a->st);
    return CASTRO_OK;
}

int castro_adj_initial_adjoint(const castro_adj* a, double* dst)
{
    if (!a || !dst) { set_error(CASTRO_ERR_ARG, "castro_adj_initial_adjoint: arguments"); return CASTRO_ERR_ARG; }
    cudaMemcpyAsync(dst, a->Vb.p, (size_t)a->Vb.n() * sizeof(double), cudaMemcpyDeviceToDevice, a->st);
    cudaStreamSynchronize(a->st);
    return CASTRO_OK;
}

double castro_adj_time_ms(const castro_adj* a, int which)
{
    if (!a) return -1.0;
    return which == 0 ? a->ms_forward : a->ms_backward;
}

size_t castro_adj_device_bytes(const castro_adj* a)
{
    if (!a) return 0;
    size_t s = 0;
    for (const Arr& r : a->all) s += (size_t)r.n() * sizeof(double);
    return s;
}

}  // extern "C"
