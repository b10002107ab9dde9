// castro_sim.cu -- single-level Sedov simulations on one GPU.
//
// CASTRO_MODE_PLAIN replays the reference's host sequence box by box through
// the per-routine entry points (Castro::advance, Source/Castro_advance.cpp:12-100,
// with construct_hydro_source's 36 launches per box, Source/Castro_hydro.cpp:31-397).
//
// CASTRO_MODE_BATCHED advances every box of every instance with ten fused
// kernels per step, each walking a static work list of (box, region, chunk)
// items built once per BoxArray, and replays the step as one CUDA graph.
// front and update walk the boxes (the state U keeps the reference's per-box
// FABs); the stages in between walk each instance's domain as one region, so
// every face state and flux is formed once for the whole domain:
//
//   front   : clean_state(S_old) -> clean_state(Sborder) -> ctoprim   (per valid zone)
//   ghost   : the domain halo of Q / Sborder by the boundary condition (periodic or outflow)
//   prep    : divu at the nodes and uflatten per zone of grow(domain,1)
//   trace   : trace_ppm pass 1 (rho, u_D, p, rhoe, gamma_1)  | two parallel graph nodes,
//   trace2  : trace_ppm pass 2 (transverse u, species)       | segments of zones along x, y, z
//   riemann1: compute_flux on tbx[d][d]                                 (normal fluxes)
//   riemann2: trans1 + compute_flux on tbx[a][b], both b != a per face of tbx[a][a] (cross fluxes)
//   riemann3: trans2 + compute_flux + apply_av + normalize_species_fluxes on ebx[d]
//   update  : fill_hydro_source + Saxpy + clean_state x2 + estdt        (per valid zone)
//   dt      : computeNewDt (change_max 1.1, stop_time clamp) on the device
//
// Because clean_state, ctoprim and estdt are pointwise, a ghost zone's value
// equals its source zone's value bit for bit, so primitive variables are formed
// once per zone and stored once per instance (Q over grow(domain,4)), where the
// box halos read them in place.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <sys/stat.h>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "castro_common.cuh"
#include "../../include/castro_b200.h"

namespace castro {

void upload_constants_sim(const EosTableDev& e, const NetworkDev& n)
{
    cudaMemcpyToSymbol(c_eos, &e, sizeof e);
    cudaMemcpyToSymbol(c_net, &n, sizeof n);
}

const castro_problem& problem();
unsigned long long* eos_fail_counter();
bool column_tiles_on();
void apply_table_l2_window(cudaStream_t st);

namespace {

constexpr int NG = 4;   // ghost zones of Sborder, Source/Castro_advance.cpp:37
// Launch shape of the fused kernels.  castro_tuned.h (written by autotune.py
// from timings of the batched step on the target GPU) sets the block size
// (= the zones of one work item) and the minimum resident blocks per SM given
// to the register allocator per kernel group; 0 leaves it to the compiler.
// The values below are the defaults without a tuned header (hand sweep on
// B200: 4 blocks for the EOS kernels, whose spills stay in L1, and for trace,
// segments of 5 zones per trace thread).  Override with -DCASTRO_BLOCK /
// -DCASTRO_MINB_* / -DCASTRO_TRACE_SEG.
#if __has_include("castro_tuned.h")
#include "castro_tuned.h"
#endif
#ifndef CASTRO_BLOCK
#define CASTRO_BLOCK 128
#endif
#ifndef CASTRO_MINB_EOS
#define CASTRO_MINB_EOS 4
#endif
#ifndef CASTRO_MINB_R3
#define CASTRO_MINB_R3 0
#endif
#ifndef CASTRO_MINB_TRACE
#define CASTRO_MINB_TRACE 3
#endif
#ifndef CASTRO_MINB_RIEMANN
#define CASTRO_MINB_RIEMANN 5
#endif
#ifndef CASTRO_TRACE_SEG
#define CASTRO_TRACE_SEG 5
#endif
constexpr int BLOCK = CASTRO_BLOCK;
constexpr int TSEG = CASTRO_TRACE_SEG;   // zones of grow(bx,1) one trace thread walks along its direction
// Passes of BLOCK consecutive faces one block of riemann2 / riemann3 makes in
// turn on the batched path: the next pass's faces are the next row, whose
// flux records the previous pass has brought into this SM's L1
#ifndef CASTRO_R2_ROWS
#define CASTRO_R2_ROWS 1
#endif
#ifndef CASTRO_R3_ROWS
#define CASTRO_R3_ROWS 2
#endif
// The 13-species instantiations carry larger records and take their own
// register budgets (CASTRO_MINB13_*, 0 = the compiler's choice; measured on the
// 13-species reference problem): the budgets tuned for 2 species make the
// Riemann kernels spill.
#ifndef CASTRO_MINB13_EOS
#define CASTRO_MINB13_EOS 4
#endif
#ifndef CASTRO_MINB13_R3
#define CASTRO_MINB13_R3 0
#endif
#ifndef CASTRO_MINB13_TRACE
#define CASTRO_MINB13_TRACE 0
#endif
#ifndef CASTRO_MINB13_RIEMANN
#define CASTRO_MINB13_RIEMANN 3
#endif
// minimum resident blocks per SM of a kernel templated on NS (0 = no bound)
#define CASTRO_LB_NS(M2, M13) __launch_bounds__(BLOCK, (NS == 2 ? ((M2) > 0 ? (M2) : 0) : ((M13) > 0 ? (M13) : 0)))
#define LB_EOS CASTRO_LB_NS(CASTRO_MINB_EOS, CASTRO_MINB13_EOS)
#define LB_R3 CASTRO_LB_NS(CASTRO_MINB_R3, CASTRO_MINB13_R3)
#define LB_TRACE CASTRO_LB_NS(CASTRO_MINB_TRACE, CASTRO_MINB13_TRACE)
#define LB_RIEMANN CASTRO_LB_NS(CASTRO_MINB_RIEMANN, CASTRO_MINB13_RIEMANN)

// ordered pair (a,b), a != b -> 0..5
__host__ __device__ __forceinline__ int pair_index(int a, int b) { return a * 2 + (b > a ? b - 1 : b); }

struct BoxDev {
    int lo[3], hi[3];
    int inst;
    long long offU, offUb, offQ, offDiv;
    long long offTr[3], offF1[3], offF2[6], offFx[3];
};

struct InstDev {
    int dom_lo[3], dom_hi[3];
    int bc;
    int g;            // owner map granularity
    int on[3];        // owner map dims
    long long owner_off;
    double dx[3];
};

struct InstState {
    double dt;        // dt of the next step
    double time, dt_est, stop_time;
    double dt_last;   // dt of the last completed step (AMReX dtLevel after the step)
    int steps, pad;
};

struct Work { int box, sub, start, count; };

enum Region { R_VALID = 0, R_G1, R_G4, R_TBX, R_EBX, R_GHOST, R_SEG };

struct Reg {
    int lx, ly, lz, nx, ny, nz;
    long long np;
};

__host__ __device__ __forceinline__ Reg make_reg(const int* lo, const int* hi, int kind, int sub)
{
    int l[3] = {lo[0], lo[1], lo[2]}, h[3] = {hi[0], hi[1], hi[2]};
    if (kind == R_G1) { for (int d = 0; d < 3; ++d) { l[d] -= 1; h[d] += 1; } }
    else if (kind == R_G4) { for (int d = 0; d < 3; ++d) { l[d] -= NG; h[d] += NG; } }
    else if (kind == R_EBX) { h[sub] += 1; }
    else if (kind == R_GHOST) {
        // slab sub of grow(bx,4) minus bx: 0/1 low/high z (all of x, y), 2/3 low/high y
        // (all of x, valid z), 4/5 low/high x (valid y, z)
        const int a = 2 - sub / 2;
        for (int d = 0; d < a; ++d) { l[d] -= NG; h[d] += NG; }
        if (sub % 2 == 0) { h[a] = l[a] - 1; l[a] -= NG; }
        else { l[a] = h[a] + 1; h[a] += NG; }
    }
    else if (kind == R_SEG) {
        // grow(bx,1) with the coordinate along direction sub replaced by the
        // index of a segment of TSEG zones
        for (int d = 0; d < 3; ++d) { l[d] -= 1; h[d] += 1; }
        const int n = h[sub] - l[sub] + 1;
        l[sub] = 0;
        h[sub] = (n + TSEG - 1) / TSEG - 1;
    }
    else if (kind == R_TBX) {
        // sub = 3*a + b: faces normal to a; grown by 1 in the directions other
        // than a and b (Source/Castro_hydro.cpp:93-101)
        int a = sub / 3, b = sub % 3;
        h[a] += 1;
        for (int d = 0; d < 3; ++d)
            if (d != a && d != b) { l[d] -= 1; h[d] += 1; }
    }
    Reg r;
    r.lx = l[0]; r.ly = l[1]; r.lz = l[2];
    r.nx = h[0] - l[0] + 1; r.ny = h[1] - l[1] + 1; r.nz = h[2] - l[2] + 1;
    r.np = (long long)r.nx * r.ny * r.nz;
    return r;
}

__device__ __forceinline__ long long ridx(const Reg& r, int i, int j, int k)
{
    return (long long)(i - r.lx) + (long long)r.nx * ((long long)(j - r.ly) + (long long)r.ny * (k - r.lz));
}

struct SimDev {
    const BoxDev* boxes;
    const BoxDev* dom;        // per instance: the domain box whose stage arrays hold the final fluxes
    const InstDev* inst;
    InstState* st;
    double* U;
    double* Ub;
    double* Q;
    double* Div;
    double* Tr;
    double* F1;
    double* F2;
    double* Fx;
    const int* owner;
};

// item of a work list -> (box, zone index) of the thread's point in pass rep
// of the item (an item holds up to BLOCK points per pass); returns false for
// idle threads
__device__ __forceinline__ bool work_point_rep(const Work& w, const SimDev& S, int kind, int subkind_tbx, int rep,
                                              int& b, int& sub, Reg& R, int& i, int& j, int& k)
{
    const int tp = rep * BLOCK + (int)threadIdx.x;
    if (tp >= w.count) return false;
    b = w.box;
    sub = w.sub;
    const BoxDev& B = S.boxes[b];
    int rs = sub;
    if (kind == R_TBX && subkind_tbx == 0) rs = 4 * sub;   // tbx[d][d]
    R = make_reg(B.lo, B.hi, kind, rs);
    long long t = (long long)w.start + tp;
    i = R.lx + (int)(t % R.nx);
    long long t2 = t / R.nx;
    j = R.ly + (int)(t2 % R.ny);
    k = R.lz + (int)(t2 / R.ny);
    return true;
}

__device__ __forceinline__ bool work_point(const Work& w, const SimDev& S, int kind, int subkind_tbx, int& b, int& sub,
                                          Reg& R, int& i, int& j, int& k)
{
    return work_point_rep(w, S, kind, subkind_tbx, 0, b, sub, R, i, j, k);
}

// Q lives on grow(domain,4) and Sborder on grow(domain,1) of the box's
// instance: one array each per instance, written at every zone by the box that
// owns it, so the halo zones of a box that lie inside the domain are the
// neighbouring boxes' zones themselves and only the domain's own halo needs a
// fill (k_ghost).  On the single-box entry points the instance domain is the box.
__host__ __device__ __forceinline__ Reg q_region(const InstDev& I) { return make_reg(I.dom_lo, I.dom_hi, R_G4, 0); }
__host__ __device__ __forceinline__ Reg u_region(const InstDev& I) { return make_reg(I.dom_lo, I.dom_hi, R_G1, 0); }

// Q record: rho, u, v, w, p, rhoe, X[NS], gamc, c
template <int NS>
struct QF {
    static constexpr int RHO = 0, U = 1, P = 4, RE = 5, X = 6, GAMC = 6 + NS, C = 7 + NS, N = 8 + NS;
};

template <int NS>
struct QLoader {
    const double* base;
    Reg R;
    __device__ __forceinline__ double at(int i, int j, int k, int c) const { return base[ridx(R, i, j, k) + R.np * c]; }
    __device__ __forceinline__ double q(int i, int j, int k, int n) const
    {
        int c = (n == QRHO) ? QF<NS>::RHO : (n <= QW) ? n : (n == QPRES) ? QF<NS>::P : (n == QREINT) ? QF<NS>::RE : QF<NS>::X + (n - QFS);
        return at(i, j, k, c);
    }
    __device__ __forceinline__ double gamc(int i, int j, int k) const { return at(i, j, k, QF<NS>::GAMC); }
    __device__ __forceinline__ double c(int i, int j, int k) const { return at(i, j, k, QF<NS>::C); }
};

__device__ __forceinline__ void atomic_min_pos(double* addr, double v)
{
    unsigned long long* a = reinterpret_cast<unsigned long long*>(addr);
    unsigned long long old = *a, assumed;
    while (true) {
        double cur = __longlong_as_double((long long)old);
        if (!(v < cur)) break;
        assumed = old;
        old = atomicCAS(a, assumed, (unsigned long long)__double_as_longlong(v));
        if (old == assumed) break;
    }
}

__device__ __forceinline__ double block_min(double m)
{
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = DMIN(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 1.79769313486231570e+308;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = DMIN(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    return m;
}

// ---------------------------------------------------------------------------
// fused kernels
// ---------------------------------------------------------------------------

// front: clean_state(S_old) -> S_new base; clean_state(Sborder); ctoprim
template <int NS, bool COUL>
__device__ __forceinline__ void front_body(const SimDev& S, const Work& w)
{
    int b, sub, i, j, k;
    Reg R;
    if (!work_point(w, S, R_VALID, -1, b, sub, R, i, j, k)) return;
    const BoxDev& B = S.boxes[b];
    constexpr int NVAR = Dims<NS>::NVAR, QVAR = Dims<NS>::QVAR;
    double u[NVAR];
    double* U = S.U + B.offU;
    long long id = ridx(R, i, j, k);
#pragma unroll
    for (int n = 0; n < NVAR; ++n) u[n] = U[id + R.np * n];
    clean_state_pt<NS, COUL>(u);                    // Castro_advance.cpp:51
#pragma unroll
    for (int n = 0; n < NVAR; ++n) U[id + R.np * n] = u[n];
    clean_state_pt<NS, COUL>(u);                    // Castro_advance.cpp:66 (valid part of Sborder)
    const InstDev& I = S.inst[B.inst];
    const Reg R1 = u_region(I);
    double* Ub = S.Ub + B.offUb;
    long long id1 = ridx(R1, i, j, k);
#pragma unroll
    for (int n = 0; n < NVAR; ++n) Ub[id1 + R1.np * n] = u[n];
    double q[QVAR], qa[NQAUX];
    ctoprim_pt<NS, COUL>(u, q, qa);                 // Castro_hydro.cpp:64-70
    const Reg R4 = q_region(I);
    double* Q = S.Q + B.offQ;
    long long id4 = ridx(R4, i, j, k);
    using F = QF<NS>;
    Q[id4 + R4.np * F::RHO] = q[QRHO];
    Q[id4 + R4.np * (F::U + 0)] = q[QU];
    Q[id4 + R4.np * (F::U + 1)] = q[QV];
    Q[id4 + R4.np * (F::U + 2)] = q[QW];
    Q[id4 + R4.np * F::P] = q[QPRES];
    Q[id4 + R4.np * F::RE] = q[QREINT];
#pragma unroll
    for (int n = 0; n < NS; ++n) Q[id4 + R4.np * (F::X + n)] = q[QFS + n];
    Q[id4 + R4.np * F::GAMC] = qa[QGAMC];
    Q[id4 + R4.np * F::C] = qa[QC];
}

template <int NS, bool COUL>
__global__ void LB_EOS k_front(SimDev S, const Work* wl)
{
    front_body<NS, COUL>(S, wl[blockIdx.x]);
}

__device__ __forceinline__ int map_bc(int i, int lo, int hi, int bc)
{
    if (bc == CASTRO_BC_PERIODIC) {
        int n = hi - lo + 1;
        int r = (i - lo) % n;
        if (r < 0) r += n;
        return lo + r;
    }
    return i < lo ? lo : (i > hi ? hi : i);
}

// ghost: Q on grow(domain,4) and Sborder on grow(domain,1) outside the domain
// of each instance, from the domain zone the boundary condition maps to
// (periodic wrap or outflow nearest zone), one thread per halo zone.  Work item:
// box = any box of the instance (for its arrays), sub = slab of the domain halo.
// Sources are domain zones, written by k_front, never halo zones.
template <int NS>
__device__ __forceinline__ void ghost_body(const SimDev& S, const Work& w)
{
    if ((int)threadIdx.x >= w.count) return;
    const BoxDev& B = S.boxes[w.box];
    const InstDev& I = S.inst[B.inst];
    const Reg RS = make_reg(I.dom_lo, I.dom_hi, R_GHOST, w.sub);
    const long long t = (long long)w.start + threadIdx.x;
    const int i = RS.lx + (int)(t % RS.nx);
    const long long t2 = t / RS.nx;
    const int j = RS.ly + (int)(t2 % RS.ny);
    const int k = RS.lz + (int)(t2 / RS.ny);
    const int ii = map_bc(i, I.dom_lo[0], I.dom_hi[0], I.bc);
    const int jj = map_bc(j, I.dom_lo[1], I.dom_hi[1], I.bc);
    const int kk = map_bc(k, I.dom_lo[2], I.dom_hi[2], I.bc);
    const Reg R = q_region(I);
    double* Q = S.Q + B.offQ;
    const long long is = ridx(R, ii, jj, kk), id = ridx(R, i, j, k);
#pragma unroll
    for (int c = 0; c < QF<NS>::N; ++c) Q[id + R.np * c] = Q[is + R.np * c];
    if (i >= I.dom_lo[0] - 1 && i <= I.dom_hi[0] + 1 && j >= I.dom_lo[1] - 1 && j <= I.dom_hi[1] + 1 &&
        k >= I.dom_lo[2] - 1 && k <= I.dom_hi[2] + 1) {
        const Reg R1 = u_region(I);
        double* Ub = S.Ub + B.offUb;
        const long long is1 = ridx(R1, ii, jj, kk), id1 = ridx(R1, i, j, k);
#pragma unroll
        for (int n = 0; n < Dims<NS>::NVAR; ++n) Ub[id1 + R1.np * n] = Ub[is1 + R1.np * n];
    }
}

template <int NS>
__global__ void __launch_bounds__(BLOCK) k_ghost(SimDev S, const Work* wl)
{
    ghost_body<NS>(S, wl[blockIdx.x]);
}

// prep: divu at the nodes of grow(bx,1) (Castro_hydro_nd.F90:45-63) and the
// flattening coefficient of every zone of grow(bx,1) (ppm.F90:11-128), which
// trace_ppm recomputes per direction in the reference and is formed once here
template <int NS>
__device__ __forceinline__ void prep_body(const SimDev& S, const Work& w)
{
    int b, sub, i, j, k;
    Reg R;
    if (!work_point(w, S, R_G1, -1, b, sub, R, i, j, k)) return;
    const BoxDev& B = S.boxes[b];
    const InstDev& I = S.inst[B.inst];
    QLoader<NS> ld;
    ld.base = S.Q + B.offQ;
    ld.R = q_region(S.inst[B.inst]);
    double dxinv = 1.0 / I.dx[0], dyinv = 1.0 / I.dx[1], dzinv = 1.0 / I.dx[2];
    auto Qv = [&](int a, int bq, int c, int n) { return ld.at(a, bq, c, QF<NS>::U + n); };
    double ux = 0.25 * (+Qv(i, j, k, 0) - Qv(i - 1, j, k, 0)
                        + Qv(i, j, k - 1, 0) - Qv(i - 1, j, k - 1, 0)
                        + Qv(i, j - 1, k, 0) - Qv(i - 1, j - 1, k, 0)
                        + Qv(i, j - 1, k - 1, 0) - Qv(i - 1, j - 1, k - 1, 0)) * dxinv;
    double vy = 0.25 * (+Qv(i, j, k, 1) - Qv(i, j - 1, k, 1)
                        + Qv(i, j, k - 1, 1) - Qv(i, j - 1, k - 1, 1)
                        + Qv(i - 1, j, k, 1) - Qv(i - 1, j - 1, k, 1)
                        + Qv(i - 1, j, k - 1, 1) - Qv(i - 1, j - 1, k - 1, 1)) * dyinv;
    double wz = 0.25 * (+Qv(i, j, k, 2) - Qv(i, j, k - 1, 2)
                        + Qv(i, j - 1, k, 2) - Qv(i, j - 1, k - 1, 2)
                        + Qv(i - 1, j, k, 2) - Qv(i - 1, j, k - 1, 2)
                        + Qv(i - 1, j - 1, k, 2) - Qv(i - 1, j - 1, k - 1, 2)) * dzinv;
    long long id = ridx(R, i, j, k);
    S.Div[B.offDiv + id] = ux + vy + wz;
    S.Div[B.offDiv + id + R.np] = uflatten(ld, i, j, k);
}

template <int NS>
__global__ void __launch_bounds__(BLOCK) k_prep(SimDev S, const Work* wl)
{
    prep_body<NS>(S, wl[blockIdx.x]);
}

// trace_ppm (Source/ppm.F90:437-737) along one segment of up to TSEG zones of
// grow(bx,1) in direction D, the other two coordinates fixed.  Each zone's
// result equals trace_zone's bit for bit: the minus edge of zone z+1 and the
// plus edge of zone z are ppm_edge on the same operands, and the van Leer slope
// of zone z enters the edges of z-1, z and z+1 unchanged, so the thread forms
// every slope and edge once and carries them along the segment in registers
// (trace_zone forms three slopes and two edges per zone and variable).  Pass 1
// walks rho, u_D, p, rhoe and gamma_c, which feed the characteristic
// projection; pass 2 walks the transverse velocities and the species, one at a
// time, each needing only the u_D wave.
template <int NS, int D, int PASSES>   // bit 0: pass 1, bit 1: pass 2
__device__ __forceinline__ void trace_segment(const SimDev& S, const BoxDev& B, int i, int j, int k, double dtdx)
{
    using F = QF<NS>;
    constexpr int NQS = Dims<NS>::NQS;
    constexpr int T1 = D == 0 ? 1 : D == 1 ? 2 : 0;   // qut - QU of trace_zone
    constexpr int T2 = D == 0 ? 2 : D == 1 ? 0 : 1;   // qutt - QU
    const Reg R4 = q_region(S.inst[B.inst]);
    const Reg R1 = make_reg(B.lo, B.hi, R_G1, 0);
    const Reg RT = make_reg(B.lo, B.hi, R_TBX, 4 * D);
    int p[3] = {i, j, k};
    const int z0 = B.lo[D] - 1 + p[D] * TSEG;          // first zone of the segment
    const int n = min(TSEG, B.hi[D] + 2 - z0);           // zones in the segment
    p[D] = z0;
    const int zlo = B.lo[D] - z0, zhi = B.hi[D] - z0;    // zone offsets with a plus / minus face in tbx[D][D]
    const double* Q = S.Q + B.offQ;
    const double* Fl = S.Div + B.offDiv + R1.np;        // flatn
    double* Tr = S.Tr + B.offTr[D];
    // linear indices of zone z0 (Q, flatn) and of its low face (face states);
    // the face of zone lo-1 lies one stride below tbx[D][D] and is never stored
    const long long q0 = ridx(R4, p[0], p[1], p[2]);
    const long long f0 = ridx(R1, p[0], p[1], p[2]);
    const long long t0 = ridx(RT, p[0], p[1], p[2]);
    const long long sq = D == 0 ? 1 : D == 1 ? (long long)R4.nx : (long long)R4.nx * R4.ny;
    const long long sf = D == 0 ? 1 : D == 1 ? (long long)R1.nx : (long long)R1.nx * R1.ny;
    const long long st = D == 0 ? 1 : D == 1 ? (long long)RT.nx : (long long)RT.nx * RT.ny;
    const long long nq = R4.np, nt = RT.np;

    // pass 1: rho, u_D, p, rhoe, gamma_c.  Window of variable v at zone z:
    // wa = s(z), wb = s(z+1), wd = slope(z), we = edge(z) (minus edge of z).
    // The loads of zone z+1 (s(z+3), flatn, c) are issued while zone z is
    // computed: s(z+3) lies at most at hi+4 and c at hi+2, inside grow(bx,4);
    // flatn exists up to hi+1 and is fetched only for a zone of the segment.
    if constexpr ((PASSES & 1) != 0) {
    constexpr int NW = 5;
    constexpr int cw[NW] = {F::RHO, F::U + D, F::P, F::RE, F::GAMC};
    double wa[NW], wb[NW], wd[NW], we[NW], nxt[NW];
#pragma unroll
    for (int v = 0; v < NW; ++v) {
        const double* c = Q + q0 + (long long)cw[v] * nq;
        double sm2 = c[-2 * sq], sm1 = c[-sq], s0 = c[0], sp1 = c[sq];
        nxt[v] = c[2 * sq];
        double dm = vl_slope(sm2, sm1, s0);
        wd[v] = vl_slope(sm1, s0, sp1);
        we[v] = ppm_edge(sm1, s0, dm, wd[v]);
        wa[v] = s0;
        wb[v] = sp1;
    }
    double flatn_n = Fl[f0], cc_n = Q[q0 + (long long)F::C * nq];
#pragma unroll 1
    for (int z = 0; z < n; ++z) {
        const double flatn = flatn_n;
        const double cc = cc_n;
        const double un = wa[1];
        double cur[NW];
#pragma unroll
        for (int v = 0; v < NW; ++v) {
            cur[v] = nxt[v];
            nxt[v] = Q[q0 + (z + 3) * sq + (long long)cw[v] * nq];
        }
        cc_n = Q[q0 + (z + 1) * sq + (long long)F::C * nq];
        if (z + 1 < n) flatn_n = Fl[f0 + (z + 1) * sf];
        double Ip[3][4], Im[3][4], gp0, gm0, gp2, gm2;
#pragma unroll
        for (int v = 0; v < NW; ++v) {
            const double s2 = cur[v];
            const double dn = vl_slope(wa[v], wb[v], s2);
            const double en = ppm_edge(wa[v], wb[v], wd[v], dn);
            double sm = we[v], sp = en;
            ppm_limit(wa[v], flatn, sm, sp);
            const double s6 = 6.0 * wa[v] - 3.0 * (sm + sp);
            if (v < 4) {
                ppm_int_wave(sm, sp, s6, un - cc, dtdx, Ip[0][v], Im[0][v]);
                ppm_int_wave(sm, sp, s6, un, dtdx, Ip[1][v], Im[1][v]);
                ppm_int_wave(sm, sp, s6, un + cc, dtdx, Ip[2][v], Im[2][v]);
            } else {
                ppm_int_wave(sm, sp, s6, un - cc, dtdx, gp0, gm0);
                ppm_int_wave(sm, sp, s6, un + cc, dtdx, gp2, gm2);
            }
            wa[v] = wb[v];
            wb[v] = s2;
            wd[v] = dn;
            we[v] = en;
        }
        if (z >= zlo) {
            double r, u, re, pr;
            trace_project(Im, gm0, un, cc, true, r, u, re, pr);
            double* t = Tr + (t0 + z * st);
            t[nt * (NQS + SRHO)] = r;
            t[nt * (NQS + SU + D)] = u;
            t[nt * (NQS + SREI)] = re;
            t[nt * (NQS + SPRES)] = pr;
        }
        if (z <= zhi) {
            double r, u, re, pr;
            trace_project(Ip, gp2, un, cc, false, r, u, re, pr);
            double* t = Tr + (t0 + (z + 1) * st);
            t[nt * SRHO] = r;
            t[nt * (SU + D)] = u;
            t[nt * SREI] = re;
            t[nt * SPRES] = pr;
        }
    }

    }

    // pass 2: transverse velocities and species, the u_D wave only
    if constexpr ((PASSES & 2) != 0) {
#pragma unroll 1
    for (int v = 0; v < 2 + NS; ++v) {
        const int comp = v == 0 ? F::U + T1 : v == 1 ? F::U + T2 : F::X + (v - 2);
        const int slot = v == 0 ? SU + T1 : v == 1 ? SU + T2 : SX + (v - 2);
        const double* c = Q + q0 + (long long)comp * nq;
        const double* cu = Q + q0 + (long long)(F::U + D) * nq;
        double sm2 = c[-2 * sq], sm1 = c[-sq], a = c[0], bq = c[sq];
        double nxt2 = c[2 * sq], un_n = cu[0], flatn_n2 = Fl[f0];
        double d = vl_slope(sm1, a, bq);
        double e = ppm_edge(sm1, a, vl_slope(sm2, sm1, a), d);
#pragma unroll 1
        for (int z = 0; z < n; ++z) {
            const double flatn = flatn_n2;
            const double un = un_n;
            const double s2 = nxt2;
            nxt2 = c[(z + 3) * sq];
            un_n = cu[(z + 1) * sq];
            if (z + 1 < n) flatn_n2 = Fl[f0 + (z + 1) * sf];
            const double dn = vl_slope(a, bq, s2);
            const double en = ppm_edge(a, bq, d, dn);
            double sm = e, sp = en;
            ppm_limit(a, flatn, sm, sp);
            const double s6 = 6.0 * a - 3.0 * (sm + sp);
            double ip, im;
            ppm_int_wave(sm, sp, s6, un, dtdx, ip, im);
            if (z >= zlo) Tr[t0 + z * st + nt * (NQS + slot)] = im;
            if (z <= zhi) Tr[t0 + (z + 1) * st + nt * slot] = ip;
            a = bq;
            bq = s2;
            d = dn;
            e = en;
        }
    }
    }
}

template <int NS, int PASSES>
__device__ __forceinline__ void trace_item(const SimDev& S, const Work& w)
{
    int b, d, i, j, k;
    Reg R;
    if (!work_point(w, S, R_SEG, -1, b, d, R, i, j, k)) return;
    const BoxDev& B = S.boxes[b];
    const InstDev& I = S.inst[B.inst];
    const double dt = S.st[B.inst].dt;
    if (d == 0) trace_segment<NS, 0, PASSES>(S, B, i, j, k, dt / I.dx[0]);
    else if (d == 1) trace_segment<NS, 1, PASSES>(S, B, i, j, k, dt / I.dx[1]);
    else trace_segment<NS, 2, PASSES>(S, B, i, j, k, dt / I.dx[2]);
}

// trace: one segment of grow(bx,1) in one direction per thread (work sub =
// direction).  With CASTRO_TRACE_SPLIT, pass 2 (transverse velocities and
// species, a few registers per variable) runs as its own kernel k_trace2 at
// the occupancy its registers allow instead of pass 1's.
#ifndef CASTRO_TRACE_SPLIT
#define CASTRO_TRACE_SPLIT 1
#endif
#ifndef CASTRO_MINB_TRACE2
#define CASTRO_MINB_TRACE2 0
#endif
#define LB_TRACE2 CASTRO_LB_NS(CASTRO_MINB_TRACE2, 0)
template <int NS>
__global__ void LB_TRACE k_trace(SimDev S, const Work* wl)
{
    trace_item<NS, CASTRO_TRACE_SPLIT ? 1 : 3>(S, wl[blockIdx.x]);
}

template <int NS>
__global__ void LB_TRACE2 k_trace2(SimDev S, const Work* wl)
{
    trace_item<NS, 2>(S, wl[blockIdx.x]);
}

// compute_flux on the face (i,j,k) normal to D: left zone i-e_D, right zone i
// returns (GDPRES, Godunov velocity normal to the face)
template <int NS, int D>
__device__ __forceinline__ double2 riemann_at(const QLoader<NS>& ld, int i, int j, int k, const double* ql,
                                              const double* qr, double* flx)
{
    constexpr int ex = D == 0, ey = D == 1, ez = D == 2;
    double qg[NGDNV];
    riemann_cgf<NS, D>(ql, qr, ld.gamc(i - ex, j - ey, k - ez), ld.gamc(i, j, k), ld.c(i - ex, j - ey, k - ez),
                       ld.c(i, j, k), flx, qg, nullptr);
    return make_double2(qg[GDPRES], qg[GDU + D]);
}

template <int NS>
__device__ __forceinline__ void store_tf(double* base, const Reg& R, long long f, const double* flx, double pg, double ug)
{
    using T = TF<NS>;
    base[f + R.np * T::RHO] = flx[URHO];
    base[f + R.np * T::MX] = flx[UMX];
    base[f + R.np * T::MY] = flx[UMY];
    base[f + R.np * T::MZ] = flx[UMZ];
    base[f + R.np * T::ED] = flx[UEDEN];
#pragma unroll
    for (int n = 0; n < NS; ++n) base[f + R.np * (T::X + n)] = flx[UFS + n];
    base[f + R.np * T::PG] = pg;
    base[f + R.np * T::UG] = ug;
}

template <int NS>
__device__ __forceinline__ void load_tf(const double* base, const Reg& R, long long f, double* r)
{
#pragma unroll
    for (int c = 0; c < TF<NS>::N; ++c) r[c] = base[f + R.np * c];
}

// riemann1: compute_flux on tbx[d][d] (Castro_hydro.cpp:214-224)
template <int NS>
__device__ __forceinline__ void riemann1_body(const SimDev& S, const Work& w)
{
    int b, d, i, j, k;
    Reg R;
    if (!work_point(w, S, R_TBX, 0, b, d, R, i, j, k)) return;
    const BoxDev& B = S.boxes[b];
    constexpr int NQS = Dims<NS>::NQS, NVAR = Dims<NS>::NVAR;
    const double* T = S.Tr + B.offTr[d];
    long long f = ridx(R, i, j, k);
    double ql[NQS], qr[NQS];
#pragma unroll
    for (int c = 0; c < NQS; ++c) { ql[c] = T[f + R.np * c]; qr[c] = T[f + R.np * (NQS + c)]; }
    QLoader<NS> ld;
    ld.base = S.Q + B.offQ;
    ld.R = q_region(S.inst[B.inst]);
    double flx[NVAR];
    double2 g;
    if (d == 0) g = riemann_at<NS, 0>(ld, i, j, k, ql, qr, flx);
    else if (d == 1) g = riemann_at<NS, 1>(ld, i, j, k, ql, qr, flx);
    else g = riemann_at<NS, 2>(ld, i, j, k, ql, qr, flx);
    store_tf<NS>(S.F1 + B.offF1[d], R, f, flx, g.x, g.y);
}

template <int NS>
__global__ void LB_RIEMANN k_riemann1(SimDev S, const Work* wl)
{
    riemann1_body<NS>(S, wl[blockIdx.x]);
}

// 8-byte asynchronous global -> shared copies (cp.async, Ampere and later):
// the copies of one thread are in flight together without holding registers,
// and the thread waits for all of them once
__device__ __forceinline__ void cp_async8(double* dst, const double* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Per-thread shared-memory slot of riemann2: the face's two A-normal trace
// states and the two side zones' gamma_1, read once for both cross fluxes of
// the face.  The stride is odd, so that the 64-bit accesses of a half-warp
// fall in distinct bank pairs.  CASTRO_R2_STAGE 0 keeps them in registers
// (measured on B200: staging is faster; staging the normal-flux records too
// was slower, as each is read by about four neighbouring threads and is best
// served from L1).
#ifndef CASTRO_R2_STAGE
#define CASTRO_R2_STAGE 1
#endif
template <int NS>
struct R2Slot {
    static constexpr int NQS = Dims<NS>::NQS;
    static constexpr int LQ = 0;                   // 2 x NQS: minus (left) state, plus (right) state
    static constexpr int G = 2 * NQS;              // gamma_1 of the left and right zones
    static constexpr int USED = G + 2;
    static constexpr int STRIDE = USED | 1;
    static constexpr bool ON = CASTRO_R2_STAGE > 0;
    static constexpr int BYTES = ON ? STRIDE * BLOCK * 8 : 0;
};

// F^{A|Bd} on the A-normal face (i,j,k) from its two trace states lq (minus
// then plus, 2 x NQS), the side zones' gamma_1 (gl, gr) and sound speeds (cl,
// cr): trans1 of each state with the Bd normal fluxes of its zone, then
// compute_flux (Castro_hydro.cpp:228-255, 280-304); the record is written to
// the F2 pool
template <int NS, int A, int Bd>
__device__ __forceinline__ void cross_flux_store(const SimDev& S, const BoxDev& B, int i, int j, int k, double cdtdx,
                                                 const double* lq, double gl, double gr, double cl, double cr)
{
    constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF, NVAR = Dims<NS>::NVAR;
    constexpr int eax = A == 0, eay = A == 1, eaz = A == 2;
    constexpr int ebx_ = Bd == 0, eby = Bd == 1, ebz = Bd == 2;
    const Reg RF = make_reg(B.lo, B.hi, R_TBX, 4 * Bd);
    const double* F = S.F1 + B.offF1[Bd];
    double st2[2][NQS];
#pragma unroll
    for (int D = -1; D <= 0; ++D) {
        double fr[NTF], fl[NTF];
        const int il = i + D * eax, jl = j + D * eay, kl = k + D * eaz;
        load_tf<NS>(F, RF, ridx(RF, il + ebx_, jl + eby, kl + ebz), fr);
        load_tf<NS>(F, RF, ridx(RF, il, jl, kl), fl);
        trans1_state<NS>(lq + (D + 1) * NQS, fr, fl, D == -1 ? gl : gr, cdtdx, st2[D + 1]);
    }
    double flx[NVAR], qg[NGDNV];
    riemann_cgf<NS, A>(st2[0], st2[1], gl, gr, cl, cr, flx, qg, nullptr);
    const Reg R = make_reg(B.lo, B.hi, R_TBX, 3 * A + Bd);
    double* out = S.F2 + B.offF2[pair_index(A, Bd)];
    const long long f = ridx(R, i, j, k);
    using T_ = TF<NS>;
    out[f + R.np * T_::RHO] = flx[URHO];
    out[f + R.np * T_::MX] = flx[UMX];
    out[f + R.np * T_::MY] = flx[UMY];
    out[f + R.np * T_::MZ] = flx[UMZ];
    out[f + R.np * T_::ED] = flx[UEDEN];
#pragma unroll
    for (int n = 0; n < NS; ++n) out[f + R.np * (T_::X + n)] = flx[UFS + n];
    out[f + R.np * T_::PG] = qg[GDPRES];
    out[f + R.np * T_::UG] = qg[GDU + A];
}

// Both cross fluxes of the A-normal face (i,j,k) of tbx[A][A]: F^{A|B1} where
// the face lies in tbx[A][B1] (its B1 coordinate inside the box), F^{A|B2}
// likewise.  The face's trace states, gamma_1 and sound speeds are read once
// for the two.
template <int NS, int A>
__device__ __forceinline__ void cross_flux_both(const SimDev& S, const BoxDev& B, const InstDev& I,
                                                const QLoader<NS>& ld, int i, int j, int k, double dt)
{
    using SL = R2Slot<NS>;
    constexpr int NQS = Dims<NS>::NQS;
    constexpr int B1 = A == 0 ? 1 : 0, B2 = A == 2 ? 1 : 2;
    constexpr int eax = A == 0, eay = A == 1, eaz = A == 2;
    const Reg RT = make_reg(B.lo, B.hi, R_TBX, 4 * A);
    const double* T = S.Tr + B.offTr[A];
    const long long ft = ridx(RT, i, j, k);
    const long long zl = ridx(ld.R, i - eax, j - eay, k - eaz), zr = ridx(ld.R, i, j, k);
    double lqr[SL::ON ? 1 : 2 * NQS];
    const double* lq;
    double gl, gr;
    if constexpr (SL::ON) {
        extern __shared__ double r2_smem[];
        double* sm = r2_smem + threadIdx.x * SL::STRIDE;
#pragma unroll
        for (int c = 0; c < 2 * NQS; ++c) cp_async8(sm + SL::LQ + c, T + ft + RT.np * c);
        cp_async8(sm + SL::G, ld.base + zl + ld.R.np * QF<NS>::GAMC);
        cp_async8(sm + SL::G + 1, ld.base + zr + ld.R.np * QF<NS>::GAMC);
        lq = sm + SL::LQ;
        cp_async_wait_all();
        gl = sm[SL::G];
        gr = sm[SL::G + 1];
    } else {
#pragma unroll
        for (int c = 0; c < 2 * NQS; ++c) lqr[c] = T[ft + RT.np * c];
        lq = lqr;
        gl = ld.base[zl + ld.R.np * QF<NS>::GAMC];
        gr = ld.base[zr + ld.R.np * QF<NS>::GAMC];
    }
    const double cl = ld.base[zl + ld.R.np * QF<NS>::C], cr = ld.base[zr + ld.R.np * QF<NS>::C];
    const int p[3] = {i, j, k};
    if (p[B1] >= B.lo[B1] && p[B1] <= B.hi[B1])
        cross_flux_store<NS, A, B1>(S, B, i, j, k, dt / I.dx[B1] / 3.0, lq, gl, gr, cl, cr);
    if (p[B2] >= B.lo[B2] && p[B2] <= B.hi[B2])
        cross_flux_store<NS, A, B2>(S, B, i, j, k, dt / I.dx[B2] / 3.0, lq, gl, gr, cl, cr);
}

// riemann2: one thread per face of tbx[a][a] (Castro_hydro.cpp:228-304)
template <int NS>
__device__ __forceinline__ void riemann2_body(const SimDev& S, const Work& w)
{
    int bx, a, i, j, k;
    Reg R;
    for (int rp = 0; rp < CASTRO_R2_ROWS; ++rp) {
        if (!work_point_rep(w, S, R_TBX, 0, rp, bx, a, R, i, j, k)) return;
        const BoxDev& B = S.boxes[bx];
        const InstDev& I = S.inst[B.inst];
        const double dt = S.st[B.inst].dt;
        QLoader<NS> ld;
        ld.base = S.Q + B.offQ;
        ld.R = q_region(S.inst[B.inst]);
        if (a == 0) cross_flux_both<NS, 0>(S, B, I, ld, i, j, k, dt);
        else if (a == 1) cross_flux_both<NS, 1>(S, B, I, ld, i, j, k, dt);
        else cross_flux_both<NS, 2>(S, B, I, ld, i, j, k, dt);
    }
}

template <int NS>
__global__ void LB_RIEMANN k_riemann2(SimDev S, const Work* wl)
{
    riemann2_body<NS>(S, wl[blockIdx.x]);
}

// CASTRO_R3_STAGE: 0 plain loads, 1 the per-face operands of riemann3 that no
// neighbouring thread reads (both trace states, gamma_1, the two zones'
// Sborder values and the four divu nodes of apply_av) staged in shared memory
// by cp.async; the cross-flux records stay plain loads served from L1
// (measured on B200: 0 is faster, 0.85 against 0.90 ms for the 128^3 step).
#ifndef CASTRO_R3_STAGE
#define CASTRO_R3_STAGE 0
#endif
#ifndef CASTRO_R3_STAGE13
#define CASTRO_R3_STAGE13 1
#endif
template <int NS>
struct R3Slot {
    static constexpr int NQS = Dims<NS>::NQS, NVAR = Dims<NS>::NVAR;
    static constexpr int LQ = 0;              // 2 x NQS: minus (left) state, plus (right) state
    static constexpr int G = 2 * NQS;         // gamma_1 of the left and right zones
    static constexpr int UB = G + 2;          // Sborder of the right zone, then of the left zone (NVAR each)
    static constexpr int DV = UB + 2 * NVAR;  // the four divu nodes of apply_av
    static constexpr int USED = DV + 4;
    static constexpr int STRIDE = USED | 1;   // odd: conflict-free 64-bit accesses
    // 2 species: while four blocks fit; 13 species (255 registers, two blocks
    // per SM either way): while two blocks fit
    static constexpr int FIT = NS == 2 ? 4 : 2;
    static constexpr bool ON = (NS == 2 ? CASTRO_R3_STAGE > 0 : CASTRO_R3_STAGE13 > 0) &&
                               STRIDE * BLOCK * 8 * FIT + FIT * 1024 <= 228 * 1024;
    static constexpr int BYTES = ON ? STRIDE * BLOCK * 8 : 0;
};

// divu nodes summed by apply_av on a D-normal face, offsets from (i,j,k) in the
// order of Castro_hydro_nd.F90:207-237 (the x and y sums repeat a node there)
__device__ constexpr int AV_NODE[3][4][3] = {{{0, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 1, 0}},
                                             {{0, 0, 0}, {1, 0, 0}, {0, 0, 1}, {1, 0, 0}},
                                             {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {1, 1, 0}}};

// The final flux on the D-normal face (i,j,k) of ebx[D]: trans2 of the face's
// two D-normal trace states with the cross fluxes F^{t1|t2} (f12) and
// F^{t2|t1} (f21), compute_flux, apply_av, normalize_species_fluxes
// (Castro_hydro.cpp:307-359), written to the final-flux record of ebx[D].
// f12(i,j,k,rec) / f21(i,j,k,rec) load the cross-flux record at a face.  With
// STG the face's own operands come from the thread's shared-memory slot sm.
template <int NS, int D, bool STG, class L12, class L21>
__device__ __forceinline__ void final_flux(const SimDev& S, const BoxDev& B, const InstDev& I, const QLoader<NS>& ld,
                                           int i, int j, int k, double dt, const L12& f12, const L21& f21, double* sm)
{
    using SL = R3Slot<NS>;
    constexpr int T1 = (D == 0) ? 1 : 0;
    constexpr int T2 = (D == 2) ? 1 : 2;
    constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF, NVAR = Dims<NS>::NVAR;
    constexpr int ex = D == 0, ey = D == 1, ez = D == 2;
    constexpr int e1x = T1 == 0, e1y = T1 == 1, e1z = T1 == 2;
    constexpr int e2x = T2 == 0, e2y = T2 == 1, e2z = T2 == 2;
    const double hdt1 = 0.5 * dt / I.dx[T1], hdt2 = 0.5 * dt / I.dx[T2];
    const Reg RT = make_reg(B.lo, B.hi, R_TBX, 4 * D);
    const Reg R1 = make_reg(B.lo, B.hi, R_G1, 0);   // divu nodes
    const Reg RU = u_region(I);                         // Sborder
    const double* T = S.Tr + B.offTr[D];
    const double* Dv = S.Div + B.offDiv;
    const double* Ub = S.Ub + B.offUb;
    const long long ft = ridx(RT, i, j, k);
    const long long c0 = ridx(RU, i, j, k), cm = ridx(RU, i - ex, j - ey, k - ez);
    const long long zl = ridx(ld.R, i - ex, j - ey, k - ez), zr = ridx(ld.R, i, j, k);
    if constexpr (STG) {
#pragma unroll
        for (int c = 0; c < 2 * NQS; ++c) cp_async8(sm + SL::LQ + c, T + ft + RT.np * c);
        cp_async8(sm + SL::G, ld.base + zl + ld.R.np * QF<NS>::GAMC);
        cp_async8(sm + SL::G + 1, ld.base + zr + ld.R.np * QF<NS>::GAMC);
#pragma unroll
        for (int n = 0; n < NVAR; ++n) {
            if (n == UTEMP) continue;
            cp_async8(sm + SL::UB + n, Ub + c0 + RU.np * n);
            cp_async8(sm + SL::UB + NVAR + n, Ub + cm + RU.np * n);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m)
            cp_async8(sm + SL::DV + m, Dv + ridx(R1, i + AV_NODE[D][m][0], j + AV_NODE[D][m][1], k + AV_NODE[D][m][2]));
    }
    const double cl = ld.base[zl + ld.R.np * QF<NS>::C], cr = ld.base[zr + ld.R.np * QF<NS>::C];
    double st2[2][NQS];
#pragma unroll
    for (int Dm = -1; Dm <= 0; ++Dm) {
        double lqr[STG ? 1 : NQS], f2r[NTF], f2l[NTF], f3r[NTF], f3l[NTF];
        const int off = (Dm == -1) ? 0 : NQS;
        if constexpr (!STG) {
#pragma unroll
            for (int c = 0; c < NQS; ++c) lqr[c] = T[ft + RT.np * (off + c)];
        }
        int il = i + Dm * ex, jl = j + Dm * ey, kl = k + Dm * ez;
        f12(il + e1x, jl + e1y, kl + e1z, f2r);
        f12(il, jl, kl, f2l);
        f21(il + e2x, jl + e2y, kl + e2z, f3r);
        f21(il, jl, kl, f3l);
        if constexpr (STG) {
            if (Dm == -1) cp_async_wait_all();
        }
        const double* lq = STG ? sm + SL::LQ + off : lqr;
        const double gam = STG ? sm[SL::G + Dm + 1] : ld.gamc(il, jl, kl);
        trans2_state<NS>(lq, f2r, f2l, f3r, f3l, gam, hdt1, hdt2, st2[Dm + 1]);
    }
    double flx[NVAR], qg[NGDNV];
    {
        const double gl = STG ? sm[SL::G] : ld.gamc(i - ex, j - ey, k - ez);
        const double gr = STG ? sm[SL::G + 1] : ld.gamc(i, j, k);
        riemann_cgf<NS, D>(st2[0], st2[1], gl, gr, cl, cr, flx, qg, nullptr);
    }
    const double2 g = make_double2(qg[GDPRES], qg[GDU + D]);

    // apply_av, Castro_hydro_nd.F90:207-237
    {
        double dvn[4];
#pragma unroll
        for (int m = 0; m < 4; ++m)
            dvn[m] = STG ? sm[SL::DV + m] : Dv[ridx(R1, i + AV_NODE[D][m][0], j + AV_NODE[D][m][1], k + AV_NODE[D][m][2])];
        const double ds = dvn[0] + dvn[1] + dvn[2] + dvn[3];
        const double dxd = I.dx[D];
#pragma unroll
        for (int n = 0; n < NVAR; ++n) {
            if (n == UTEMP) continue;
            const double u0 = STG ? sm[SL::UB + n] : Ub[c0 + RU.np * n];
            const double um = STG ? sm[SL::UB + NVAR + n] : Ub[cm + RU.np * n];
            double div1 = av_term(ds, u0 - um);
            flx[n] = flx[n] + dxd * div1;
        }
    }
    // normalize_species_fluxes, Castro_hydro_nd.F90:277-291
    {
        double sum = 0.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) sum = sum + flx[UFS + n];
        double fac = (sum != 0.0) ? flx[URHO] / sum : 1.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) flx[UFS + n] = flx[UFS + n] * fac;
    }
    // final record: every flux component but UTEMP (always zero), GDPRES, GDU_D
    Reg R = make_reg(B.lo, B.hi, R_EBX, D);
    double* X = S.Fx + B.offFx[D];
    long long f = ridx(R, i, j, k);
#pragma unroll
    for (int n = 0; n < NVAR; ++n) {
        if (n == UTEMP) continue;
        X[f + R.np * (n < UTEMP ? n : n - 1)] = flx[n];
    }
    X[f + R.np * (NVAR - 1)] = g.x;
    X[f + R.np * NVAR] = g.y;
}

template <int NS>
struct GlobalTF {   // cross-flux records in the F2 pool
    const double* base;
    Reg R;
    __device__ __forceinline__ void operator()(int i, int j, int k, double* r) const { load_tf<NS>(base, R, ridx(R, i, j, k), r); }
};

template <int NS, int D>
__device__ __forceinline__ void riemann3_dir(const SimDev& S, const BoxDev& B, const InstDev& I, const QLoader<NS>& ld,
                                             int i, int j, int k, double dt)
{
    constexpr int T1 = (D == 0) ? 1 : 0;
    constexpr int T2 = (D == 2) ? 1 : 2;
    GlobalTF<NS> f12{S.F2 + B.offF2[pair_index(T1, T2)], make_reg(B.lo, B.hi, R_TBX, 3 * T1 + T2)};
    GlobalTF<NS> f21{S.F2 + B.offF2[pair_index(T2, T1)], make_reg(B.lo, B.hi, R_TBX, 3 * T2 + T1)};
    if constexpr (R3Slot<NS>::ON) {
        extern __shared__ double r3_smem[];
        final_flux<NS, D, true>(S, B, I, ld, i, j, k, dt, f12, f21, r3_smem + threadIdx.x * R3Slot<NS>::STRIDE);
    } else {
        final_flux<NS, D, false>(S, B, I, ld, i, j, k, dt, f12, f21, nullptr);
    }
}

// riemann3: the final fluxes on ebx[d] from the F2 pool
template <int NS>
__device__ __forceinline__ void riemann3_body(const SimDev& S, const Work& w)
{
    int bx, d, i, j, k;
    Reg R;
    for (int rp = 0; rp < CASTRO_R3_ROWS; ++rp) {
        if (!work_point_rep(w, S, R_EBX, -1, rp, bx, d, R, i, j, k)) return;
        const BoxDev& B = S.boxes[bx];
        const InstDev& I = S.inst[B.inst];
        const double dt = S.st[B.inst].dt;
        QLoader<NS> ld;
        ld.base = S.Q + B.offQ;
        ld.R = q_region(S.inst[B.inst]);
        if (d == 0) riemann3_dir<NS, 0>(S, B, I, ld, i, j, k, dt);
        else if (d == 1) riemann3_dir<NS, 1>(S, B, I, ld, i, j, k, dt);
        else riemann3_dir<NS, 2>(S, B, I, ld, i, j, k, dt);
    }
}

template <int NS>
__global__ void LB_R3 k_riemann3(SimDev S, const Work* wl)
{
    riemann3_body<NS>(S, wl[blockIdx.x]);
}

// ---------------------------------------------------------------------------
// riemann23 (castro_set_column_tiles; off by default, measured slower on B200
// than riemann2 + riemann3): riemann2 and riemann3 fused per column tile.  One block owns the
// zone columns [xa, xb] x [ya, yb] of an instance domain over a chunk of
// planes [za, zb] and marches up through it; the six cross fluxes
// (Castro_hydro.cpp:228-304) are formed into shared memory, two planes of
// each at most, and the final fluxes (Castro_hydro.cpp:307-359) read them
// there: the cross-flux records never go through HBM.  Every flux is formed by
// the same per-face stages as riemann2 / riemann3 on the same inputs, so the
// results are those of the two kernels, bit for bit.
//
// Iteration m (m = za-1 .. zb', zb' = zb + 1 at the domain's top, else zb):
//   A: XY(m), YX(m)                    planes za-1 .. zb'  (F^z of the faces m-1/2, m+1/2)
//      XZ(m), YZ(m)                    planes za .. zb     (F^y(m), F^x(m))
//      ZY(m+1), ZX(m+1)                z-faces m+1/2, for m+1 in za .. zb+1
//   B: F^x(m), F^y(m)                  planes za .. zb
//      F^z(m) (the face m-1/2)         za .. zb'
// XY is the F^{x|y} record of an x-face, ZY the F^{z|y} record of a z-face, and
// so on; z-face index k is the face k-1/2.  The block's x-faces are [xa, xb]
// (and xb+1 at the domain's high x end), likewise in y and z; the cross
// fluxes its final fluxes need reach one zone column beyond the tile.
// ---------------------------------------------------------------------------
#ifndef CASTRO_R23_TX
#define CASTRO_R23_TX 8
#endif
#ifndef CASTRO_R23_TY
#define CASTRO_R23_TY 8
#endif
#ifndef CASTRO_R23_ZC
#define CASTRO_R23_ZC 16      // planes per block
#endif
#ifndef CASTRO_R23_NT
#define CASTRO_R23_NT 128     // threads per block
#endif
#ifndef CASTRO_R23_MINB
#define CASTRO_R23_MINB 3
#endif

struct TileItem { int inst, x0, y0, z0; };

// A cross-flux record buffer in shared memory: planes of nx x ny records whose
// slot (0,0) is zone column (x0, y0); component c of slot s at base[c * slots + s]
struct SmemTF {
    double* base;
    int slots, x0, y0, nx, ny, two;
    __device__ __forceinline__ int slot(int i, int j, int k) const
    {
        return (i - x0) + nx * ((j - y0) + ny * (two ? (k & 1) : 0));
    }
    template <int NS>
    __device__ __forceinline__ void load(int i, int j, int k, double* r) const
    {
        const double* p = base + slot(i, j, k);
#pragma unroll
        for (int c = 0; c < TF<NS>::N; ++c) r[c] = p[c * slots];
    }
};

template <int NS>
struct SmemTFLoader {
    SmemTF b;
    __device__ __forceinline__ void operator()(int i, int j, int k, double* r) const { b.template load<NS>(i, j, k, r); }
};

template <int NS>
struct R23Layout {
    static constexpr int TX = CASTRO_R23_TX, TY = CASTRO_R23_TY, NTF = TF<NS>::N;
    // records per buffer (all planes): XY, YX, XZ, YZ, ZY, ZX
    static constexpr int S_XY = (TX + 1) * TY * 2, S_YX = TX * (TY + 1) * 2;
    static constexpr int S_XZ = (TX + 1) * (TY + 2), S_YZ = (TX + 2) * (TY + 1);
    static constexpr int S_ZY = (TX + 2) * TY * 2, S_ZX = TX * (TY + 2) * 2;
    static constexpr int O_XY = 0, O_YX = O_XY + NTF * S_XY, O_XZ = O_YX + NTF * S_YX, O_YZ = O_XZ + NTF * S_XZ,
                         O_ZY = O_YZ + NTF * S_YZ, O_ZX = O_ZY + NTF * S_ZY, DOUBLES = O_ZX + NTF * S_ZX;
    static constexpr int BYTES = DOUBLES * 8;
};

// F^{A|Bd} of the A-normal face (i,j,k) into the record slot out[c * stride]:
// cross_flux_store's arithmetic (trans1 of both trace states, compute_flux)
template <int NS, int A, int Bd>
__device__ __forceinline__ void cross_flux_rec(const SimDev& S, const BoxDev& B, int i, int j, int k, double cdtdx,
                                               const double* lq, double gl, double gr, double cl, double cr,
                                               double* out, int stride)
{
    constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF, NVAR = Dims<NS>::NVAR;
    constexpr int eax = A == 0, eay = A == 1, eaz = A == 2;
    constexpr int ebx_ = Bd == 0, eby = Bd == 1, ebz = Bd == 2;
    const Reg RF = make_reg(B.lo, B.hi, R_TBX, 4 * Bd);
    const double* F = S.F1 + B.offF1[Bd];
    double st2[2][NQS];
#pragma unroll
    for (int D = -1; D <= 0; ++D) {
        double fr[NTF], fl[NTF];
        const int il = i + D * eax, jl = j + D * eay, kl = k + D * eaz;
        load_tf<NS>(F, RF, ridx(RF, il + ebx_, jl + eby, kl + ebz), fr);
        load_tf<NS>(F, RF, ridx(RF, il, jl, kl), fl);
        trans1_state<NS>(lq + (D + 1) * NQS, fr, fl, D == -1 ? gl : gr, cdtdx, st2[D + 1]);
    }
    double flx[NVAR], qg[NGDNV];
    riemann_cgf<NS, A>(st2[0], st2[1], gl, gr, cl, cr, flx, qg, nullptr);
    using T_ = TF<NS>;
    out[stride * T_::RHO] = flx[URHO];
    out[stride * T_::MX] = flx[UMX];
    out[stride * T_::MY] = flx[UMY];
    out[stride * T_::MZ] = flx[UMZ];
    out[stride * T_::ED] = flx[UEDEN];
#pragma unroll
    for (int n = 0; n < NS; ++n) out[stride * (T_::X + n)] = flx[UFS + n];
    out[stride * T_::PG] = qg[GDPRES];
    out[stride * T_::UG] = qg[GDU + A];
}

// one cross flux F^{A|Bd} of the A-normal face (i,j,k) into out[c * stride]
template <int NS, int A, int Bd>
__device__ __forceinline__ void cross_one(const SimDev& S, const BoxDev& B, const InstDev& I, const QLoader<NS>& ld,
                                          int i, int j, int k, double dt, double* out, int stride)
{
    constexpr int NQS = Dims<NS>::NQS;
    constexpr int eax = A == 0, eay = A == 1, eaz = A == 2;
    const Reg RT = make_reg(B.lo, B.hi, R_TBX, 4 * A);
    const double* T = S.Tr + B.offTr[A];
    const long long ft = ridx(RT, i, j, k);
    double lq[2 * NQS];
#pragma unroll
    for (int c = 0; c < 2 * NQS; ++c) lq[c] = T[ft + RT.np * c];
    const long long zl = ridx(ld.R, i - eax, j - eay, k - eaz), zr = ridx(ld.R, i, j, k);
    const double gl = ld.base[zl + ld.R.np * QF<NS>::GAMC], gr = ld.base[zr + ld.R.np * QF<NS>::GAMC];
    const double cl = ld.base[zl + ld.R.np * QF<NS>::C], cr = ld.base[zr + ld.R.np * QF<NS>::C];
    cross_flux_rec<NS, A, Bd>(S, B, i, j, k, dt / I.dx[Bd] / 3.0, lq, gl, gr, cl, cr, out, stride);
}

template <int NS>
__global__ void __launch_bounds__(CASTRO_R23_NT, CASTRO_R23_MINB) k_riemann23(SimDev S, const TileItem* items)
{
    using L = R23Layout<NS>;
    extern __shared__ double r23_smem[];
    const TileItem it = items[blockIdx.x];
    const BoxDev& B = S.boxes[it.inst];                 // the instance domain (the stage arrays' box)
    const InstDev& I = S.inst[B.inst];
    const double dt = S.st[B.inst].dt;
    QLoader<NS> ld;
    ld.base = S.Q + B.offQ;
    ld.R = q_region(I);
    const int xa = it.x0, xb = min(it.x0 + L::TX - 1, B.hi[0]);
    const int ya = it.y0, yb = min(it.y0 + L::TY - 1, B.hi[1]);
    const int za = it.z0, zb = min(it.z0 + CASTRO_R23_ZC - 1, B.hi[2]);
    const int fxb = xb + (xb == B.hi[0]), fyb = yb + (yb == B.hi[1]), fzb = zb + (zb == B.hi[2]);
    SmemTF XY{r23_smem + L::O_XY, L::S_XY, xa, ya, L::TX + 1, L::TY, 1};
    SmemTF YX{r23_smem + L::O_YX, L::S_YX, xa, ya, L::TX, L::TY + 1, 1};
    SmemTF XZ{r23_smem + L::O_XZ, L::S_XZ, xa, ya - 1, L::TX + 1, L::TY + 2, 0};
    SmemTF YZ{r23_smem + L::O_YZ, L::S_YZ, xa - 1, ya, L::TX + 2, L::TY + 1, 0};
    SmemTF ZY{r23_smem + L::O_ZY, L::S_ZY, xa - 1, ya, L::TX + 2, L::TY, 1};
    SmemTF ZX{r23_smem + L::O_ZX, L::S_ZX, xa, ya - 1, L::TX, L::TY + 2, 1};
    // Phase A: six task lists, one cross flux per task, each list starting on a
    // warp boundary, so that a warp runs one face direction and record pair.
    const int wX = xb + 2 - xa, wT = xb - xa + 1, wH = fxb - xa + 2;      // x extents: [xa, xb+1], [xa, xb], [xa-1, fxb]
    const int hT = yb - ya + 1, hT1 = yb - ya + 2, hH = fyb - ya + 2;     // y extents: [ya, yb], [ya, yb+1], [ya-1, fyb]
    const int n[6] = {wX * hT, wX * hH, wT * hT1, wH * hT1, wH * hT, wT * hH};   // XY XZ YX YZ ZY ZX
    // phase B: x-faces [xa, fxb] x [ya, yb], y-faces [xa, xb] x [ya, fyb], z-faces [xa, xb] x [ya, yb]
    const int wF = fxb - xa + 1;
    const int nb[3] = {wF * hT, wT * (fyb - ya + 1), wT * hT};
    for (int m = za - 1; m <= fzb; ++m) {
        const bool pXZ = m >= za && m <= zb;               // XZ, YZ of plane m
        const bool pZ = m <= zb;                           // ZY, ZX of the z-face m+1 (in [za, zb+1])
        const bool act[6] = {true, pXZ, true, pXZ, pZ, pZ};
        int o[7];
        o[0] = 0;
#pragma unroll
        for (int q = 0; q < 6; ++q) o[q + 1] = o[q] + (act[q] ? (n[q] + 31) & ~31 : 0);
        for (int t = threadIdx.x; t < o[6]; t += CASTRO_R23_NT) {
            int q = 0;
#pragma unroll
            for (int r = 1; r < 6; ++r) q += t >= o[r];
            const int u = t - o[q];
            if (u >= n[q]) continue;
            switch (q) {
            case 0: {
                const int i = xa + u % wX, j = ya + u / wX;
                cross_one<NS, 0, 1>(S, B, I, ld, i, j, m, dt, XY.base + XY.slot(i, j, m), XY.slots);
            } break;
            case 1: {
                const int i = xa + u % wX, j = ya - 1 + u / wX;
                cross_one<NS, 0, 2>(S, B, I, ld, i, j, m, dt, XZ.base + XZ.slot(i, j, m), XZ.slots);
            } break;
            case 2: {
                const int i = xa + u % wT, j = ya + u / wT;
                cross_one<NS, 1, 0>(S, B, I, ld, i, j, m, dt, YX.base + YX.slot(i, j, m), YX.slots);
            } break;
            case 3: {
                const int i = xa - 1 + u % wH, j = ya + u / wH;
                cross_one<NS, 1, 2>(S, B, I, ld, i, j, m, dt, YZ.base + YZ.slot(i, j, m), YZ.slots);
            } break;
            case 4: {
                const int i = xa - 1 + u % wH, j = ya + u / wH;
                cross_one<NS, 2, 1>(S, B, I, ld, i, j, m + 1, dt, ZY.base + ZY.slot(i, j, m + 1), ZY.slots);
            } break;
            default: {
                const int i = xa + u % wT, j = ya - 1 + u / wT;
                cross_one<NS, 2, 0>(S, B, I, ld, i, j, m + 1, dt, ZX.base + ZX.slot(i, j, m + 1), ZX.slots);
            } break;
            }
        }
        __syncthreads();
        const bool fxy = m >= za && m <= zb;               // F^x(m), F^y(m)
        const bool fz = m >= za;                           // F^z of the face m-1/2 (m <= fzb)
        const bool bact[3] = {fxy, fxy, fz};
        int ob[4];
        ob[0] = 0;
#pragma unroll
        for (int q = 0; q < 3; ++q) ob[q + 1] = ob[q] + (bact[q] ? (nb[q] + 31) & ~31 : 0);
        for (int t = threadIdx.x; t < ob[3]; t += CASTRO_R23_NT) {
            const int q = (t >= ob[1]) + (t >= ob[2]);
            const int u = t - ob[q];
            if (u >= nb[q]) continue;
            if (q == 0) {
                const int i = xa + u % wF, j = ya + u / wF;
                final_flux<NS, 0, false>(S, B, I, ld, i, j, m, dt, SmemTFLoader<NS>{YZ}, SmemTFLoader<NS>{ZY}, nullptr);
            } else if (q == 1) {
                const int i = xa + u % wT, j = ya + u / wT;
                final_flux<NS, 1, false>(S, B, I, ld, i, j, m, dt, SmemTFLoader<NS>{XZ}, SmemTFLoader<NS>{ZX}, nullptr);
            } else {
                const int i = xa + u % wT, j = ya + u / wT;
                final_flux<NS, 2, false>(S, B, I, ld, i, j, m, dt, SmemTFLoader<NS>{XY}, SmemTFLoader<NS>{YX}, nullptr);
            }
        }
        __syncthreads();
    }
}

// update: fill_hydro_source, Saxpy, clean_state (advance), clean_state
// (post_timestep), estdt of the new state
template <int NS, bool COUL>
__device__ __forceinline__ void update_body(const SimDev& S, const Work& w)
{
    int b, sub, i, j, k;
    Reg R;
    bool active = work_point(w, S, R_VALID, -1, b, sub, R, i, j, k);
    const BoxDev& B = S.boxes[w.box];
    const InstDev& I = S.inst[B.inst];
    double m = 1.79769313486231570e+308;
    if (active) {
        constexpr int NVAR = Dims<NS>::NVAR;
        const double dt = S.st[B.inst].dt;
        const double a0 = I.dx[1] * I.dx[2], a1 = I.dx[0] * I.dx[2], a2 = I.dx[0] * I.dx[1];
        const double volinv = 1.0 / (I.dx[0] * I.dx[1] * I.dx[2]);
        Reg RX[3];
        const double* X[3];
        long long f0[3], f1[3];
        const BoxDev& DB = S.dom[B.inst];   // final fluxes live on the domain's faces
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            RX[d] = make_reg(DB.lo, DB.hi, R_EBX, d);
            X[d] = S.Fx + DB.offFx[d];
            f0[d] = ridx(RX[d], i, j, k);
            f1[d] = ridx(RX[d], i + (d == 0), j + (d == 1), k + (d == 2));
        }
        double* U = S.U + B.offU;
        long long id = ridx(R, i, j, k);
        double u[NVAR];
#pragma unroll
        for (int n = 0; n < NVAR; ++n) {
            double un = U[id + R.np * n];
            if (n == UTEMP) { u[n] = un + dt * 0.0; continue; }
            const int c = n < UTEMP ? n : n - 1;
            double src = 0.0 + (X[0][f0[0] + RX[0].np * c] * a0 - X[0][f1[0] + RX[0].np * c] * a0
                              + X[1][f0[1] + RX[1].np * c] * a1 - X[1][f1[1] + RX[1].np * c] * a1
                              + X[2][f0[2] + RX[2].np * c] * a2 - X[2][f1[2] + RX[2].np * c] * a2) * volinv;
            if (n == UEINT) {
                const int P = NVAR - 1, V = NVAR;
                double pdivu = 0.5 * (X[0][f1[0] + RX[0].np * P] + X[0][f0[0] + RX[0].np * P]) *
                                   (X[0][f1[0] + RX[0].np * V] - X[0][f0[0] + RX[0].np * V]) / I.dx[0] +
                               0.5 * (X[1][f1[1] + RX[1].np * P] + X[1][f0[1] + RX[1].np * P]) *
                                   (X[1][f1[1] + RX[1].np * V] - X[1][f0[1] + RX[1].np * V]) / I.dx[1] +
                               0.5 * (X[2][f1[2] + RX[2].np * P] + X[2][f0[2] + RX[2].np * P]) *
                                   (X[2][f1[2] + RX[2].np * V] - X[2][f0[2] + RX[2].np * V]) / I.dx[2];
                src = src - pdivu;
            }
            u[n] = un + dt * src;                        // MultiFab::Saxpy, Castro_advance.cpp:74
        }
        clean_state_pt<NS, COUL>(u);                     // Castro_advance.cpp:78
        clean_state_pt<NS, COUL>(u);                     // Castro.cpp:369
#pragma unroll
        for (int n = 0; n < NVAR; ++n) U[id + R.np * n] = u[n];
        m = estdt_pt<NS, COUL>(u, I.dx[0], I.dx[1], I.dx[2]);   // Castro.cpp:191-203 of the next coarse step
    }
    // one box per block: the block reduction has a single instance target
    m = block_min(m);
    if (threadIdx.x == 0) atomic_min_pos(&S.st[B.inst].dt_est, m);
}

template <int NS, bool COUL>
__global__ void LB_EOS k_update(SimDev S, const Work* wl)
{
    update_body<NS, COUL>(S, wl[blockIdx.x]);
}

// estdt on the current state (computeInitialDt / castro_sim_est_time_step)
template <int NS, bool COUL>
__device__ __forceinline__ void estdt_state_body(const SimDev& S, const Work& w)
{
    int b, sub, i, j, k;
    Reg R;
    bool active = work_point(w, S, R_VALID, -1, b, sub, R, i, j, k);
    const BoxDev& B = S.boxes[w.box];
    const InstDev& I = S.inst[B.inst];
    double m = 1.79769313486231570e+308;
    if (active) {
        constexpr int NVAR = Dims<NS>::NVAR;
        const double* U = S.U + B.offU;
        long long id = ridx(R, i, j, k);
        double u[NVAR];
#pragma unroll
        for (int n = 0; n < NVAR; ++n) u[n] = U[id + R.np * n];
        m = estdt_pt<NS, COUL>(u, I.dx[0], I.dx[1], I.dx[2]);
    }
    m = block_min(m);
    if (threadIdx.x == 0) atomic_min_pos(&S.st[B.inst].dt_est, m);
}

template <int NS, bool COUL>
__global__ void __launch_bounds__(BLOCK) k_estdt_state(SimDev S, const Work* wl)
{
    estdt_state_body<NS, COUL>(S, wl[blockIdx.x]);
}

// computeInitialDt (DT_FIRST) or, after a step, time/step bookkeeping and
// computeNewDt (DT_STEP; Source/Castro.cpp:162-341).  DT_RESTART is
// computeNewDt alone, for a state restored from a checkpoint whose st.dt holds
// the last step's dt: the same dt the uninterrupted run formed at that step's end.
enum { DT_STEP = 0, DT_FIRST = 1, DT_RESTART = 2 };
__device__ __forceinline__ void next_dt(InstState& st, int first)
{
    double est = st.dt_est * cfl;                       // estTimeStep, Castro.cpp:212-213
    double dt_0;
    if (first == DT_FIRST) {
        dt_0 = DMIN(1.0e+100, 0.01 * est);               // initialTimeStep, Castro.cpp:168-170
    } else {
        if (first == DT_STEP) {
            st.time = st.time + st.dt;
            st.steps = st.steps + 1;
            st.dt_last = st.dt;
        }
        double dt_min = DMIN(est, 1.1e0 * st.dt);        // Castro.cpp:264-267
        dt_0 = DMIN(1.0e+100, dt_min);
    }
    double eps = 0.001 * dt_0;
    if (st.stop_time >= 0.0) {
        if ((st.time + dt_0) > (st.stop_time - eps)) dt_0 = st.stop_time - st.time;
    }
    st.dt = dt_0;
    st.dt_est = 1.79769313486231570e+308;
}

__global__ void k_dt(SimDev S, int ninst, int first)
{
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= ninst) return;
    next_dt(S.st[n], first);
}

// ---------------------------------------------------------------------------
// CASTRO_MODE_PERSISTENT: the whole batched step in ONE cooperative launch.
// Every CTA stays resident for the step and pulls work items -- (box or
// domain box, region, chunk) descriptors of every instance -- from one device
// queue per stage with an atomic counter, so the CTAs that finish early take
// the remaining items of the ragged BoxArrays and instance sizes.  The stages
// are those of the ten-kernel graph (front, ghost, prep, trace with both of its
// passes in one queue, riemann1-3, update); between two stages the CTAs meet
// at a grid barrier.  Co-residency is guaranteed by the cooperative launch, and
// every barrier wait is bounded: after PersistArgs::spin_limit polls it
// records the stage in the control block's error word and the CTA returns,
// as does every other CTA that sees the word, so a stuck step ends with an
// error the host reads (castro_sim_sync) instead of a hang.  The update stage
// folds each box's estdt into its instance's dt_est (warp-shuffle block minimum,
// one atomic per item: a reduction segmented by instance); the last CTA to
// finish the step forms every instance's next dt (computeNewDt) in the epilogue.
// ---------------------------------------------------------------------------
enum { PS_FRONT = 0, PS_GHOST, PS_PREP, PS_TRACE, PS_R1, PS_R2, PS_R3, PS_UPDATE, PS_COUNT };

struct PersistCtl {
    unsigned int queue[PS_COUNT];    // next item of each stage's queue
    unsigned int arrive[PS_COUNT];   // CTAs past each stage
    unsigned int done;               // CTAs that finished the step
    int error;                       // 0, or 1 + the stage whose barrier wait ran out
};

struct PersistArgs {
    const Work* wl[PS_COUNT];
    int n[PS_COUNT];                 // items per stage (trace: pass 1 items, then pass 2 items)
    int trace_items;                 // items of one trace pass
    PersistCtl* ctl;
    int ninst;
    long long spin_limit;            // polls of a barrier wait before it gives up
    int test_stage;                  // test hook: the barrier after this stage ...
    int test_extra;                  // ... waits for this many CTAs more than exist (0: none)
};

#ifndef CASTRO_MINB_PERSIST
#define CASTRO_MINB_PERSIST 3
#endif
#ifndef CASTRO_MINB13_PERSIST
#define CASTRO_MINB13_PERSIST 2
#endif
#define LB_PERSIST CASTRO_LB_NS(CASTRO_MINB_PERSIST, CASTRO_MINB13_PERSIST)

__device__ __forceinline__ unsigned int ld_acquire_u32(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_acquire_s32(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// grid barrier after stage st; false when a wait ran out (this CTA's or another's)
__device__ __forceinline__ bool persist_barrier(const PersistArgs& P, int st)
{
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        __threadfence();                                   // this CTA's stage writes, device-wide
        atomicAdd(&P.ctl->arrive[st], 1u);
        const unsigned int target = gridDim.x + (st == P.test_stage ? (unsigned int)P.test_extra : 0u);
        int ok = 1;
        long long polls = 0;
        while (ld_acquire_u32(&P.ctl->arrive[st]) < target) {
            if (ld_acquire_s32(&P.ctl->error) != 0) { ok = 0; break; }
            if (++polls > P.spin_limit) {
                atomicCAS(&P.ctl->error, 0, st + 1);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <int NS, bool COUL>
__device__ __forceinline__ void persist_item(const SimDev& S, const SimDev& Sd, const PersistArgs& P, int st, int item)
{
    switch (st) {
    case PS_FRONT: front_body<NS, COUL>(S, P.wl[PS_FRONT][item]); break;
    case PS_GHOST: ghost_body<NS>(S, P.wl[PS_GHOST][item]); break;
    case PS_PREP: prep_body<NS>(Sd, P.wl[PS_PREP][item]); break;
    case PS_TRACE:
        if (!CASTRO_TRACE_SPLIT) trace_item<NS, 3>(Sd, P.wl[PS_TRACE][item]);
        else if (item < P.trace_items) trace_item<NS, 1>(Sd, P.wl[PS_TRACE][item]);
        else trace_item<NS, 2>(Sd, P.wl[PS_TRACE][item - P.trace_items]);
        break;
    case PS_R1: riemann1_body<NS>(Sd, P.wl[PS_R1][item]); break;
    case PS_R2: riemann2_body<NS>(Sd, P.wl[PS_R2][item]); break;
    case PS_R3: riemann3_body<NS>(Sd, P.wl[PS_R3][item]); break;
    default: update_body<NS, COUL>(S, P.wl[PS_UPDATE][item]); break;
    }
}

template <int NS, bool COUL>
__global__ void LB_PERSIST k_step_persistent(SimDev S, PersistArgs P)
{
    __shared__ int s_item;
    SimDev Sd = S;
    Sd.boxes = S.dom;                                      // the stage kernels' items name domain boxes
    for (int st = 0; st < PS_COUNT; ++st) {
        const int n = P.n[st];
        while (true) {
            if (threadIdx.x == 0) s_item = (int)atomicAdd(&P.ctl->queue[st], 1u);
            __syncthreads();
            const int item = s_item;
            __syncthreads();                               // every thread has the item before the slot is reused
            if (item >= n) break;
            persist_item<NS, COUL>(S, Sd, P, st, item);
        }
        if (st + 1 < PS_COUNT && !persist_barrier(P, st)) return;
    }
    // epilogue: the last CTA to finish forms every instance's next dt from the
    // dt_est minima its update items folded in
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&P.ctl->done, 1u) == gridDim.x - 1) {
            __threadfence();
            for (int n = 0; n < P.ninst; ++n) next_dt(S.st[n], DT_STEP);
        }
    }
}

// FillPatch of Sborder for the plain path: every zone of grow(bx,4) from the
// owning box's state under the instance boundary condition
template <int NS>
__global__ void __launch_bounds__(BLOCK) k_fill_sborder(SimDev S, int b, double* sb)
{
    const BoxDev& B = S.boxes[b];
    Reg R = make_reg(B.lo, B.hi, R_G4, 0);
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= R.np) return;
    int i = R.lx + (int)(t % R.nx);
    long long t2 = t / R.nx;
    int j = R.ly + (int)(t2 % R.ny);
    int k = R.lz + (int)(t2 / R.ny);
    const InstDev& I = S.inst[B.inst];
    int ii = map_bc(i, I.dom_lo[0], I.dom_hi[0], I.bc);
    int jj = map_bc(j, I.dom_lo[1], I.dom_hi[1], I.bc);
    int kk = map_bc(k, I.dom_lo[2], I.dom_hi[2], I.bc);
    int ob = S.owner[I.owner_off + (long long)((ii - I.dom_lo[0]) / I.g) +
                     (long long)I.on[0] * ((long long)((jj - I.dom_lo[1]) / I.g) + (long long)I.on[1] * ((kk - I.dom_lo[2]) / I.g))];
    const BoxDev& O = S.boxes[ob];
    Reg RO = make_reg(O.lo, O.hi, R_VALID, 0);
    const double* Us = S.U + O.offU;
    long long is = ridx(RO, ii, jj, kk);
#pragma unroll
    for (int n = 0; n < Dims<NS>::NVAR; ++n) sb[t + R.np * n] = Us[is + RO.np * n];
}

// primitive variables straight from a caller's Sborder over grow(bx,4)
// (construct_hydro_source's ctoprim, Source/Castro_hydro.cpp:64-70)
template <int NS, bool COUL>
__global__ void __launch_bounds__(BLOCK) k_box_prim(SimDev S, const Work* wl, Fab SB)
{
    const Work& w = wl[blockIdx.x];
    int b, sub, i, j, k;
    Reg R;
    if (!work_point(w, S, R_G4, -1, b, sub, R, i, j, k)) return;
    const BoxDev& B = S.boxes[b];
    constexpr int NVAR = Dims<NS>::NVAR, QVAR = Dims<NS>::QVAR;
    double u[NVAR], q[QVAR], qa[NQAUX];
#pragma unroll
    for (int n = 0; n < NVAR; ++n) u[n] = SB(i, j, k, n);
    ctoprim_pt<NS, COUL>(u, q, qa);
    const InstDev& I = S.inst[B.inst];
    const Reg RQ = q_region(I);   // grow(bx,4): the instance domain is the box here
    double* Q = S.Q + B.offQ;
    long long id = ridx(RQ, i, j, k);
    using F = QF<NS>;
    Q[id + RQ.np * F::RHO] = q[QRHO];
    Q[id + RQ.np * (F::U + 0)] = q[QU];
    Q[id + RQ.np * (F::U + 1)] = q[QV];
    Q[id + RQ.np * (F::U + 2)] = q[QW];
    Q[id + RQ.np * F::P] = q[QPRES];
    Q[id + RQ.np * F::RE] = q[QREINT];
#pragma unroll
    for (int n = 0; n < NS; ++n) Q[id + RQ.np * (F::X + n)] = q[QFS + n];
    Q[id + RQ.np * F::GAMC] = qa[QGAMC];
    Q[id + RQ.np * F::C] = qa[QC];
    if (i >= B.lo[0] - 1 && i <= B.hi[0] + 1 && j >= B.lo[1] - 1 && j <= B.hi[1] + 1 && k >= B.lo[2] - 1 && k <= B.hi[2] + 1) {
        const Reg R1 = u_region(I);
        double* Ub = S.Ub + B.offUb;
        long long i1 = ridx(R1, i, j, k);
#pragma unroll
        for (int n = 0; n < NVAR; ++n) Ub[i1 + R1.np * n] = u[n];
    }
}

// fill_hydro_source into the caller's source FAB (Castro_hydro_nd.F90:411-439)
template <int NS>
__global__ void __launch_bounds__(BLOCK) k_box_source(SimDev S, const Work* wl, Fab SRC)
{
    const Work& w = wl[blockIdx.x];
    int b, sub, i, j, k;
    Reg R;
    if (!work_point(w, S, R_VALID, -1, b, sub, R, i, j, k)) return;
    const BoxDev& B = S.boxes[b];
    const InstDev& I = S.inst[B.inst];
    constexpr int NVAR = Dims<NS>::NVAR;
    const double a0 = I.dx[1] * I.dx[2], a1 = I.dx[0] * I.dx[2], a2 = I.dx[0] * I.dx[1];
    const double volinv = 1.0 / (I.dx[0] * I.dx[1] * I.dx[2]);
    Reg RX[3];
    const double* X[3];
    long long f0[3], f1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        RX[d] = make_reg(B.lo, B.hi, R_EBX, d);
        X[d] = S.Fx + B.offFx[d];
        f0[d] = ridx(RX[d], i, j, k);
        f1[d] = ridx(RX[d], i + (d == 0), j + (d == 1), k + (d == 2));
    }
#pragma unroll
    for (int n = 0; n < NVAR; ++n) {
        if (n == UTEMP) { SRC(i, j, k, n) = SRC(i, j, k, n) + 0.0 * volinv; continue; }
        const int c = n < UTEMP ? n : n - 1;
        double s = SRC(i, j, k, n) + (X[0][f0[0] + RX[0].np * c] * a0 - X[0][f1[0] + RX[0].np * c] * a0
                                    + X[1][f0[1] + RX[1].np * c] * a1 - X[1][f1[1] + RX[1].np * c] * a1
                                    + X[2][f0[2] + RX[2].np * c] * a2 - X[2][f1[2] + RX[2].np * c] * a2) * volinv;
        if (n == UEINT) {
            const int P = NVAR - 1, V = NVAR;
            double pdivu = 0.5 * (X[0][f1[0] + RX[0].np * P] + X[0][f0[0] + RX[0].np * P]) *
                               (X[0][f1[0] + RX[0].np * V] - X[0][f0[0] + RX[0].np * V]) / I.dx[0] +
                           0.5 * (X[1][f1[1] + RX[1].np * P] + X[1][f0[1] + RX[1].np * P]) *
                               (X[1][f1[1] + RX[1].np * V] - X[1][f0[1] + RX[1].np * V]) / I.dx[1] +
                           0.5 * (X[2][f1[2] + RX[2].np * P] + X[2][f0[2] + RX[2].np * P]) *
                               (X[2][f1[2] + RX[2].np * V] - X[2][f0[2] + RX[2].np * V]) / I.dx[2];
            s = s - pdivu;
        }
        SRC(i, j, k, n) = s;
    }
}

// store_flux (Castro_hydro_nd.F90:330-338): dt * F * A on the faces of ebx[d]
template <int NS>
__global__ void __launch_bounds__(BLOCK) k_box_store_flux(SimDev S, const Work* wl, Fab FO0, Fab FO1, Fab FO2, double dt)
{
    const Work& w = wl[blockIdx.x];
    int b, d, i, j, k;
    Reg R;
    if (!work_point(w, S, R_EBX, -1, b, d, R, i, j, k)) return;
    const BoxDev& B = S.boxes[b];
    const InstDev& I = S.inst[B.inst];
    const Fab& FO = d == 0 ? FO0 : d == 1 ? FO1 : FO2;
    if (!FO.p) return;
    const double area = d == 0 ? I.dx[1] * I.dx[2] : d == 1 ? I.dx[0] * I.dx[2] : I.dx[0] * I.dx[1];
    const double* X = S.Fx + B.offFx[d];
    long long f = ridx(R, i, j, k);
#pragma unroll
    for (int n = 0; n < Dims<NS>::NVAR; ++n) {
        double F = (n == UTEMP) ? 0.0 : X[f + R.np * (n < UTEMP ? n : n - 1)];
        FO(i, j, k, n) = dt * F * area;
    }
}

__global__ void k_saxpy(double* u, const double* s, long long n, const double* dtp)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) u[t] += *dtp * s[t];
}

__global__ void k_fill(double* p, long long n, double v)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) p[t] = v;
}

}  // namespace
}  // namespace castro

using namespace castro;

// ===========================================================================
// the simulation object
// ===========================================================================
struct castro_sim {
    int mode = CASTRO_MODE_BATCHED;
    int ns = 2;
    int nvar = 9;
    int ninst = 0;
    cudaStream_t st = nullptr;
    // second stream and events of the captured step: the two trace kernels,
    // independent of each other, become parallel graph nodes
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    std::vector<castro_instance_desc> desc;
    std::vector<castro_problem> probs;
    std::vector<std::vector<int>> inst_boxes;   // global box ids per instance
    std::vector<BoxDev> hboxes;
    std::vector<BoxDev> hdom;     // per instance: the domain as one box (stage arrays)
    std::vector<InstDev> hinst;
    std::vector<double> hdx;                    // 3 per instance
    BoxDev* dboxes = nullptr;
    BoxDev* ddom = nullptr;
    InstDev* dinst = nullptr;
    InstState* dstate = nullptr;
    int* downer = nullptr;
    double *U = nullptr, *Ub = nullptr, *Q = nullptr, *Div = nullptr;
    double *Tr = nullptr, *F1 = nullptr, *F2 = nullptr, *Fx = nullptr;
    long long nU = 0;
    // work lists
    Work *w_valid = nullptr, *w_g4 = nullptr, *w_g1 = nullptr, *w_trace = nullptr, *w_tbx = nullptr,
         *w_ebx = nullptr, *w_r2 = nullptr, *w_r3 = nullptr, *w_ghost = nullptr;
    int n_valid = 0, n_g4 = 0, n_g1 = 0, n_trace = 0, n_tbx = 0, n_ebx = 0, n_r2 = 0, n_r3 = 0, n_ghost = 0;
    // column tiles of riemann23 (2 species, batched mode): the step runs it in place of riemann2 + riemann3
    TileItem* w_r23 = nullptr;
    int n_r23 = 0;
    bool r23 = false;
    bool dt_ready = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    bool graph_coul = false;   // the Coulomb setting the captured step's EOS kernels were instantiated for
    int launches = 0;
    // EOS Newton non-convergences (library-wide counter) already reported
    // through castro_last_error when this sim last synchronized
    unsigned long long eos_seen = 0;
    unsigned long long eos_base = 0;   // the counter when this sim was created
    // CASTRO_MODE_PERSISTENT: control block, arguments and launch shape of the
    // one cooperative launch per step
    PersistCtl* pctl = nullptr;
    PersistArgs pargs;
    int pgrid = 0;
    size_t psmem = 0;
    bool pdirect = false;      // the driver refused to capture the cooperative launch: launch it directly
    bool failed = false;       // a device wait ran out: the state is void
    // plain-path scratch (largest box)
    double* sb = nullptr;      // Sborder per box (grow 4) for all boxes
    double* src = nullptr;     // hydro_source per box for all boxes
    std::vector<long long> offSb, offSrc;
    long long scratch_n = 0;
    // The per-box host sequence deals its boxes round-robin to PLAIN_STREAMS
    // streams, as AMReX's MFIter does with its GPU streams (4 by default,
    // amrex.max_gpu_streams), each with its own construct_hydro_source
    // scratch; every loop over the boxes starts after the step's stream
    // (fork) and ends before its next work (join), as an MFIter loop ends with
    // a synchronisation of its streams.
    static constexpr int PLAIN_STREAMS = 4;
    cudaStream_t pst[PLAIN_STREAMS] = {};
    cudaEvent_t pev[PLAIN_STREAMS] = {};
    cudaEvent_t pfork = nullptr;
    double* scratch[PLAIN_STREAMS] = {};
    double* d_dtloc = nullptr; // managed-style reduction target of estdt
    double* d_dtbox = nullptr; // dt per instance for the plain saxpy
    SimDev dev() const
    {
        SimDev S;
        S.boxes = dboxes; S.dom = ddom; S.inst = dinst; S.st = dstate;
        S.U = U; S.Ub = Ub; S.Q = Q; S.Div = Div; S.Tr = Tr; S.F1 = F1; S.F2 = F2; S.Fx = Fx;
        S.owner = downer;
        return S;
    }
    // the stage kernels' view: their work items name domain boxes
    SimDev dev_dom() const
    {
        SimDev S = dev();
        S.boxes = ddom;
        return S;
    }
};

namespace {

long long npts_reg(const int* lo, const int* hi, int kind, int sub)
{
    Reg r = make_reg(lo, hi, kind, sub);
    return r.np;
}

bool cuda_ok(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        char buf[256];
        snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
        set_error(CASTRO_ERR_CUDA, buf);
        return false;
    }
    return true;
}

template <class T>
bool dalloc(T** p, size_t n, const char* what)
{
    if (n == 0) n = 1;
    return cuda_ok(cudaMalloc((void**)p, n * sizeof(T)), what);
}

void build_work(const std::vector<BoxDev>& boxes, int kind, int nsub, int tbx_mode, Work** out, int* count,
                int passes = 1)
{
    // sub-major order: every box's items of one direction before the next, so
    // the blocks resident on an SM run the same code path
    std::vector<Work> w;
    for (int sub = 0; sub < nsub; ++sub) {
        for (size_t b = 0; b < boxes.size(); ++b) {
            const BoxDev& B = boxes[b];
            int rs = sub;
            if (kind == R_TBX && tbx_mode == 0) rs = 4 * sub;
            long long np = npts_reg(B.lo, B.hi, kind, rs);
            if (np > 2147483647LL - BLOCK) {   // work items carry 32-bit offsets
                set_error(CASTRO_ERR_ARG, "castro_sim_create: a domain region exceeds 2^31 points");
                *count = 0;
                return;
            }
            const long long chunk = (long long)BLOCK * passes;
            for (long long st = 0; st < np; st += chunk) {
                Work it;
                it.box = (int)b;
                it.sub = sub;
                it.start = (int)st;
                it.count = (int)std::min<long long>(chunk, np - st);
                w.push_back(it);
            }
        }
    }
    *count = (int)w.size();
    if (dalloc(out, w.size(), "work list"))
        cuda_ok(cudaMemcpy(*out, w.data(), w.size() * sizeof(Work), cudaMemcpyHostToDevice), "work list copy");
}

// Shared-memory sizing of the kernels that stage operands (set outside any
// graph capture, before the first launch on the current device)
template <int NS>
bool set_kernel_attributes()
{
    if (R3Slot<NS>::BYTES > 48 * 1024 &&
        !cuda_ok(cudaFuncSetAttribute(k_riemann3<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, R3Slot<NS>::BYTES),
                 "riemann3 shared memory"))
        return false;
    if (R2Slot<NS>::BYTES > 48 * 1024 &&
        !cuda_ok(cudaFuncSetAttribute(k_riemann2<NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, R2Slot<NS>::BYTES),
                 "riemann2 shared memory"))
        return false;
    return true;
}

// work list of k_ghost: the six slabs of grow(domain,4) \ domain of every
// instance, items naming the instance's first box
void build_ghost_work(castro_sim* s)
{
    std::vector<Work> w;
    for (int sub = 0; sub < 6; ++sub)
        for (int in = 0; in < s->ninst; ++in) {
            const InstDev& I = s->hinst[in];
            const long long np = npts_reg(I.dom_lo, I.dom_hi, R_GHOST, sub);
            for (long long st = 0; st < np; st += BLOCK) {
                Work it;
                it.box = s->inst_boxes[in][0];
                it.sub = sub;
                it.start = (int)st;
                it.count = (int)std::min<long long>(BLOCK, np - st);
                w.push_back(it);
            }
        }
    s->n_ghost = (int)w.size();
    if (dalloc(&s->w_ghost, w.size(), "ghost work list"))
        cuda_ok(cudaMemcpy(s->w_ghost, w.data(), w.size() * sizeof(Work), cudaMemcpyHostToDevice), "ghost work list copy");
}

// Launch of a kernel that calls the EOS: the instantiation with or without the
// Coulomb corrections, as the library is set (castro_set_coulomb_corrections).
#define CASTRO_EOS_LAUNCH(K, NS, GRID, BLK, SMEM, ST, ...)                         \
    do {                                                                           \
        if (coulomb_on()) K<NS, true><<<GRID, BLK, SMEM, ST>>>(__VA_ARGS__);        \
        else K<NS, false><<<GRID, BLK, SMEM, ST>>>(__VA_ARGS__);                     \
    } while (0)

// riemann23's column tiles over every instance domain; its shared memory
bool build_r23_work(castro_sim* s)
{
    std::vector<TileItem> w;
    for (size_t in = 0; in < s->hdom.size(); ++in) {
        const BoxDev& D = s->hdom[in];
        for (int z = D.lo[2]; z <= D.hi[2]; z += CASTRO_R23_ZC)
            for (int y = D.lo[1]; y <= D.hi[1]; y += CASTRO_R23_TY)
                for (int x = D.lo[0]; x <= D.hi[0]; x += CASTRO_R23_TX) w.push_back(TileItem{(int)in, x, y, z});
    }
    if (!cuda_ok(cudaFuncSetAttribute(k_riemann23<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, R23Layout<2>::BYTES),
                 "riemann23 shared memory") ||
        !dalloc(&s->w_r23, w.size(), "riemann23 tiles") ||
        !cuda_ok(cudaMemcpy(s->w_r23, w.data(), w.size() * sizeof(TileItem), cudaMemcpyHostToDevice), "riemann23 tiles"))
        return false;
    s->n_r23 = (int)w.size();
    s->r23 = true;
    return true;
}

template <int NS>
void launch_riemann23(castro_sim* s, const SimDev& Sd, cudaStream_t st)
{
    if constexpr (NS == 2)
        k_riemann23<2><<<s->n_r23, CASTRO_R23_NT, R23Layout<2>::BYTES, st>>>(Sd, s->w_r23);
}

template <int NS>
void batched_step_kernels(castro_sim* s)
{
    SimDev S = s->dev(), Sd = s->dev_dom();
    cudaStream_t st = s->st;
    CASTRO_EOS_LAUNCH(k_front, NS, s->n_valid, BLOCK, 0, st, S, s->w_valid);
    k_ghost<NS><<<s->n_ghost, BLOCK, 0, st>>>(S, s->w_ghost);
    k_prep<NS><<<s->n_g1, BLOCK, 0, st>>>(Sd, s->w_g1);
    if (CASTRO_TRACE_SPLIT) {
        // pass 2 writes face-state components pass 1 does not, from the same inputs
        cudaEventRecord(s->ev_fork, st);
        cudaStreamWaitEvent(s->st2, s->ev_fork, 0);
        k_trace2<NS><<<s->n_trace, BLOCK, 0, s->st2>>>(Sd, s->w_trace);
        k_trace<NS><<<s->n_trace, BLOCK, 0, st>>>(Sd, s->w_trace);
        cudaEventRecord(s->ev_join, s->st2);
        cudaStreamWaitEvent(st, s->ev_join, 0);
    } else {
        k_trace<NS><<<s->n_trace, BLOCK, 0, st>>>(Sd, s->w_trace);
    }
    k_riemann1<NS><<<s->n_tbx, BLOCK, 0, st>>>(Sd, s->w_tbx);
    if (s->r23) {
        launch_riemann23<NS>(s, Sd, st);
    } else {
        k_riemann2<NS><<<s->n_r2, BLOCK, R2Slot<NS>::BYTES, st>>>(Sd, s->w_r2);
        k_riemann3<NS><<<s->n_r3, BLOCK, R3Slot<NS>::BYTES, st>>>(Sd, s->w_r3);
    }
    CASTRO_EOS_LAUNCH(k_update, NS, s->n_valid, BLOCK, 0, st, S, s->w_valid);
    k_dt<<<(s->ninst + 63) / 64, 64, 0, st>>>(S, s->ninst, 0);
}

template <int NS>
void profile_kernel(castro_sim* s, const SimDev& S, int k)
{
    static const char* names[10] = {"front", "ghost", "prep", "trace", "riemann1", "riemann2", "riemann3", "update", "dt",
                                    "trace2"};
    NvtxRange r(k >= 0 && k < 10 ? names[k] : "kernel");
    cudaStream_t st = s->st;
    SimDev Sd = S;
    Sd.boxes = S.dom;
    switch (k) {
    case 0: CASTRO_EOS_LAUNCH(k_front, NS, s->n_valid, BLOCK, 0, st, S, s->w_valid); break;
    case 1: k_ghost<NS><<<s->n_ghost, BLOCK, 0, st>>>(S, s->w_ghost); break;
    case 2: k_prep<NS><<<s->n_g1, BLOCK, 0, st>>>(Sd, s->w_g1); break;
    case 3: k_trace<NS><<<s->n_trace, BLOCK, 0, st>>>(Sd, s->w_trace); break;
    case 9: k_trace2<NS><<<s->n_trace, BLOCK, 0, st>>>(Sd, s->w_trace); break;
    case 4: k_riemann1<NS><<<s->n_tbx, BLOCK, 0, st>>>(Sd, s->w_tbx); break;
    case 5:
        if (s->r23) launch_riemann23<NS>(s, Sd, st);   // riemann2 and riemann3 in one kernel
        else k_riemann2<NS><<<s->n_r2, BLOCK, R2Slot<NS>::BYTES, st>>>(Sd, s->w_r2);
        break;
    case 6:
        if (!s->r23) k_riemann3<NS><<<s->n_r3, BLOCK, R3Slot<NS>::BYTES, st>>>(Sd, s->w_r3);
        break;
    case 7: CASTRO_EOS_LAUNCH(k_update, NS, s->n_valid, BLOCK, 0, st, S, s->w_valid); break;
    default: k_dt<<<(s->ninst + 63) / 64, 64, 0, st>>>(S, s->ninst, 0); break;
    }
}

template <int NS>
void initial_dt_kernels(castro_sim* s)
{
    SimDev S = s->dev();
    CASTRO_EOS_LAUNCH(k_estdt_state, NS, s->n_valid, BLOCK, 0, s->st, S, s->w_valid);
    k_dt<<<(s->ninst + 63) / 64, 64, 0, s->st>>>(S, s->ninst, 1);
}

// ---- plain path: the reference host sequence through the per-routine ABI ----

struct PlainScratch {
    // FABs of Castro_hydro.cpp:54-170 for one box
    double *q, *qaux, *flux[3], *qe[3], *qm[3][3], *qp[3][3], *div, *q_int, *ftmp1, *ftmp2, *qg1, *qg2, *ql, *qr;
    double *area[3], *vol;
};

struct IBox { int lo[3], hi[3]; };
IBox grow(IBox b, int gx, int gy, int gz)
{
    b.lo[0] -= gx; b.lo[1] -= gy; b.lo[2] -= gz;
    b.hi[0] += gx; b.hi[1] += gy; b.hi[2] += gz;
    return b;
}
long long npts(const IBox& b) { return (long long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1); }

// Castro::clean_state, Source/Castro.cpp:563-591: the reference's four calls
// (the per-routine path), or the coarse castro_clean_state (the drop-in path)
void plain_clean(const castro_sim* s, const int* lo, const int* hi, double* u, const int* ulo, const int* uhi)
{
    if (s->mode == CASTRO_MODE_PLAIN_BOX) {
        castro_clean_state(lo, hi, u, ulo, uhi);
        return;
    }
    enforce_minimum_density(lo, hi, u, ulo, uhi);
    normalize_species(lo, hi, u, ulo, uhi);
    reset_internal_e(lo, hi, u, ulo, uhi);
    compute_temp(lo, hi, u, ulo, uhi);
}

// Castro::construct_hydro_source for one box through the per-routine entry
// points, Source/Castro_hydro.cpp:31-397
void plain_hydro_box(castro_sim* s, double* scratch, const IBox& bx, double* sbp, double* srcp, const int* domlo,
                     const int* domhi, const double* dx, double dt)
{
    const int NV = s->nvar, QV = s->nvar + 1;
    IBox obx = grow(bx, 1, 1, 1), qbx = grow(bx, NG, NG, NG);
    IBox sbx = qbx;
    IBox ebx[3], gebx[3], tbx[3][3];
    double* cur = scratch;
    auto take = [&](const IBox& b, int nc) { double* p = cur; cur += npts(b) * nc; return p; };
    PlainScratch P;
    P.q = take(qbx, QV);
    P.qaux = take(qbx, NQAUX);
    ctoprim(qbx.lo, qbx.hi, sbp, sbx.lo, sbx.hi, P.q, qbx.lo, qbx.hi, P.qaux, qbx.lo, qbx.hi);
    for (int d = 0; d < 3; ++d) {
        ebx[d] = bx; ebx[d].hi[d] += 1;
        gebx[d] = grow(ebx[d], 1, 1, 1);
        P.flux[d] = take(gebx[d], NV);
        P.qe[d] = take(gebx[d], NGDNV);
        P.area[d] = take(gebx[d], 1);
    }
    tbx[0][0] = grow(ebx[0], 0, 1, 1); tbx[0][1] = grow(ebx[0], 0, 0, 1); tbx[0][2] = grow(ebx[0], 0, 1, 0);
    tbx[1][0] = grow(ebx[1], 0, 0, 1); tbx[1][1] = grow(ebx[1], 1, 0, 1); tbx[1][2] = grow(ebx[1], 1, 0, 0);
    tbx[2][0] = grow(ebx[2], 0, 1, 0); tbx[2][1] = grow(ebx[2], 1, 0, 0); tbx[2][2] = grow(ebx[2], 1, 1, 0);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) { P.qm[a][b] = take(tbx[a][b], QV); P.qp[a][b] = take(tbx[a][b], QV); }
    P.div = take(obx, 1);
    divu(obx.lo, obx.hi, P.q, qbx.lo, qbx.hi, dx, P.div, obx.lo, obx.hi);
    P.q_int = take(obx, QV);
    P.ftmp1 = take(obx, NV);
    P.ftmp2 = take(obx, NV);
    P.qg1 = take(obx, NGDNV);
    P.qg2 = take(obx, NGDNV);
    P.ql = take(obx, QV);
    P.qr = take(obx, QV);
    P.vol = take(bx, 1);
    if (cur - scratch > s->scratch_n) { set_error(CASTRO_ERR_ARG, "plain path scratch overflow"); return; }

    double hdtdx[3], cdtdx[3];
    for (int d = 0; d < 3; ++d) { hdtdx[d] = 0.5 * dt / dx[d]; cdtdx[d] = dt / dx[d] / 3.0; }
    for (int d = 0; d < 3; ++d)
        trace_ppm(obx.lo, obx.hi, bx.lo, bx.hi, d + 1, P.q, qbx.lo, qbx.hi, P.qaux, qbx.lo, qbx.hi,
                  P.qm[d][d], tbx[d][d].lo, tbx[d][d].hi, P.qp[d][d], tbx[d][d].lo, tbx[d][d].hi, domlo, domhi, dx, dt);
    for (int d = 0; d < 3; ++d) {
        int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
        const IBox& b = tbx[d][d];
        compute_flux(b.lo, b.hi, P.qm[d][d], b.lo, b.hi, P.qp[d][d], b.lo, b.hi, P.ftmp1, obx.lo, obx.hi,
                     P.q_int, obx.lo, obx.hi, P.qg1, obx.lo, obx.hi, P.qaux, qbx.lo, qbx.hi, d + 1);
        trans1(tbx[t1][d].lo, tbx[t1][d].hi, d + 1, t1 + 1, P.qm[t1][t1], tbx[t1][t1].lo, tbx[t1][t1].hi,
               P.qm[t1][d], tbx[t1][d].lo, tbx[t1][d].hi, P.qp[t1][t1], tbx[t1][t1].lo, tbx[t1][t1].hi,
               P.qp[t1][d], tbx[t1][d].lo, tbx[t1][d].hi, P.qaux, qbx.lo, qbx.hi, P.ftmp1, obx.lo, obx.hi,
               P.qg1, obx.lo, obx.hi, cdtdx[d]);
        trans1(tbx[t2][d].lo, tbx[t2][d].hi, d + 1, t2 + 1, P.qm[t2][t2], tbx[t2][t2].lo, tbx[t2][t2].hi,
               P.qm[t2][d], tbx[t2][d].lo, tbx[t2][d].hi, P.qp[t2][t2], tbx[t2][t2].lo, tbx[t2][t2].hi,
               P.qp[t2][d], tbx[t2][d].lo, tbx[t2][d].hi, P.qaux, qbx.lo, qbx.hi, P.ftmp1, obx.lo, obx.hi,
               P.qg1, obx.lo, obx.hi, cdtdx[d]);
    }
    for (int d = 0; d < 3; ++d) {
        int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
        compute_flux(tbx[t1][t2].lo, tbx[t1][t2].hi, P.qm[t1][t2], tbx[t1][t2].lo, tbx[t1][t2].hi,
                     P.qp[t1][t2], tbx[t1][t2].lo, tbx[t1][t2].hi, P.ftmp1, obx.lo, obx.hi, P.q_int, obx.lo, obx.hi,
                     P.qg1, obx.lo, obx.hi, P.qaux, qbx.lo, qbx.hi, t1 + 1);
        compute_flux(tbx[t2][t1].lo, tbx[t2][t1].hi, P.qm[t2][t1], tbx[t2][t1].lo, tbx[t2][t1].hi,
                     P.qp[t2][t1], tbx[t2][t1].lo, tbx[t2][t1].hi, P.ftmp2, obx.lo, obx.hi, P.q_int, obx.lo, obx.hi,
                     P.qg2, obx.lo, obx.hi, P.qaux, qbx.lo, qbx.hi, t2 + 1);
        trans2(ebx[d].lo, ebx[d].hi, d + 1, t1 + 1, t2 + 1, P.qm[d][d], tbx[d][d].lo, tbx[d][d].hi,
               P.ql, obx.lo, obx.hi, P.qp[d][d], tbx[d][d].lo, tbx[d][d].hi, P.qr, obx.lo, obx.hi,
               P.qaux, qbx.lo, qbx.hi, P.ftmp1, obx.lo, obx.hi, P.ftmp2, obx.lo, obx.hi,
               P.qg1, obx.lo, obx.hi, P.qg2, obx.lo, obx.hi, hdtdx[d], hdtdx[t1], hdtdx[t2]);
        compute_flux(ebx[d].lo, ebx[d].hi, P.ql, obx.lo, obx.hi, P.qr, obx.lo, obx.hi, P.flux[d], gebx[d].lo,
                     gebx[d].hi, P.q_int, obx.lo, obx.hi, P.qe[d], gebx[d].lo, gebx[d].hi, P.qaux, qbx.lo, qbx.hi,
                     d + 1);
    }
    for (int d = 0; d < 3; ++d) {
        apply_av(ebx[d].lo, ebx[d].hi, d + 1, dx, P.div, obx.lo, obx.hi, sbp, sbx.lo, sbx.hi, P.flux[d], gebx[d].lo,
                 gebx[d].hi);
        normalize_species_fluxes(ebx[d].lo, ebx[d].hi, P.flux[d], gebx[d].lo, gebx[d].hi);
    }
    // geometry (Cartesian GetFaceArea / GetVolume)
    double area[3] = {dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1]};
    for (int d = 0; d < 3; ++d) {
        long long n = npts(gebx[d]);
        k_fill<<<(unsigned)((n + 255) / 256), 256, 0, castro::stream()>>>(P.area[d], n, area[d]);
    }
    {
        long long n = npts(bx);
        k_fill<<<(unsigned)((n + 255) / 256), 256, 0, castro::stream()>>>(P.vol, n, dx[0] * dx[1] * dx[2]);
    }
    fill_hydro_source(bx.lo, bx.hi, sbp, sbx.lo, sbx.hi, P.q, qbx.lo, qbx.hi, srcp, bx.lo, bx.hi,
                      P.flux[0], gebx[0].lo, gebx[0].hi, P.flux[1], gebx[1].lo, gebx[1].hi,
                      P.flux[2], gebx[2].lo, gebx[2].hi, P.qe[0], gebx[0].lo, gebx[0].hi,
                      P.qe[1], gebx[1].lo, gebx[1].hi, P.qe[2], gebx[2].lo, gebx[2].hi,
                      P.area[0], gebx[0].lo, gebx[0].hi, P.area[1], gebx[1].lo, gebx[1].hi,
                      P.area[2], gebx[2].lo, gebx[2].hi, P.vol, bx.lo, bx.hi, dx, dt);
}

long long plain_scratch_size(const IBox& bx, int nvar)
{
    const int NV = nvar, QV = nvar + 1;
    IBox obx = grow(bx, 1, 1, 1), qbx = grow(bx, NG, NG, NG);
    long long n = npts(qbx) * (QV + NQAUX);
    for (int d = 0; d < 3; ++d) {
        IBox e = bx; e.hi[d] += 1;
        IBox g = grow(e, 1, 1, 1);
        n += npts(g) * (NV + NGDNV + 1);
    }
    n += 18 * npts(obx) * QV;   // qm/qp: tbx boxes are contained in obx-sized boxes plus one face
    n += npts(obx) * (1 + QV + 2 * NV + 2 * NGDNV + 2 * QV);
    n += npts(bx);
    return n + 1024;
}

template <int NS>
void plain_step(castro_sim* s)
{
    SimDev S = s->dev();
    cudaStream_t saved = castro::stream();
    constexpr int NPS = castro_sim::PLAIN_STREAMS;
    // an MFIter loop: its boxes dealt round-robin to the pool's streams, which
    // start after the work issued so far on s->st and end before its next work
    auto fork = [&]() {
        cudaEventRecord(s->pfork, s->st);
        for (int k = 0; k < NPS; ++k) cudaStreamWaitEvent(s->pst[k], s->pfork, 0);
    };
    auto join = [&]() {
        for (int k = 0; k < NPS; ++k) {
            cudaEventRecord(s->pev[k], s->pst[k]);
            cudaStreamWaitEvent(s->st, s->pev[k], 0);
        }
        castro_set_stream(s->st);
    };
    auto box_stream = [&](int i) {
        castro_set_stream(s->pst[i % NPS]);
        return s->pst[i % NPS];
    };
    castro_set_stream(s->st);
    for (int in = 0; in < s->ninst; ++in) {
        InstState hs;
        cudaMemcpyAsync(&hs, s->dstate + in, sizeof hs, cudaMemcpyDeviceToHost, s->st);
        cudaStreamSynchronize(s->st);
        const castro_instance_desc& D = s->desc[in];
        const double* dx = &s->hdx[3 * in];
        const std::vector<int>& boxes = s->inst_boxes[in];
        const int nb = (int)boxes.size();
        // computeInitialDt / computeNewDt, Source/Castro.cpp:175-341
        {
            NvtxRange r("computeNewDt: estTimeStep");
            double big = 1.79769313486231570e+308;
            cudaMemcpyAsync(s->d_dtloc, &big, sizeof big, cudaMemcpyHostToDevice, s->st);
            fork();
            for (int i = 0; i < nb; ++i) {      // each box lowers the one minimum (atomically)
                box_stream(i);
                const BoxDev& B = s->hboxes[boxes[i]];
                estdt(B.lo, B.hi, s->U + B.offU, B.lo, B.hi, dx, s->d_dtloc);
            }
            join();
            double dtl;
            cudaMemcpyAsync(&dtl, s->d_dtloc, sizeof dtl, cudaMemcpyDeviceToHost, s->st);
            cudaStreamSynchronize(s->st);
            dtl *= cfl;
            double dt_0;
            if (hs.steps == 0) dt_0 = std::min(1.0e+100, 0.01 * dtl);
            else dt_0 = std::min(1.0e+100, std::min(dtl, 1.1e0 * hs.dt));
            double eps = 0.001 * dt_0;
            if (hs.stop_time >= 0.0 && (hs.time + dt_0) > (hs.stop_time - eps)) dt_0 = hs.stop_time - hs.time;
            hs.dt = dt_0;
        }
        const double dt = hs.dt;
        cudaMemcpyAsync(s->d_dtbox, &hs.dt, sizeof(double), cudaMemcpyHostToDevice, s->st);
        // Castro::advance, Source/Castro_advance.cpp:32-97
        NvtxRange adv("Castro::advance");
        {
            NvtxRange r("clean_state(S_old)");
            fork();
            for (int i = 0; i < nb; ++i) {
                box_stream(i);
                const BoxDev& B = s->hboxes[boxes[i]];
                plain_clean(s, B.lo, B.hi, s->U + B.offU, B.lo, B.hi);
            }
            join();
        }
        {
            // every box's ghost zones come from its neighbours' cleaned S_old
            NvtxRange r("FillPatch(Sborder) + clean_state(Sborder)");
            fork();
            for (int i = 0; i < nb; ++i) {
                const int b = boxes[i];
                cudaStream_t st = box_stream(i);
                const BoxDev& B = s->hboxes[b];
                long long n = npts_reg(B.lo, B.hi, R_G4, 0);
                k_fill_sborder<NS><<<(unsigned)((n + BLOCK - 1) / BLOCK), BLOCK, 0, st>>>(S, b, s->sb + s->offSb[b]);
                IBox bx{{B.lo[0], B.lo[1], B.lo[2]}, {B.hi[0], B.hi[1], B.hi[2]}};
                IBox g = grow(bx, NG, NG, NG);
                plain_clean(s, g.lo, g.hi, s->sb + s->offSb[b], g.lo, g.hi);
            }
            join();
        }
        {
            // construct_hydro_source, the update (Saxpy) and clean_state(S_new) of
            // post_timestep (Source/Castro.cpp:369) touch the box's own arrays only
            NvtxRange r("construct_hydro_source + Saxpy + clean_state(S_new)");
            fork();
            for (int i = 0; i < nb; ++i) {
                const int b = boxes[i];
                cudaStream_t st = box_stream(i);
                const BoxDev& B = s->hboxes[b];
                IBox bx{{B.lo[0], B.lo[1], B.lo[2]}, {B.hi[0], B.hi[1], B.hi[2]}};
                long long n = npts(bx) * s->nvar;
                cudaMemsetAsync(s->src + s->offSrc[b], 0, n * sizeof(double), st);   // hydro_source.setVal(0)
                if (s->mode == CASTRO_MODE_PLAIN_BOX) {
                    IBox g = grow(bx, NG, NG, NG);
                    castro_construct_hydro_source_box(bx.lo, bx.hi, s->sb + s->offSb[b], g.lo, g.hi,
                                                      s->src + s->offSrc[b], bx.lo, bx.hi, nullptr, nullptr, nullptr,
                                                      D.dom_lo, D.dom_hi, dx, dt);
                } else {
                    plain_hydro_box(s, s->scratch[i % NPS], bx, s->sb + s->offSb[b], s->src + s->offSrc[b], D.dom_lo,
                                    D.dom_hi, dx, dt);
                }
                long long nv = npts_reg(B.lo, B.hi, R_VALID, 0) * s->nvar;
                k_saxpy<<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(s->U + B.offU, s->src + s->offSrc[b], nv, s->d_dtbox);
                plain_clean(s, B.lo, B.hi, s->U + B.offU, B.lo, B.hi);
                plain_clean(s, B.lo, B.hi, s->U + B.offU, B.lo, B.hi);
            }
            join();
        }
        hs.time = hs.time + hs.dt;
        hs.steps += 1;
        hs.dt_last = hs.dt;
        cudaMemcpyAsync(s->dstate + in, &hs, sizeof hs, cudaMemcpyHostToDevice, s->st);
        cudaStreamSynchronize(s->st);
    }
    castro_set_stream(saved);
}

// CASTRO_MODE_PERSISTENT set-up: the stage queues (the batched path's work
// lists), the control block, and the launch shape -- one CTA per resident slot
// of every SM, which the cooperative launch guarantees to be co-resident.
template <int NS>
bool persistent_setup(castro_sim* s)
{
    if (!dalloc(&s->pctl, 1, "persistent control")) return false;
    PersistArgs& P = s->pargs;
    memset(&P, 0, sizeof P);
    P.wl[PS_FRONT] = s->w_valid;  P.n[PS_FRONT] = s->n_valid;
    P.wl[PS_GHOST] = s->w_ghost;  P.n[PS_GHOST] = s->n_ghost;
    P.wl[PS_PREP] = s->w_g1;      P.n[PS_PREP] = s->n_g1;
    P.wl[PS_TRACE] = s->w_trace;  P.n[PS_TRACE] = s->n_trace * (CASTRO_TRACE_SPLIT ? 2 : 1);
    P.trace_items = s->n_trace;
    P.wl[PS_R1] = s->w_tbx;       P.n[PS_R1] = s->n_tbx;
    P.wl[PS_R2] = s->w_r2;        P.n[PS_R2] = s->n_r2;
    P.wl[PS_R3] = s->w_r3;        P.n[PS_R3] = s->n_r3;
    P.wl[PS_UPDATE] = s->w_valid; P.n[PS_UPDATE] = s->n_valid;
    P.ctl = s->pctl;
    P.ninst = s->ninst;
    P.spin_limit = 1LL << 24;
    P.test_stage = -1;
    s->psmem = std::max((size_t)R2Slot<NS>::BYTES, (size_t)R3Slot<NS>::BYTES);
    if (s->psmem > 48 * 1024 &&
        (!cuda_ok(cudaFuncSetAttribute(k_step_persistent<NS, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)s->psmem), "persistent step shared memory") ||
         !cuda_ok(cudaFuncSetAttribute(k_step_persistent<NS, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)s->psmem), "persistent step shared memory")))
        return false;
    // the grid is co-resident for both instantiations (with and without the
    // Coulomb corrections): the smaller of their occupancies
    int dev = 0, nsm = 0, coop = 0, per_sm = 0, per_sm_c = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "device") ||
        !cuda_ok(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count") ||
        !cuda_ok(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev), "cooperative launch") ||
        !cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_step_persistent<NS, false>, BLOCK, s->psmem),
                 "occupancy") ||
        !cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_c, k_step_persistent<NS, true>, BLOCK, s->psmem),
                 "occupancy"))
        return false;
    per_sm = std::min(per_sm, per_sm_c);
    if (!coop || per_sm < 1) {
        set_error(CASTRO_ERR_CUDA, "castro_sim_create: the device cannot run the persistent step (no cooperative launch)");
        return false;
    }
    s->pgrid = nsm * per_sm;
    return true;
}

template <int NS>
void persistent_launch(castro_sim* s)
{
    SimDev S = s->dev();
    PersistArgs P = s->pargs;
    void* args[] = {&S, &P};
    cuda_ok(cudaMemsetAsync(s->pctl, 0, sizeof(PersistCtl), s->st), "persistent queue reset");
    const void* kern = coulomb_on() ? (const void*)k_step_persistent<NS, true> : (const void*)k_step_persistent<NS, false>;
    cuda_ok(cudaLaunchCooperativeKernel(kern, dim3(s->pgrid), dim3(BLOCK), args, s->psmem, s->st),
            "persistent step launch");
}

template <int NS>
int persistent_step(castro_sim* s)
{
    if (s->failed) {
        set_error(CASTRO_ERR_TIMEOUT, "castro_sim_step: an earlier step ran out of a device wait; the state is void");
        return CASTRO_ERR_TIMEOUT;
    }
    if (!s->gexec && !s->pdirect) {
        // one graph per step: the queue reset and the cooperative launch
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        bool ok = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            persistent_launch<NS>(s);
            ok = cudaStreamEndCapture(s->st, &g) == cudaSuccess && g &&
                 cudaGraphInstantiate(&ge, g, 0) == cudaSuccess && castro_last_error() == 0;
        }
        if (ok) {
            s->graph = g;
            s->gexec = ge;
            s->graph_coul = coulomb_on();
        } else {
            if (ge) cudaGraphExecDestroy(ge);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            castro_clear_error();
            s->pdirect = true;
        }
    }
    if (s->pdirect) persistent_launch<NS>(s);
    else cuda_ok(cudaGraphLaunch(s->gexec, s->st), "graph launch");
    s->launches = 1;
    return castro_last_error();
}

template <int NS>
int step_impl(castro_sim* s)
{
    if (s->mode == CASTRO_MODE_PLAIN || s->mode == CASTRO_MODE_PLAIN_BOX) {
        plain_step<NS>(s);
        // per box: estdt, fill_sborder, Saxpy and 4 x 4 clean kernels, plus construct_hydro_source's
        // 36 per-routine launches or the fused box path's kernels (prim, prep, trace (x2), riemann1-3, source)
        const int per_box = 19 + (s->mode == CASTRO_MODE_PLAIN ? 36 : 6 + (CASTRO_TRACE_SPLIT ? 2 : 1));
        s->launches = 0;
        for (int in = 0; in < s->ninst; ++in) s->launches += per_box * (int)s->inst_boxes[in].size();
        return castro_last_error();
    }
    if (!s->dt_ready) {
        initial_dt_kernels<NS>(s);
        s->dt_ready = true;
    }
    if (s->gexec && s->graph_coul != coulomb_on()) {
        // the Coulomb setting changed since the step was captured: capture again
        cudaGraphExecDestroy(s->gexec);
        cudaGraphDestroy(s->graph);
        s->gexec = nullptr;
        s->graph = nullptr;
    }
    if (s->mode == CASTRO_MODE_PERSISTENT) return persistent_step<NS>(s);
    if (!s->gexec) {
        if (!cuda_ok(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal), "begin capture")) return castro_last_error();
        batched_step_kernels<NS>(s);
        if (!cuda_ok(cudaStreamEndCapture(s->st, &s->graph), "end capture")) return castro_last_error();
        if (!cuda_ok(cudaGraphInstantiate(&s->gexec, s->graph, 0), "graph instantiate")) return castro_last_error();
        s->graph_coul = coulomb_on();
    }
    cuda_ok(cudaGraphLaunch(s->gexec, s->st), "graph launch");
    s->launches = 9 + (CASTRO_TRACE_SPLIT ? 1 : 0) - (s->r23 ? 1 : 0);
    return castro_last_error();
}

// The BoxArray and geometry of one instance, checked before anything is
// allocated: a non-empty domain with cubic zones (the reference aborts on
// dx != dy != dz, Source/Castro.cpp:95-100), a known boundary condition, and
// non-empty boxes inside the domain that cover it without overlapping (the
// owner map then assigns every zone exactly once).  Returns false with msg set.
bool validate_instance(const castro_instance_desc& D, int in, char* msg, size_t nmsg)
{
    long long dvol = 1;
    for (int d = 0; d < 3; ++d) {
        if (D.dom_hi[d] < D.dom_lo[d]) { snprintf(msg, nmsg, "castro_sim_create: instance %d: empty domain", in); return false; }
        if (!(D.probhi[d] > D.problo[d])) { snprintf(msg, nmsg, "castro_sim_create: instance %d: probhi <= problo", in); return false; }
        dvol *= (long long)(D.dom_hi[d] - D.dom_lo[d] + 1);
    }
    double dx[3];
    for (int d = 0; d < 3; ++d) dx[d] = (D.probhi[d] - D.problo[d]) / (double)(D.dom_hi[d] - D.dom_lo[d] + 1);
    if (fabs(dx[0] - dx[1]) > 1.e-13 * dx[0] || fabs(dx[0] - dx[2]) > 1.e-13 * dx[0]) {
        snprintf(msg, nmsg, "castro_sim_create: instance %d: zones are not cubic (dx != dy != dz)", in);
        return false;
    }
    if (D.bc != CASTRO_BC_PERIODIC && D.bc != CASTRO_BC_OUTFLOW) {
        snprintf(msg, nmsg, "castro_sim_create: instance %d: unknown boundary condition %d", in, D.bc);
        return false;
    }
    if (D.nbox < 1 || !D.box_lo || !D.box_hi) { snprintf(msg, nmsg, "castro_sim_create: instance %d: no boxes", in); return false; }
    long long vol = 0;
    for (int b = 0; b < D.nbox; ++b) {
        long long v = 1;
        for (int d = 0; d < 3; ++d) {
            const int l = D.box_lo[3 * b + d], h = D.box_hi[3 * b + d];
            if (h < l) { snprintf(msg, nmsg, "castro_sim_create: instance %d box %d: empty box", in, b); return false; }
            if (l < D.dom_lo[d] || h > D.dom_hi[d]) {
                snprintf(msg, nmsg, "castro_sim_create: instance %d box %d: outside the domain", in, b);
                return false;
            }
            v *= (long long)(h - l + 1);
        }
        vol += v;
    }
    if (vol != dvol) {
        snprintf(msg, nmsg, "castro_sim_create: instance %d: boxes hold %lld zones, the domain %lld (overlap or gap)",
                 in, vol, dvol);
        return false;
    }
    return true;
}

}  // namespace

// ===========================================================================
// extern "C"
// ===========================================================================
extern "C" {

castro_sim* castro_sim_create(int ninst, const castro_instance_desc* desc, int mode)
{
    if (!table_ready()) { set_error(CASTRO_ERR_NO_TABLE, "castro_sim_create: eos_init has not run"); return nullptr; }
    if (ninst < 1 || !desc) { set_error(CASTRO_ERR_ARG, "castro_sim_create: no instances"); return nullptr; }
    if (mode != CASTRO_MODE_PLAIN && mode != CASTRO_MODE_BATCHED && mode != CASTRO_MODE_PLAIN_BOX &&
        mode != CASTRO_MODE_PERSISTENT) {
        set_error(CASTRO_ERR_ARG, "castro_sim_create: unknown mode");
        return nullptr;
    }
    int ns = nspec();
    if (ns != 2 && ns != 13) { set_error(CASTRO_ERR_NSPEC, "castro_sim_create: nspec"); return nullptr; }
    for (int in = 0; in < ninst; ++in) {
        char msg[200];
        if (!validate_instance(desc[in], in, msg, sizeof msg)) { set_error(CASTRO_ERR_ARG, msg); return nullptr; }
    }
    if (!(ns == 2 ? set_kernel_attributes<2>() : set_kernel_attributes<13>())) return nullptr;
    castro_sim* s = new castro_sim();
    s->mode = mode;
    s->ns = ns;
    s->nvar = 7 + ns;
    s->ninst = ninst;
    s->desc.assign(desc, desc + ninst);
    cuda_ok(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking), "stream create");
    cuda_ok(cudaStreamCreateWithFlags(&s->st2, cudaStreamNonBlocking), "stream create");
    cuda_ok(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming), "event create");
    cuda_ok(cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming), "event create");
    // the EOS table's L2 window on both streams; stream capture copies it into the step graph's nodes
    apply_table_l2_window(s->st);
    apply_table_l2_window(s->st2);
    const int NQS = 6 + ns, NTF = 7 + ns, NQF = 8 + ns, NV = 7 + ns;

    long long oU = 0, oUb = 0, oQ = 0, oDiv = 0, oTr = 0, oF1 = 0, oF2 = 0, oFx = 0;
    std::vector<int> owner_all;
    for (int in = 0; in < ninst; ++in) {
        const castro_instance_desc& D = desc[in];
        InstDev I;
        memset(&I, 0, sizeof I);
        for (int d = 0; d < 3; ++d) {
            I.dom_lo[d] = D.dom_lo[d];
            I.dom_hi[d] = D.dom_hi[d];
            I.dx[d] = (D.probhi[d] - D.problo[d]) / (double)(D.dom_hi[d] - D.dom_lo[d] + 1);
            s->hdx.push_back(I.dx[d]);
        }
        I.bc = D.bc;
        // owner map granularity: gcd of every box edge offset
        int g = 0;
        for (int d = 0; d < 3; ++d) g = std::gcd(g, D.dom_hi[d] - D.dom_lo[d] + 1);
        std::vector<int> ids;
        for (int b = 0; b < D.nbox; ++b)
            for (int d = 0; d < 3; ++d) {
                g = std::gcd(g, D.box_lo[3 * b + d] - D.dom_lo[d]);
                g = std::gcd(g, D.box_hi[3 * b + d] + 1 - D.dom_lo[d]);
            }
        if (g <= 0) g = 1;
        I.g = g;
        for (int d = 0; d < 3; ++d) I.on[d] = (D.dom_hi[d] - D.dom_lo[d] + 1) / g;
        I.owner_off = (long long)owner_all.size();
        // The instance's domain box: Q and Sborder over grow(domain,4) / grow(domain,1),
        // and the stage arrays of prep, trace and the three Riemann kernels over the
        // domain's regions, so that each face is computed once for the whole domain
        BoxDev P;
        memset(&P, 0, sizeof P);
        for (int d = 0; d < 3; ++d) { P.lo[d] = I.dom_lo[d]; P.hi[d] = I.dom_hi[d]; }
        P.inst = in;
        P.offQ = oQ; oQ += npts_reg(P.lo, P.hi, R_G4, 0) * NQF;
        P.offUb = oUb; oUb += npts_reg(P.lo, P.hi, R_G1, 0) * NV;
        P.offDiv = oDiv; oDiv += npts_reg(P.lo, P.hi, R_G1, 0) * 2;   // divu, flatn
        for (int d = 0; d < 3; ++d) {
            P.offTr[d] = oTr; oTr += npts_reg(P.lo, P.hi, R_TBX, 4 * d) * 2 * NQS;
            P.offF1[d] = oF1; oF1 += npts_reg(P.lo, P.hi, R_TBX, 4 * d) * NTF;
            P.offFx[d] = oFx; oFx += npts_reg(P.lo, P.hi, R_EBX, d) * (NV + 1);
        }
        for (int a = 0; a < 3; ++a)
            for (int bb = 0; bb < 3; ++bb)
                if (a != bb) { P.offF2[pair_index(a, bb)] = oF2; oF2 += npts_reg(P.lo, P.hi, R_TBX, 3 * a + bb) * NTF; }
        size_t nown = (size_t)I.on[0] * I.on[1] * I.on[2];
        owner_all.resize(owner_all.size() + nown, -1);
        for (int b = 0; b < D.nbox; ++b) {
            BoxDev B;
            memset(&B, 0, sizeof B);
            for (int d = 0; d < 3; ++d) { B.lo[d] = D.box_lo[3 * b + d]; B.hi[d] = D.box_hi[3 * b + d]; }
            B.inst = in;
            B.offU = oU; oU += npts_reg(B.lo, B.hi, R_VALID, 0) * NV;
            // the instance's arrays; the stage-array offsets describe the domain's
            // regions and are read through the domain box (a box's own only when
            // it is the whole domain)
            B.offUb = P.offUb;
            B.offQ = P.offQ;
            B.offDiv = P.offDiv;
            for (int d = 0; d < 3; ++d) { B.offTr[d] = P.offTr[d]; B.offF1[d] = P.offF1[d]; B.offFx[d] = P.offFx[d]; }
            for (int q = 0; q < 6; ++q) B.offF2[q] = P.offF2[q];
            if (b == 0) P.offU = B.offU;
            int gid = (int)s->hboxes.size();
            ids.push_back(gid);
            s->hboxes.push_back(B);
            bool overlap = false;
            for (int k = B.lo[2]; k <= B.hi[2]; k += g)
                for (int j = B.lo[1]; j <= B.hi[1]; j += g)
                    for (int i = B.lo[0]; i <= B.hi[0]; i += g) {
                        int& o = owner_all[I.owner_off + (i - D.dom_lo[0]) / g +
                                           (long long)I.on[0] * ((j - D.dom_lo[1]) / g + (long long)I.on[1] * ((k - D.dom_lo[2]) / g))];
                        overlap = overlap || o >= 0;
                        o = gid;
                    }
            if (overlap) { set_error(CASTRO_ERR_ARG, "castro_sim_create: boxes overlap"); castro_sim_destroy(s); return nullptr; }
        }
        for (size_t m = I.owner_off; m < owner_all.size(); ++m)
            if (owner_all[m] < 0) { set_error(CASTRO_ERR_ARG, "castro_sim_create: boxes do not cover the domain"); castro_sim_destroy(s); return nullptr; }
        s->inst_boxes.push_back(ids);
        s->hinst.push_back(I);
        s->hdom.push_back(P);
    }
    s->nU = oU;
    bool ok = dalloc(&s->dboxes, s->hboxes.size(), "boxes") && dalloc(&s->ddom, s->hdom.size(), "domain boxes") &&
              dalloc(&s->dinst, s->hinst.size(), "instances") &&
              dalloc(&s->dstate, ninst, "state") && dalloc(&s->downer, owner_all.size(), "owner") &&
              dalloc(&s->U, oU, "U") && dalloc(&s->d_dtloc, 1, "dtloc") && dalloc(&s->d_dtbox, 1, "dtbox");
    if (ok) {
        cuda_ok(cudaMemcpy(s->dboxes, s->hboxes.data(), s->hboxes.size() * sizeof(BoxDev), cudaMemcpyHostToDevice), "boxes");
        cuda_ok(cudaMemcpy(s->ddom, s->hdom.data(), s->hdom.size() * sizeof(BoxDev), cudaMemcpyHostToDevice), "domain boxes");
        cuda_ok(cudaMemcpy(s->dinst, s->hinst.data(), s->hinst.size() * sizeof(InstDev), cudaMemcpyHostToDevice), "inst");
        cuda_ok(cudaMemcpy(s->downer, owner_all.data(), owner_all.size() * sizeof(int), cudaMemcpyHostToDevice), "owner");
        std::vector<InstState> hs(ninst);
        for (int in = 0; in < ninst; ++in) {
            memset(&hs[in], 0, sizeof(InstState));
            hs[in].dt_est = 1.79769313486231570e+308;
            hs[in].stop_time = desc[in].stop_time;
        }
        cuda_ok(cudaMemcpy(s->dstate, hs.data(), ninst * sizeof(InstState), cudaMemcpyHostToDevice), "state");
    }
    if (ok && (mode == CASTRO_MODE_BATCHED || mode == CASTRO_MODE_PERSISTENT)) {
        ok = dalloc(&s->Ub, oUb, "Ub") && dalloc(&s->Q, oQ, "Q") && dalloc(&s->Div, oDiv, "Div") &&
             dalloc(&s->Tr, oTr, "Tr") && dalloc(&s->F1, oF1, "F1") && dalloc(&s->F2, oF2, "F2") && dalloc(&s->Fx, oFx, "Fx");
        build_work(s->hboxes, R_VALID, 1, -1, &s->w_valid, &s->n_valid);
        build_work(s->hboxes, R_G4, 1, -1, &s->w_g4, &s->n_g4);
        // the stage kernels walk the domain boxes (launched with dev_dom())
        build_work(s->hdom, R_G1, 1, -1, &s->w_g1, &s->n_g1);
        build_work(s->hdom, R_SEG, 3, -1, &s->w_trace, &s->n_trace);
        build_work(s->hdom, R_TBX, 3, 0, &s->w_tbx, &s->n_tbx);
        build_work(s->hdom, R_EBX, 3, -1, &s->w_ebx, &s->n_ebx);
        build_work(s->hdom, R_TBX, 3, 0, &s->w_r2, &s->n_r2, CASTRO_R2_ROWS);
        build_work(s->hdom, R_EBX, 3, -1, &s->w_r3, &s->n_r3, CASTRO_R3_ROWS);
        build_ghost_work(s);
        if (ok && ns == 2 && column_tiles_on() && mode == CASTRO_MODE_BATCHED) ok = build_r23_work(s);
        if (ok && mode == CASTRO_MODE_PERSISTENT) ok = ns == 2 ? persistent_setup<2>(s) : persistent_setup<13>(s);
    }
    if (ok && (mode == CASTRO_MODE_PLAIN || mode == CASTRO_MODE_PLAIN_BOX)) {
        long long nsb = 0, nsrc = 0, mx = 0;
        for (const BoxDev& B : s->hboxes) {
            s->offSb.push_back(nsb);
            nsb += npts_reg(B.lo, B.hi, R_G4, 0) * NV;
            s->offSrc.push_back(nsrc);
            nsrc += npts_reg(B.lo, B.hi, R_VALID, 0) * NV;
            IBox bx{{B.lo[0], B.lo[1], B.lo[2]}, {B.hi[0], B.hi[1], B.hi[2]}};
            mx = std::max(mx, plain_scratch_size(bx, NV));
        }
        s->scratch_n = mx;
        ok = dalloc(&s->sb, nsb, "Sborder") && dalloc(&s->src, nsrc, "hydro_source");
        for (int k = 0; ok && k < castro_sim::PLAIN_STREAMS; ++k) {
            ok = cuda_ok(cudaStreamCreateWithFlags(&s->pst[k], cudaStreamNonBlocking), "stream create") &&
                 cuda_ok(cudaEventCreateWithFlags(&s->pev[k], cudaEventDisableTiming), "event create") &&
                 (mode == CASTRO_MODE_PLAIN_BOX || dalloc(&s->scratch[k], mx, "scratch"));
        }
        ok = ok && cuda_ok(cudaEventCreateWithFlags(&s->pfork, cudaEventDisableTiming), "event create");
        // the work list of the valid region is still used by estdt of the sim API
        build_work(s->hboxes, R_VALID, 1, -1, &s->w_valid, &s->n_valid);
    }
    s->probs.resize(ninst);
    for (int in = 0; in < ninst; ++in) s->probs[in] = desc[in].prob;
    if (ok && eos_fail_counter())
        cuda_ok(cudaMemcpy(&s->eos_seen, eos_fail_counter(), sizeof s->eos_seen, cudaMemcpyDeviceToHost), "eos counter");
    s->eos_base = s->eos_seen;
    if (!ok || castro_last_error()) { castro_sim_destroy(s); return nullptr; }
    return s;
}

void castro_sim_destroy(castro_sim* s)
{
    if (!s) return;
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->graph) cudaGraphDestroy(s->graph);
    void* ptrs[] = {s->dboxes, s->ddom, s->dinst, s->dstate, s->downer, s->U, s->Ub, s->Q, s->Div, s->Tr, s->F1, s->F2, s->Fx,
                    s->w_valid, s->w_g4, s->w_g1, s->w_trace, s->w_tbx, s->w_ebx, s->w_r2, s->w_r3, s->w_ghost, s->sb, s->src,
                    s->d_dtloc, s->d_dtbox, s->pctl, s->w_r23};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    for (int k = 0; k < castro_sim::PLAIN_STREAMS; ++k) {
        if (s->scratch[k]) cudaFree(s->scratch[k]);
        if (s->pst[k]) cudaStreamDestroy(s->pst[k]);
        if (s->pev[k]) cudaEventDestroy(s->pev[k]);
    }
    if (s->pfork) cudaEventDestroy(s->pfork);
    if (s->st) cudaStreamDestroy(s->st);
    if (s->st2) cudaStreamDestroy(s->st2);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    delete s;
}

int castro_sim_nbox(const castro_sim* s, int inst) { return (int)s->inst_boxes[inst].size(); }

size_t castro_sim_box_size(const castro_sim* s, int inst, int b)
{
    const BoxDev& B = s->hboxes[s->inst_boxes[inst][b]];
    return (size_t)npts_reg(B.lo, B.hi, R_VALID, 0) * s->nvar;
}

double* castro_sim_box_state(castro_sim* s, int inst, int b)
{
    return s->U + s->hboxes[s->inst_boxes[inst][b]].offU;
}

size_t castro_sim_total_size(const castro_sim* s) { return (size_t)s->nU; }

int castro_sim_init_data(castro_sim* s)
{
    NvtxRange r("castro_sim_init_data: Castro::initData");
    cudaStream_t saved = castro::stream();
    castro_set_stream(s->st);
    for (int in = 0; in < s->ninst; ++in) {
        castro_set_problem(&s->probs[in]);
        const castro_instance_desc& D = s->desc[in];
        for (int b : s->inst_boxes[in]) {
            const BoxDev& B = s->hboxes[b];
            initdata(B.lo, B.hi, s->U + B.offU, B.lo, B.hi, &s->hdx[3 * in], D.problo, D.probhi);
        }
    }
    castro_set_stream(saved);
    cuda_ok(cudaStreamSynchronize(s->st), "init_data");
    return castro_last_error();
}

int castro_sim_upload(castro_sim* s, const double* host)
{
    cuda_ok(cudaMemcpyAsync(s->U, host, (size_t)s->nU * sizeof(double), cudaMemcpyHostToDevice, s->st), "upload");
    return castro_last_error();
}

int castro_sim_download(castro_sim* s, double* host)
{
    cuda_ok(cudaMemcpyAsync(host, s->U, (size_t)s->nU * sizeof(double), cudaMemcpyDeviceToHost, s->st), "download");
    return castro_last_error();
}

int castro_sim_step(castro_sim* s)
{
    NvtxRange r(s->mode == CASTRO_MODE_BATCHED      ? "castro_sim_step: Castro::advance (batched step graph)"
                : s->mode == CASTRO_MODE_PERSISTENT ? "castro_sim_step: Castro::advance (one persistent launch)"
                                                     : "castro_sim_step: Castro::advance (per-box sequence)");
    if (s->ns == 2) return step_impl<2>(s);
    return step_impl<13>(s);
}

int castro_sim_run(castro_sim* s, int nsteps)
{
    for (int n = 0; n < nsteps; ++n) {
        int e = castro_sim_step(s);
        if (e) return e;
    }
    return castro_last_error();
}

int castro_sim_run_host(castro_sim* s, const double* host_in, int nsteps, double* host_out)
{
    castro_sim_upload(s, host_in);
    castro_sim_run(s, nsteps);
    castro_sim_download(s, host_out);
    cuda_ok(cudaStreamSynchronize(s->st), "run_host");
    return castro_last_error();
}

int castro_sim_sync(castro_sim* s)
{
    if (!cuda_ok(cudaStreamSynchronize(s->st), "sync")) return castro_last_error();
    if (s->pctl && !s->failed) {
        PersistCtl c;
        if (cuda_ok(cudaMemcpy(&c, s->pctl, sizeof c, cudaMemcpyDeviceToHost), "persistent control") && c.error != 0) {
            static const char* stage[PS_COUNT] = {"front", "ghost", "prep", "trace", "riemann1", "riemann2", "riemann3",
                                                  "update"};
            char msg[200];
            snprintf(msg, sizeof msg, "castro_sim: the grid-barrier wait after stage %s ran out of its limit; the step "
                     "is void", c.error >= 1 && c.error <= PS_COUNT ? stage[c.error - 1] : "?");
            s->failed = true;
            set_error(CASTRO_ERR_TIMEOUT, msg);
            return castro_last_error();
        }
    }
    // an EOS Newton iteration that reached its 100-iteration limit (a NaN or
    // otherwise unphysical state) is silent in the reference; here it is an error
    unsigned long long v = 0;
    if (eos_fail_counter() && cuda_ok(cudaMemcpy(&v, eos_fail_counter(), sizeof v, cudaMemcpyDeviceToHost), "eos counter") &&
        v > s->eos_seen) {
        char msg[160];
        snprintf(msg, sizeof msg, "castro_sim: %llu EOS Newton solves did not converge (non-finite or unphysical state)",
                 v - s->eos_seen);
        s->eos_seen = v;
        set_error(CASTRO_ERR_EOS, msg);
    }
    return castro_last_error();
}

static InstState read_state(castro_sim* s, int inst)
{
    InstState h;
    memset(&h, 0, sizeof h);
    cudaStreamSynchronize(s->st);
    cuda_ok(cudaMemcpy(&h, s->dstate + inst, sizeof h, cudaMemcpyDeviceToHost), "read state");
    return h;
}

double castro_sim_time(castro_sim* s, int inst) { return read_state(s, inst).time; }
double castro_sim_dt(castro_sim* s, int inst)
{
    InstState h = read_state(s, inst);
    return h.steps > 0 ? h.dt_last : h.dt;
}
int castro_sim_steps(castro_sim* s, int inst) { return read_state(s, inst).steps; }

double castro_sim_est_time_step(castro_sim* s, int inst)
{
    NvtxRange r("castro_sim_est_time_step: Castro::estTimeStep");
    double big = 1.79769313486231570e+308;
    cuda_ok(cudaMemcpyAsync(s->d_dtloc, &big, sizeof big, cudaMemcpyHostToDevice, s->st), "est");
    cudaStream_t saved = castro::stream();
    castro_set_stream(s->st);
    for (int b : s->inst_boxes[inst]) {
        const BoxDev& B = s->hboxes[b];
        estdt(B.lo, B.hi, s->U + B.offU, B.lo, B.hi, &s->hdx[3 * inst], s->d_dtloc);
    }
    castro_set_stream(saved);
    double dt;
    cuda_ok(cudaMemcpyAsync(&dt, s->d_dtloc, sizeof dt, cudaMemcpyDeviceToHost, s->st), "est read");
    cudaStreamSynchronize(s->st);
    return dt * cfl;
}

// AMReX native plotfile ("HyperCLaw-V1.1") of one instance's level: Header,
// Level_0/Cell_H (the MultiFab header with every box, its offset in the data
// file and per-component minima and maxima) and Level_0/Cell_D_00000 (every
// FAB: a text header line, then the values in Fortran order, component
// slowest, little-endian IEEE doubles).  Components are named as Castro's
// state: density, xmom, ymom, zmom, rho_E, rho_e, Temp, rho_<species>.
int castro_sim_write_plotfile(castro_sim* s, int inst, const char* dir)
{
    NvtxRange r("castro_sim_write_plotfile");
    if (!s || !dir || inst < 0 || inst >= s->ninst) {
        set_error(CASTRO_ERR_ARG, "castro_sim_write_plotfile: arguments");
        return CASTRO_ERR_ARG;
    }
    const castro_instance_desc& D = s->desc[inst];
    InstState hs;
    if (!cuda_ok(cudaMemcpyAsync(&hs, s->dstate + inst, sizeof hs, cudaMemcpyDeviceToHost, s->st), "plotfile state") ||
        !cuda_ok(cudaStreamSynchronize(s->st), "plotfile sync"))
        return castro_last_error();
    const std::string root(dir), lev = root + "/Level_0";
    mkdir(root.c_str(), 0755);
    mkdir(lev.c_str(), 0755);
    const int nc = s->nvar;
    std::vector<std::string> names = {"density", "xmom", "ymom", "zmom", "rho_E", "rho_e", "Temp"};
    for (int n = 0; n < s->ns; ++n) names.push_back("rho_spec" + std::to_string(n));
    const double* dx = &s->hdx[3 * inst];
    const std::vector<int>& boxes = s->inst_boxes[inst];

    // data file: one FAB per box
    std::string dname = lev + "/Cell_D_00000";
    FILE* fd = fopen(dname.c_str(), "wb");
    if (!fd) {
        set_error(CASTRO_ERR_ARG, ("castro_sim_write_plotfile: cannot write " + dname).c_str());
        return CASTRO_ERR_ARG;
    }
    std::vector<long long> offsets;
    std::vector<std::vector<double>> mins, maxs;
    std::vector<double> h;
    for (int b : boxes) {
        const BoxDev& B = s->hboxes[b];
        long long np = npts_reg(B.lo, B.hi, R_VALID, 0);
        h.resize((size_t)(np * nc));
        if (!cuda_ok(cudaMemcpy(h.data(), s->U + B.offU, h.size() * sizeof(double), cudaMemcpyDeviceToHost),
                     "plotfile read")) {
            fclose(fd);
            return castro_last_error();
        }
        offsets.push_back((long long)ftell(fd));
        fprintf(fd, "FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))((%d,%d,%d) (%d,%d,%d) (0,0,0)) %d\n",
                B.lo[0], B.lo[1], B.lo[2], B.hi[0], B.hi[1], B.hi[2], nc);
        fwrite(h.data(), sizeof(double), h.size(), fd);
        std::vector<double> mn(nc), mx(nc);
        for (int n = 0; n < nc; ++n) {
            const double* c = h.data() + (size_t)np * n;
            mn[n] = *std::min_element(c, c + np);
            mx[n] = *std::max_element(c, c + np);
        }
        mins.push_back(mn);
        maxs.push_back(mx);
    }
    fclose(fd);

    // MultiFab header
    FILE* fh = fopen((lev + "/Cell_H").c_str(), "w");
    if (!fh) { set_error(CASTRO_ERR_ARG, "castro_sim_write_plotfile: Cell_H"); return CASTRO_ERR_ARG; }
    fprintf(fh, "1\n0\n%d\n0\n(%d 0\n", nc, (int)boxes.size());
    for (int b : boxes) {
        const BoxDev& B = s->hboxes[b];
        fprintf(fh, "((%d,%d,%d) (%d,%d,%d) (0,0,0))\n", B.lo[0], B.lo[1], B.lo[2], B.hi[0], B.hi[1], B.hi[2]);
    }
    fprintf(fh, ")\n%d\n", (int)boxes.size());
    for (long long o : offsets) fprintf(fh, "FabOnDisk: Cell_D_00000 %lld\n", o);
    for (int pass = 0; pass < 2; ++pass) {
        fprintf(fh, "\n%d,%d\n", (int)boxes.size(), nc);
        for (const auto& v : (pass == 0 ? mins : maxs)) {
            for (double x : v) fprintf(fh, "%.17g,", x);
            fprintf(fh, "\n");
        }
    }
    fclose(fh);

    // plotfile header
    FILE* fp = fopen((root + "/Header").c_str(), "w");
    if (!fp) { set_error(CASTRO_ERR_ARG, "castro_sim_write_plotfile: Header"); return CASTRO_ERR_ARG; }
    fprintf(fp, "HyperCLaw-V1.1\n%d\n", nc);
    for (const auto& nm : names) fprintf(fp, "%s\n", nm.c_str());
    fprintf(fp, "3\n%.17g\n0\n", hs.time);
    fprintf(fp, "%.17g %.17g %.17g\n", D.problo[0], D.problo[1], D.problo[2]);
    fprintf(fp, "%.17g %.17g %.17g\n", D.probhi[0], D.probhi[1], D.probhi[2]);
    fprintf(fp, "\n((%d,%d,%d) (%d,%d,%d) (0,0,0))\n", D.dom_lo[0], D.dom_lo[1], D.dom_lo[2], D.dom_hi[0], D.dom_hi[1],
            D.dom_hi[2]);
    fprintf(fp, "%d\n%.17g %.17g %.17g\n0\n0\n", hs.steps, dx[0], dx[1], dx[2]);
    fprintf(fp, "0 %d %.17g\n%d\n", (int)boxes.size(), hs.time, hs.steps);
    for (int b : boxes) {
        const BoxDev& B = s->hboxes[b];
        for (int d = 0; d < 3; ++d)
            fprintf(fp, "%.17g %.17g\n", D.problo[d] + B.lo[d] * dx[d], D.problo[d] + (B.hi[d] + 1) * dx[d]);
    }
    fprintf(fp, "Level_0/Cell\n");
    fclose(fp);
    return castro_last_error();
}

// Checkpoint / restart of every instance (the reference registers State_Type for
// AMReX checkpoints, Source/Castro_setup.cpp:50-53).  dir/Header is text: the
// format line, nspec, nvar, then per instance its domain, BoxArray, time,
// completed steps, last dt and stop time (floating-point values as C99
// hexadecimal, so they round-trip exactly); dir/State_<n> holds instance n's box
// FABs in box order as raw doubles (the castro_sim_download layout).
int castro_sim_write_checkpoint(castro_sim* s, const char* dir)
{
    NvtxRange r("castro_sim_write_checkpoint");
    if (!s || !dir) { set_error(CASTRO_ERR_ARG, "castro_sim_write_checkpoint: arguments"); return CASTRO_ERR_ARG; }
    if (!cuda_ok(cudaStreamSynchronize(s->st), "checkpoint sync")) return castro_last_error();
    mkdir(dir, 0755);
    const std::string root(dir);
    FILE* fp = fopen((root + "/Header").c_str(), "w");
    if (!fp) { set_error(CASTRO_ERR_IO, ("castro_sim_write_checkpoint: cannot write " + root + "/Header").c_str()); return CASTRO_ERR_IO; }
    fprintf(fp, "castro_b200_checkpoint 1\nnspec %d\nnvar %d\nninst %d\n", s->ns, s->nvar, s->ninst);
    std::vector<double> h;
    bool ok = true;
    for (int in = 0; in < s->ninst && ok; ++in) {
        const castro_instance_desc& D = s->desc[in];
        InstState hs;
        ok = cuda_ok(cudaMemcpy(&hs, s->dstate + in, sizeof hs, cudaMemcpyDeviceToHost), "checkpoint state");
        // the plain mode keeps the last step's dt in dt as well
        fprintf(fp, "instance %d\ndomain %d %d %d %d %d %d\nnbox %d\n", in, D.dom_lo[0], D.dom_lo[1], D.dom_lo[2],
                D.dom_hi[0], D.dom_hi[1], D.dom_hi[2], (int)s->inst_boxes[in].size());
        for (int b : s->inst_boxes[in]) {
            const BoxDev& B = s->hboxes[b];
            fprintf(fp, "box %d %d %d %d %d %d\n", B.lo[0], B.lo[1], B.lo[2], B.hi[0], B.hi[1], B.hi[2]);
        }
        fprintf(fp, "time %a\nsteps %d\ndt_last %a\nstop_time %a\n", hs.time, hs.steps, hs.dt_last, hs.stop_time);
        char name[32];
        snprintf(name, sizeof name, "/State_%05d", in);
        FILE* fd = fopen((root + name).c_str(), "wb");
        if (!fd) { set_error(CASTRO_ERR_IO, ("castro_sim_write_checkpoint: cannot write " + root + name).c_str()); ok = false; break; }
        for (int b : s->inst_boxes[in]) {
            const BoxDev& B = s->hboxes[b];
            h.resize((size_t)(npts_reg(B.lo, B.hi, R_VALID, 0) * s->nvar));
            ok = cuda_ok(cudaMemcpy(h.data(), s->U + B.offU, h.size() * sizeof(double), cudaMemcpyDeviceToHost), "checkpoint read");
            if (ok && fwrite(h.data(), sizeof(double), h.size(), fd) != h.size()) {
                set_error(CASTRO_ERR_IO, "castro_sim_write_checkpoint: short write");
                ok = false;
            }
            if (!ok) break;
        }
        fclose(fd);
    }
    fprintf(fp, "end\n");
    if (fclose(fp) != 0 && ok) { set_error(CASTRO_ERR_IO, "castro_sim_write_checkpoint: cannot close Header"); ok = false; }
    return castro_last_error();
}

}  // extern "C"

namespace {

bool ck_expect(FILE* fp, const char* key)
{
    char w[64];
    return fscanf(fp, "%63s", w) == 1 && strcmp(w, key) == 0;
}

template <int NS>
void restart_dt_kernels(castro_sim* s)
{
    SimDev S = s->dev();
    CASTRO_EOS_LAUNCH(k_estdt_state, NS, s->n_valid, BLOCK, 0, s->st, S, s->w_valid);
    k_dt<<<(s->ninst + 63) / 64, 64, 0, s->st>>>(S, s->ninst, DT_RESTART);
}

}  // namespace

extern "C" {

int castro_sim_read_checkpoint(castro_sim* s, const char* dir)
{
    NvtxRange r("castro_sim_read_checkpoint");
    if (!s || !dir) { set_error(CASTRO_ERR_ARG, "castro_sim_read_checkpoint: arguments"); return CASTRO_ERR_ARG; }
    const std::string root(dir);
    FILE* fp = fopen((root + "/Header").c_str(), "r");
    if (!fp) { set_error(CASTRO_ERR_IO, ("castro_sim_read_checkpoint: cannot open " + root + "/Header").c_str()); return CASTRO_ERR_IO; }
    auto fail = [&](int code, const std::string& m) {
        fclose(fp);
        set_error(code, ("castro_sim_read_checkpoint: " + m).c_str());
        return code;
    };
    int ver = 0, ns = 0, nvar = 0, ninst = 0;
    if (!ck_expect(fp, "castro_b200_checkpoint") || fscanf(fp, "%d", &ver) != 1 || ver != 1 || !ck_expect(fp, "nspec") ||
        fscanf(fp, "%d", &ns) != 1 || !ck_expect(fp, "nvar") || fscanf(fp, "%d", &nvar) != 1 || !ck_expect(fp, "ninst") ||
        fscanf(fp, "%d", &ninst) != 1)
        return fail(CASTRO_ERR_IO, "malformed Header");
    if (ns != s->ns || nvar != s->nvar || ninst != s->ninst)
        return fail(CASTRO_ERR_ARG, "species count or instance count differs from this sim's");
    std::vector<InstState> hs(ninst);
    std::vector<std::vector<double>> states(ninst);
    for (int in = 0; in < ninst; ++in) {
        const castro_instance_desc& D = s->desc[in];
        int idx = -1, dom[6], nbox = 0;
        if (!ck_expect(fp, "instance") || fscanf(fp, "%d", &idx) != 1 || idx != in || !ck_expect(fp, "domain") ||
            fscanf(fp, "%d %d %d %d %d %d", dom, dom + 1, dom + 2, dom + 3, dom + 4, dom + 5) != 6 || !ck_expect(fp, "nbox") ||
            fscanf(fp, "%d", &nbox) != 1)
            return fail(CASTRO_ERR_IO, "malformed Header");
        bool same = nbox == (int)s->inst_boxes[in].size();
        for (int d = 0; d < 3; ++d) same = same && dom[d] == D.dom_lo[d] && dom[3 + d] == D.dom_hi[d];
        for (int b = 0; b < nbox; ++b) {
            int bx[6];
            if (!ck_expect(fp, "box") || fscanf(fp, "%d %d %d %d %d %d", bx, bx + 1, bx + 2, bx + 3, bx + 4, bx + 5) != 6)
                return fail(CASTRO_ERR_IO, "malformed Header");
            if (same) {
                const BoxDev& B = s->hboxes[s->inst_boxes[in][b]];
                for (int d = 0; d < 3; ++d) same = same && bx[d] == B.lo[d] && bx[3 + d] == B.hi[d];
            }
        }
        if (!same) return fail(CASTRO_ERR_ARG, "domain or BoxArray differs from this sim's");
        InstState& st = hs[in];
        memset(&st, 0, sizeof st);
        if (!ck_expect(fp, "time") || fscanf(fp, "%la", &st.time) != 1 || !ck_expect(fp, "steps") ||
            fscanf(fp, "%d", &st.steps) != 1 || !ck_expect(fp, "dt_last") || fscanf(fp, "%la", &st.dt_last) != 1 ||
            !ck_expect(fp, "stop_time") || fscanf(fp, "%la", &st.stop_time) != 1)
            return fail(CASTRO_ERR_IO, "malformed Header");
        st.dt = st.dt_last;   // the last step's dt: computeNewDt's growth limit reads it
        st.dt_est = 1.79769313486231570e+308;
        char name[32];
        snprintf(name, sizeof name, "/State_%05d", in);
        FILE* fd = fopen((root + name).c_str(), "rb");
        if (!fd) return fail(CASTRO_ERR_IO, "cannot open " + root + name);
        size_t n = 0;
        for (int b : s->inst_boxes[in]) n += (size_t)(npts_reg(s->hboxes[b].lo, s->hboxes[b].hi, R_VALID, 0) * s->nvar);
        states[in].resize(n);
        const size_t got = fread(states[in].data(), sizeof(double), n, fd);
        const bool extra = fgetc(fd) != EOF;
        fclose(fd);
        if (got != n || extra) return fail(CASTRO_ERR_IO, std::string(name + 1) + " does not hold the instance's state");
    }
    if (!ck_expect(fp, "end")) return fail(CASTRO_ERR_IO, "malformed Header");
    fclose(fp);
    // everything read and checked: install it
    for (int in = 0; in < ninst; ++in) {
        size_t off = 0;
        for (int b : s->inst_boxes[in]) {
            const BoxDev& B = s->hboxes[b];
            const size_t n = (size_t)(npts_reg(B.lo, B.hi, R_VALID, 0) * s->nvar);
            if (!cuda_ok(cudaMemcpy(s->U + B.offU, states[in].data() + off, n * sizeof(double), cudaMemcpyHostToDevice),
                         "restart state"))
                return castro_last_error();
            off += n;
        }
    }
    if (!cuda_ok(cudaMemcpy(s->dstate, hs.data(), ninst * sizeof(InstState), cudaMemcpyHostToDevice), "restart dt"))
        return castro_last_error();
    if (s->mode == CASTRO_MODE_BATCHED || s->mode == CASTRO_MODE_PERSISTENT) {
        bool started = false;
        for (const InstState& st : hs) started = started || st.steps > 0;
        if (started) {
            // the batched step reads the next dt from the state record: form it as
            // the end of the checkpointed step did (estdt of the state, computeNewDt)
            if (s->ns == 2) restart_dt_kernels<2>(s);
            else restart_dt_kernels<13>(s);
        }
        s->dt_ready = started;
        check_launch("castro_sim_read_checkpoint");
    }
    cuda_ok(cudaStreamSynchronize(s->st), "restart sync");
    return castro_last_error();
}

double castro_sim_blast_radius(castro_sim* s, int inst, double* blast_mass)
{
    // max density on the host (diagnostic only), then the device reduction
    double maxd = -1.79769313486231570e+308;
    std::vector<double> h;
    for (int b : s->inst_boxes[inst]) {
        const BoxDev& B = s->hboxes[b];
        long long n = npts_reg(B.lo, B.hi, R_VALID, 0);
        h.resize(n);
        cudaStreamSynchronize(s->st);
        cuda_ok(cudaMemcpy(h.data(), s->U + B.offU, n * sizeof(double), cudaMemcpyDeviceToHost), "blast read");
        for (double v : h) maxd = std::max(maxd, v);
    }
    double* d2;
    if (!dalloc(&d2, 2, "blast")) return 0.0;
    cudaMemset(d2, 0, 2 * sizeof(double));
    cudaStream_t saved = castro::stream();
    castro_set_stream(s->st);
    const castro_instance_desc& D = s->desc[inst];
    for (int b : s->inst_boxes[inst]) {
        const BoxDev& B = s->hboxes[b];
        calculate_blast_radius(B.lo, B.hi, s->U + B.offU, B.lo, B.hi, &s->hdx[3 * inst], D.problo, D.probhi, d2, d2 + 1, maxd);
    }
    castro_set_stream(saved);
    double hr[2];
    cudaStreamSynchronize(s->st);
    cuda_ok(cudaMemcpy(hr, d2, sizeof hr, cudaMemcpyDeviceToHost), "blast result");
    cudaFree(d2);
    if (blast_mass) *blast_mass = hr[0];
    return hr[1] / hr[0];
}

}  // extern "C"

// ---------------------------------------------------------------------------
// castro_construct_hydro_source_box_noalloc: the same fused per-box hydro
// source, with every scratch array carved out of one file-scope device array
// instead of device memory the library allocates.  For callers that cannot
// allocate device memory while they advance a box: hosts that hand out all
// device memory from their own preallocated pool (an AMReX-style arena sized
// at start-up), and hosts that must not call cudaMalloc from inside the time
// step because it synchronizes the device.
// ---------------------------------------------------------------------------
namespace castro {
namespace {

// 18 MiB: a box of up to 16^3 zones with 13 species, or up to 21^3 zones with
// 2 species, including the box / work-list records at its head.
constexpr long long NOALLOC_DOUBLES = 2359296;
constexpr int NOALLOC_MAX_DEVICES = 64;
constexpr long long NOALLOC_META_BYTES = 65536;   // BoxDev, InstDev, InstState, work lists

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

// device address of g_noalloc_scratch per device, from cudaGetSymbolAddress,
// looked up once per device together with the kernel attributes of each
// species count (std::call_once: host threads making their first call on a
// device together do it once and all see the result)
double* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};
std::once_flag g_noalloc_once[NOALLOC_MAX_DEVICES][2];
int g_noalloc_setup_rc[NOALLOC_MAX_DEVICES][2] = {};

enum { NL_VALID = 0, NL_G4, NL_G1, NL_TRACE, NL_TBX, NL_EBX, NL_COUNT };

struct NoallocLists {
    int nsub[NL_COUNT];
    long long np[NL_COUNT][6];    // points of each sub-region
    int first[NL_COUNT];          // first work item of each list
    int total;
};

__global__ void k_noalloc_setup(BoxDev B, InstDev I, InstState st, NoallocLists NLs, BoxDev* dB, InstDev* dI,
                                InstState* dS, Work* work)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 0) {
        *dB = B;
        *dI = I;
        *dS = st;
    }
    if (t >= NLs.total) return;
    int l = NL_COUNT - 1;
    while (l > 0 && t < NLs.first[l]) --l;
    int item = t - NLs.first[l];
    for (int sub = 0; sub < NLs.nsub[l]; ++sub) {
        long long np = NLs.np[l][sub];
        int nb = (int)((np + BLOCK - 1) / BLOCK);
        if (item < nb) {
            Work w;
            w.box = 0;
            w.sub = sub;
            w.start = item * BLOCK;
            w.count = (int)(np - (long long)item * BLOCK < BLOCK ? np - (long long)item * BLOCK : BLOCK);
            work[t] = w;
            return;
        }
        item -= nb;
    }
}

// Layout of one box's stage arrays and work lists, shared by both box entry
// points: records and work lists at the head of the scratch (meta), then the
// stage arrays (pools) at the offsets BoxDev carries.
struct BoxPlan {
    BoxDev B;
    NoallocLists NLs;
    int nblocks[NL_COUNT];
    long long meta_bytes;     // BoxDev, InstDev, InstState records and the work list
    long long pool_doubles;   // the stage arrays
};

template <int NS>
BoxPlan box_plan(const int* lo, const int* hi)
{
    BoxPlan P;
    memset(&P, 0, sizeof P);
    const int NV = Dims<NS>::NVAR, NQF = QF<NS>::N, NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF;
    BoxDev& B = P.B;
    for (int d = 0; d < 3; ++d) { B.lo[d] = lo[d]; B.hi[d] = hi[d]; }
    B.inst = 0;
    long long o = 0;
    auto take = [&](long long n) { long long r = o; o += (n + 31) / 32 * 32; return r; };   // 256-byte aligned
    B.offU = 0;
    B.offUb = take(npts_reg(B.lo, B.hi, R_G1, 0) * NV);
    B.offQ = take(npts_reg(B.lo, B.hi, R_G4, 0) * NQF);
    B.offDiv = take(npts_reg(B.lo, B.hi, R_G1, 0) * 2);
    for (int d = 0; d < 3; ++d) {
        B.offTr[d] = take(npts_reg(B.lo, B.hi, R_TBX, 4 * d) * 2 * NQS);
        B.offF1[d] = take(npts_reg(B.lo, B.hi, R_TBX, 4 * d) * NTF);
        B.offFx[d] = take(npts_reg(B.lo, B.hi, R_EBX, d) * (NV + 1));
    }
    for (int a = 0; a < 3; ++a)
        for (int bb = 0; bb < 3; ++bb)
            if (a != bb) B.offF2[pair_index(a, bb)] = take(npts_reg(B.lo, B.hi, R_TBX, 3 * a + bb) * NTF);
    P.pool_doubles = o;

    const int kinds[NL_COUNT] = {R_VALID, R_G4, R_G1, R_SEG, R_TBX, R_EBX};
    const int nsubs[NL_COUNT] = {1, 1, 1, 3, 3, 3};
    int total = 0;
    for (int l = 0; l < NL_COUNT; ++l) {
        P.NLs.nsub[l] = nsubs[l];
        P.NLs.first[l] = total;
        int nb = 0;
        for (int sub = 0; sub < nsubs[l]; ++sub) {
            int rs = sub;
            if (l == NL_TBX) rs = 4 * sub;
            P.NLs.np[l][sub] = npts_reg(B.lo, B.hi, kinds[l], rs);
            nb += (int)((P.NLs.np[l][sub] + BLOCK - 1) / BLOCK);
        }
        P.nblocks[l] = nb;
        total += nb;
    }
    P.NLs.total = total;
    P.meta_bytes = 1024 + (long long)total * (long long)sizeof(Work);
    return P;
}

// The per-box hydro source over a scratch whose first meta_doubles hold the
// records and work lists and the rest the stage arrays of plan P.
template <int NS>
int box_hydro_launch(const BoxPlan& P, double* base, long long meta_doubles, const double* sb, const int* sb_lo,
                     const int* sb_hi, double* source, const int* sr_lo, const int* sr_hi, double* const* fo,
                     const int* fo_lo, const int* fo_hi, const double* dx, double dt, const char* who)
{
    char* mb = reinterpret_cast<char*>(base);
    BoxDev* dB = reinterpret_cast<BoxDev*>(mb);
    InstDev* dI = reinterpret_cast<InstDev*>(mb + 256);
    InstState* dS = reinterpret_cast<InstState*>(mb + 512);
    Work* work = reinterpret_cast<Work*>(mb + 1024);
    double* pools = base + meta_doubles;

    InstDev I;
    memset(&I, 0, sizeof I);
    for (int d = 0; d < 3; ++d) { I.dom_lo[d] = P.B.lo[d]; I.dom_hi[d] = P.B.hi[d]; I.dx[d] = dx[d]; }
    I.bc = CASTRO_BC_OUTFLOW;
    I.g = 1;
    InstState st;
    memset(&st, 0, sizeof st);
    st.dt = dt;
    st.stop_time = -1.0;

    const int total = P.NLs.total;
    const int* nblocks = P.nblocks;
    const NoallocLists& NLs = P.NLs;
    cudaStream_t cs = castro::stream();
    k_noalloc_setup<<<(total + 127) / 128, 128, 0, cs>>>(P.B, I, st, NLs, dB, dI, dS, work);
    SimDev S;
    memset(&S, 0, sizeof S);
    S.boxes = dB; S.dom = dB; S.inst = dI; S.st = dS;   // the box is the instance domain
    S.Ub = pools; S.Q = pools; S.Div = pools; S.Tr = pools; S.F1 = pools; S.F2 = pools; S.Fx = pools;
    const Work* W = work;
    CASTRO_EOS_LAUNCH(k_box_prim, NS, nblocks[NL_G4], BLOCK, 0, cs, S, W + NLs.first[NL_G4], make_fab(sb, sb_lo, sb_hi));
    k_prep<NS><<<nblocks[NL_G1], BLOCK, 0, cs>>>(S, W + NLs.first[NL_G1]);
    k_trace<NS><<<nblocks[NL_TRACE], BLOCK, 0, cs>>>(S, W + NLs.first[NL_TRACE]);
    if (CASTRO_TRACE_SPLIT) k_trace2<NS><<<nblocks[NL_TRACE], BLOCK, 0, cs>>>(S, W + NLs.first[NL_TRACE]);
    k_riemann1<NS><<<nblocks[NL_TBX], BLOCK, 0, cs>>>(S, W + NLs.first[NL_TBX]);
    k_riemann2<NS><<<nblocks[NL_TBX], BLOCK, R2Slot<NS>::BYTES, cs>>>(S, W + NLs.first[NL_TBX]);
    k_riemann3<NS><<<nblocks[NL_EBX], BLOCK, R3Slot<NS>::BYTES, cs>>>(S, W + NLs.first[NL_EBX]);
    k_box_source<NS><<<nblocks[NL_VALID], BLOCK, 0, cs>>>(S, W + NLs.first[NL_VALID], make_fab(source, sr_lo, sr_hi));
    if (fo) {
        Fab F[3];
        for (int d = 0; d < 3; ++d) {
            F[d] = fo[d] ? make_fab(fo[d], fo_lo + 3 * d, fo_hi + 3 * d) : Fab{};
            if (!fo[d]) F[d].p = nullptr;
        }
        k_box_store_flux<NS><<<nblocks[NL_EBX], BLOCK, 0, cs>>>(S, W + NLs.first[NL_EBX], F[0], F[1], F[2], dt);
    }
    check_launch(who);
    return castro_last_error();
}

// The arrays a box call touches cover what it touches: Sborder grow(box, 4), the
// source the box, each requested flux array its face box.  Checked on the host
// before anything is launched.
bool box_call_args_ok(const char* who, const int* lo, const int* hi, const int* sb_lo, const int* sb_hi,
                      const int* sr_lo, const int* sr_hi, double* const* fo, const int* fo_lo, const int* fo_hi)
{
    char msg[200];
    for (int d = 0; d < 3; ++d) {
        if (lo[d] > hi[d]) { snprintf(msg, sizeof msg, "%s: empty box", who); set_error(CASTRO_ERR_ARG, msg); return false; }
        if (sb_lo[d] > lo[d] - NG || sb_hi[d] < hi[d] + NG) {
            snprintf(msg, sizeof msg, "%s: Sborder needs 4 ghost zones", who);
            set_error(CASTRO_ERR_ARG, msg);
            return false;
        }
        if (sr_lo[d] > lo[d] || sr_hi[d] < hi[d]) {
            snprintf(msg, sizeof msg, "%s: the source array does not cover the box", who);
            set_error(CASTRO_ERR_ARG, msg);
            return false;
        }
    }
    if (fo)
        for (int f = 0; f < 3; ++f) {
            if (!fo[f]) continue;
            for (int d = 0; d < 3; ++d)
                if (fo_lo[3 * f + d] > lo[d] || fo_hi[3 * f + d] < hi[d] + (d == f)) {
                    snprintf(msg, sizeof msg, "%s: flux array %d does not cover the box's faces", who, f);
                    set_error(CASTRO_ERR_ARG, msg);
                    return false;
                }
        }
    return true;
}

template <int NS>
int box_hydro_noalloc_impl(const int* lo, const int* hi, const double* sb, const int* sb_lo, const int* sb_hi,
                           double* source, const int* sr_lo, const int* sr_hi, double* const* fo, const int* fo_lo,
                           const int* fo_hi, const double* dx, double dt)
{
    NvtxRange r("castro_construct_hydro_source_box_noalloc");
    if (!box_call_args_ok("castro_construct_hydro_source_box_noalloc", lo, hi, sb_lo, sb_hi, sr_lo, sr_hi, fo, fo_lo,
                          fo_hi))
        return CASTRO_ERR_ARG;
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "castro_construct_hydro_source_box_noalloc: cudaGetDevice")) return CASTRO_ERR_CUDA;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        set_error(CASTRO_ERR_ARG, "castro_construct_hydro_source_box_noalloc: device index beyond 63");
        return CASTRO_ERR_ARG;
    }
    const int nsi = NS == 2 ? 0 : 1;
    std::call_once(g_noalloc_once[dev][nsi], [dev, nsi]() {
        // the host-side name of a __device__ array is only a stand-in; kernels
        // need its device address on this device
        void* p = nullptr;
        if (!set_kernel_attributes<NS>() ||
            !cuda_ok(cudaGetSymbolAddress(&p, g_noalloc_scratch),
                     "castro_construct_hydro_source_box_noalloc: cudaGetSymbolAddress")) {
            g_noalloc_setup_rc[dev][nsi] = CASTRO_ERR_CUDA;
            return;
        }
        g_noalloc_addr[dev] = static_cast<double*>(p);
    });
    if (g_noalloc_setup_rc[dev][nsi] != 0 || !g_noalloc_addr[dev]) {
        set_error(CASTRO_ERR_CUDA, "castro_construct_hydro_source_box_noalloc: device set-up failed on this device");
        return CASTRO_ERR_CUDA;
    }
    const BoxPlan P = box_plan<NS>(lo, hi);
    const long long meta_doubles = NOALLOC_META_BYTES / 8;
    if (P.meta_bytes > NOALLOC_META_BYTES || meta_doubles + P.pool_doubles > NOALLOC_DOUBLES) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "castro_construct_hydro_source_box_noalloc: box needs %lld doubles of scratch, the static array holds %lld "
                 "(at most 16^3 zones with 13 species, 21^3 with 2)", meta_doubles + P.pool_doubles, NOALLOC_DOUBLES);
        set_error(CASTRO_ERR_ARG, msg);
        return CASTRO_ERR_ARG;
    }
    return box_hydro_launch<NS>(P, g_noalloc_addr[dev], meta_doubles, sb, sb_lo, sb_hi, source, sr_lo, sr_hi, fo, fo_lo,
                                fo_hi, dx, dt, "castro_construct_hydro_source_box_noalloc");
}

// Library-managed scratch of castro_construct_hydro_source_box: one device
// array per (device, stream) -- calls on different streams may overlap on the
// GPU, as an AMReX host's MFIter loop does over its GPU streams -- grown to the
// largest box seen on that stream so far (the stage arrays and work lists of
// any box fit a scratch sized for a larger one, and every call lays its box out
// afresh), so that a BoxArray of any mix of shapes allocates once per new
// largest box, not once per shape.  Up to BOX_ARENAS streams per device; the
// least recently used one's array is released (after a device synchronisation)
// for a stream beyond that.
struct BoxArena {
    cudaStream_t st = nullptr;
    double* p = nullptr;
    long long cap = 0;   // doubles
    unsigned long long used = 0;
};
constexpr int BOX_MAX_DEVICES = 64;
constexpr int BOX_ARENAS = 16;
BoxArena g_box_arena[BOX_MAX_DEVICES][BOX_ARENAS];
unsigned long long g_box_clock[BOX_MAX_DEVICES] = {};
std::mutex g_box_mu[BOX_MAX_DEVICES];
std::once_flag g_box_once[BOX_MAX_DEVICES][2];
int g_box_setup_rc[BOX_MAX_DEVICES][2] = {};

template <int NS>
int box_hydro_impl(const int* lo, const int* hi, const double* sb, const int* sb_lo, const int* sb_hi,
                   double* source, const int* sr_lo, const int* sr_hi, double* const* fo, const int* fo_lo,
                   const int* fo_hi, const double* dx, double dt)
{
    NvtxRange r("castro_construct_hydro_source_box");
    if (!box_call_args_ok("castro_construct_hydro_source_box", lo, hi, sb_lo, sb_hi, sr_lo, sr_hi, fo, fo_lo, fo_hi))
        return CASTRO_ERR_ARG;
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "castro_construct_hydro_source_box: cudaGetDevice")) return CASTRO_ERR_CUDA;
    if (dev < 0 || dev >= BOX_MAX_DEVICES) {
        set_error(CASTRO_ERR_ARG, "castro_construct_hydro_source_box: device index beyond 63");
        return CASTRO_ERR_ARG;
    }
    const int nsi = NS == 2 ? 0 : 1;
    std::call_once(g_box_once[dev][nsi], [dev, nsi]() {
        if (!set_kernel_attributes<NS>()) g_box_setup_rc[dev][nsi] = CASTRO_ERR_CUDA;
    });
    if (g_box_setup_rc[dev][nsi] != 0) {
        set_error(CASTRO_ERR_CUDA, "castro_construct_hydro_source_box: device set-up failed on this device");
        return CASTRO_ERR_CUDA;
    }
    const BoxPlan P = box_plan<NS>(lo, hi);
    const long long meta_doubles = (P.meta_bytes + 255) / 256 * 32;
    const long long need = meta_doubles + P.pool_doubles;
    double* base = nullptr;
    const cudaStream_t cs = castro::stream();
    {
        std::lock_guard<std::mutex> lock(g_box_mu[dev]);
        BoxArena* A = nullptr;
        BoxArena* victim = &g_box_arena[dev][0];
        for (int c = 0; c < BOX_ARENAS && !A; ++c) {
            BoxArena& e = g_box_arena[dev][c];
            if (e.p && e.st == cs) A = &e;
            else if (!e.p ? victim->p != nullptr : (victim->p && e.used < victim->used)) victim = &e;
        }
        if (!A) {   // a stream new to this device: a free slot, or the least recently used stream's array
            A = victim;
            if (A->p && !cuda_ok(cudaDeviceSynchronize(), "castro_construct_hydro_source_box: synchronize before reuse"))
                return CASTRO_ERR_CUDA;   // kernels of that stream's calls may still read it
            A->st = cs;
        }
        if (A->cap < need) {
            // kernels of earlier calls may still read the old array
            if (A->p && !cuda_ok(cudaDeviceSynchronize(), "castro_construct_hydro_source_box: synchronize before growing"))
                return CASTRO_ERR_CUDA;
            if (A->p) cudaFree(A->p);
            A->p = nullptr;
            A->cap = 0;
            if (!dalloc(&A->p, (size_t)need, "castro_construct_hydro_source_box: scratch")) return CASTRO_ERR_CUDA;
            A->cap = need;
        }
        A->used = ++g_box_clock[dev];
        base = A->p;
    }
    return box_hydro_launch<NS>(P, base, meta_doubles, sb, sb_lo, sb_hi, source, sr_lo, sr_hi, fo, fo_lo, fo_hi, dx, dt,
                                "castro_construct_hydro_source_box");
}

}  // namespace
}  // namespace castro

extern "C" {

int castro_construct_hydro_source_box(const int* lo, const int* hi, const double* sborder, const int* sb_lo,
                                      const int* sb_hi, double* source, const int* sr_lo, const int* sr_hi,
                                      double* const* fluxes_out, const int* fo_lo3x3, const int* fo_hi3x3,
                                      const int* domlo, const int* domhi, const double* dx, double dt)
{
    (void)domlo; (void)domhi;
    if (!table_ready()) { set_error(CASTRO_ERR_NO_TABLE, "castro_construct_hydro_source_box: eos_init has not run"); return CASTRO_ERR_NO_TABLE; }
    if (nspec() == 2) return box_hydro_impl<2>(lo, hi, sborder, sb_lo, sb_hi, source, sr_lo, sr_hi, fluxes_out, fo_lo3x3, fo_hi3x3, dx, dt);
    if (nspec() == 13) return box_hydro_impl<13>(lo, hi, sborder, sb_lo, sb_hi, source, sr_lo, sr_hi, fluxes_out, fo_lo3x3, fo_hi3x3, dx, dt);
    set_error(CASTRO_ERR_NSPEC, "castro_construct_hydro_source_box: nspec");
    return CASTRO_ERR_NSPEC;
}

int castro_construct_hydro_source_box_noalloc(const int* lo, const int* hi, const double* sborder, const int* sb_lo,
                                              const int* sb_hi, double* source, const int* sr_lo, const int* sr_hi,
                                              double* const* fluxes_out, const int* fo_lo3x3, const int* fo_hi3x3,
                                              const int* domlo, const int* domhi, const double* dx, double dt)
{
    (void)domlo; (void)domhi;
    if (!table_ready()) {
        set_error(CASTRO_ERR_NO_TABLE, "castro_construct_hydro_source_box_noalloc: eos_init has not run");
        return CASTRO_ERR_NO_TABLE;
    }
    if (nspec() == 2)
        return box_hydro_noalloc_impl<2>(lo, hi, sborder, sb_lo, sb_hi, source, sr_lo, sr_hi, fluxes_out, fo_lo3x3,
                                         fo_hi3x3, dx, dt);
    if (nspec() == 13)
        return box_hydro_noalloc_impl<13>(lo, hi, sborder, sb_lo, sb_hi, source, sr_lo, sr_hi, fluxes_out, fo_lo3x3,
                                          fo_hi3x3, dx, dt);
    set_error(CASTRO_ERR_NSPEC, "castro_construct_hydro_source_box_noalloc: nspec");
    return CASTRO_ERR_NSPEC;
}

int castro_sim_launches_per_step(const castro_sim* s) { return s->launches; }

int castro_sim_set_wait_limit(castro_sim* s, long long polls, int stage, int extra)
{
    if (!s || s->mode != CASTRO_MODE_PERSISTENT || polls < 1 || extra < 0) {
        set_error(CASTRO_ERR_ARG, "castro_sim_set_wait_limit: a persistent-mode sim, polls >= 1, extra >= 0");
        return CASTRO_ERR_ARG;
    }
    s->pargs.spin_limit = polls;
    s->pargs.test_stage = extra > 0 ? stage : -1;
    s->pargs.test_extra = extra;
    // the arguments are baked into the captured step: capture again
    if (s->gexec) cudaGraphExecDestroy(s->gexec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->gexec = nullptr;
    s->graph = nullptr;
    return CASTRO_OK;
}

void* castro_sim_stream(castro_sim* s) { return (void*)s->st; }

int castro_sim_profile_step(castro_sim* s, double* ms, const char** names)
{
    if (s->mode != CASTRO_MODE_BATCHED) { set_error(CASTRO_ERR_ARG, "castro_sim_profile_step: batched mode only"); return 0; }
    // profile_kernel ids in step order; 9 = trace's pass 2 when it is a kernel of its own
    static const int ids[10] = {0, 1, 2, 3, 9, 4, 5, 6, 7, 8};
    static const char* kn[10] = {"front", "ghost", "prep", "trace", "trace2", "riemann1", "riemann2", "riemann3", "update",
                                 "dt"};
    int order[10], m = 0;
    const char* nm[10];
    for (int q = 0; q < 10; ++q) {
        if (ids[q] == 9 && !CASTRO_TRACE_SPLIT) continue;
        if (ids[q] == 6 && s->r23) continue;          // riemann23 runs as id 5
        order[m] = ids[q];
        nm[m++] = (ids[q] == 5 && s->r23) ? "riemann23" : kn[q];
    }
    const int NK = m;
    cudaEvent_t ev[11];
    for (int k = 0; k < 11; ++k) cudaEventCreate(&ev[k]);
    if (!s->dt_ready) {
        if (s->ns == 2) initial_dt_kernels<2>(s); else initial_dt_kernels<13>(s);
        s->dt_ready = true;
    }
    SimDev S = s->dev();
    cudaStream_t st = s->st;
    cudaEventRecord(ev[0], st);
    for (int k = 0; k < NK; ++k) {
        if (s->ns == 2) profile_kernel<2>(s, S, order[k]); else profile_kernel<13>(s, S, order[k]);
        cudaEventRecord(ev[k + 1], st);
    }
    cudaEventSynchronize(ev[NK]);
    for (int k = 0; k < NK; ++k) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
        ms[k] = t;
        names[k] = nm[k];
    }
    for (int k = 0; k < 11; ++k) cudaEventDestroy(ev[k]);
    check_launch("castro_sim_profile_step");
    return NK;
}

long long castro_sim_eos_failures(castro_sim* s)
{
    unsigned long long* p = eos_fail_counter();
    if (!p) return 0;
    unsigned long long v = 0;
    cudaStreamSynchronize(s->st);
    cuda_ok(cudaMemcpy(&v, p, sizeof v, cudaMemcpyDeviceToHost), "eos failures");
    return v >= s->eos_base ? (long long)(v - s->eos_base) : (long long)v;
}

}  // extern "C"
