// castro_abi.cu -- the Source/Castro_F.H entry points as box-wide kernels.
//
// Each extern "C" function keeps the reference prototype and launches one
// kernel over [lo,hi] (one thread per zone or face) on the library stream.
// The per-zone math lives in castro_device.cuh.
#include "castro_common.cuh"
#include "../../include/castro_b200.h"

using namespace castro;

namespace {

// view of FAB q (full QVAR layout) + qaux for the trace / flatten stencils
struct FabLoader {
    Fab qf, qaf;
    __device__ __forceinline__ double q(int i, int j, int k, int n) const { return qf(i, j, k, n); }
    __device__ __forceinline__ double gamc(int i, int j, int k) const { return qaf(i, j, k, QGAMC); }
    __device__ __forceinline__ double c(int i, int j, int k) const { return qaf(i, j, k, QC); }
};

// compact face state <-> full QVAR record
template <int NS>
__device__ __forceinline__ void load_state(const Fab& f, int i, int j, int k, double* s)
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
__device__ __forceinline__ void store_state(const Fab& f, int i, int j, int k, const double* s)
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

// flux record for the transverse corrections from a flux FAB and a qgdnv FAB
template <int NS>
__device__ __forceinline__ void load_tflux(const Fab& f, const Fab& qg, int i, int j, int k, int normal, double* r)
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

// Routines that call the EOS run the instantiation with or without the Coulomb
// corrections (COUL), as the library is set.
template <int NS, bool COUL>
void ctoprim_run(const int* lo, const int* hi, Fab U, Fab Q, Fab QA)
{
    launch_box("ctoprim", lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NVAR = Dims<NS>::NVAR, QVAR = Dims<NS>::QVAR;
        double u[NVAR], q[QVAR], qa[NQAUX];
#pragma unroll
        for (int n = 0; n < NVAR; ++n) u[n] = U(i, j, k, n);
        ctoprim_pt<NS, COUL>(u, q, qa);
#pragma unroll
        for (int n = 0; n < QVAR; ++n) Q(i, j, k, n) = q[n];
#pragma unroll
        for (int n = 0; n < NQAUX; ++n) QA(i, j, k, n) = qa[n];
    });
}

template <int NS>
void ctoprim_impl(const int* lo, const int* hi, Fab U, Fab Q, Fab QA)
{
    if (coulomb_on()) ctoprim_run<NS, true>(lo, hi, U, Q, QA);
    else ctoprim_run<NS, false>(lo, hi, U, Q, QA);
}

template <int NS, int WHICH, bool COUL>
void clean_run(const char* what, const int* lo, const int* hi, Fab U)
{
    launch_box(what, lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NVAR = Dims<NS>::NVAR;
        double u[NVAR];
#pragma unroll
        for (int n = 0; n < NVAR; ++n) u[n] = U(i, j, k, n);
        if (WHICH == 0) enforce_minimum_density_pt<NS, COUL>(u);
        else if (WHICH == 1) normalize_species_pt<NS>(u);
        else if (WHICH == 2) reset_internal_e_pt<NS, COUL>(u);
        else if (WHICH == 3) compute_temp_pt<NS, COUL>(u);
        else clean_state_pt<NS, COUL>(u);   // the four in a row: each is pointwise
#pragma unroll
        for (int n = 0; n < NVAR; ++n) U(i, j, k, n) = u[n];
    });
}

template <int NS, int WHICH>
void clean_impl(const char* what, const int* lo, const int* hi, Fab U)
{
    if (WHICH != 1 && coulomb_on()) clean_run<NS, WHICH, true>(what, lo, hi, U);
    else clean_run<NS, WHICH, false>(what, lo, hi, U);
}

__device__ __forceinline__ void atomic_min_double(double* addr, double v)
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

template <int NS, bool COUL>
__global__ void k_estdt(BoxRange r, Fab U, double dx0, double dx1, double dx2, double* dt)
{
    __shared__ double red[32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double m = 1.79769313486231570e+308;
    if (t < r.n) {
        int i = r.lx + (int)(t % r.nx);
        long long t2 = t / r.nx;
        int j = r.ly + (int)(t2 % r.ny);
        int k = r.lz + (int)(t2 / r.ny);
        double u[Dims<NS>::NVAR];
#pragma unroll
        for (int n = 0; n < Dims<NS>::NVAR; ++n) u[n] = U(i, j, k, n);
        m = estdt_pt<NS, COUL>(u, dx0, dx1, dx2);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = DMIN(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = (threadIdx.x < (blockDim.x >> 5)) ? red[threadIdx.x] : 1.79769313486231570e+308;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = DMIN(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) atomic_min_double(dt, m);
    }
}

template <int NS>
void estdt_impl(const int* lo, const int* hi, Fab U, const double* dx, double* dt)
{
    BoxRange r = make_range(lo, hi);
    if (r.n == 0) return;
    const int B = 128;
    const unsigned g = (unsigned)((r.n + B - 1) / B);
    if (coulomb_on()) k_estdt<NS, true><<<g, B, 0, stream()>>>(r, U, dx[0], dx[1], dx[2], dt);
    else k_estdt<NS, false><<<g, B, 0, stream()>>>(r, U, dx[0], dx[1], dx[2], dt);
    check_launch("estdt");
}

template <int NS, int D>
void trace_dir(const int* lo, const int* hi, int vl, int vh, FabLoader ld, Fab QM, Fab QP, double dtdx)
{
    launch_box("trace_ppm", lo, hi, [=] __device__(int i, int j, int k) {
        double flatn = uflatten(ld, i, j, k);
        double qplus[Dims<NS>::NQS], qminus[Dims<NS>::NQS];
        trace_zone<NS, D>(ld, i, j, k, dtdx, flatn, qplus, qminus);
        int idx = D == 0 ? i : D == 1 ? j : k;
        if (idx >= vl) store_state<NS>(QP, i, j, k, qplus);
        if (idx <= vh) store_state<NS>(QM, i + (D == 0), j + (D == 1), k + (D == 2), qminus);
    });
}

template <int NS>
void trace_impl(const int* lo, const int* hi, const int* vlo, const int* vhi, int idir,
                Fab Q, Fab QA, Fab QM, Fab QP, double dtdx)
{
    FabLoader ld{Q, QA};
    if (idir == 0) trace_dir<NS, 0>(lo, hi, vlo[0], vhi[0], ld, QM, QP, dtdx);
    else if (idir == 1) trace_dir<NS, 1>(lo, hi, vlo[1], vhi[1], ld, QM, QP, dtdx);
    else trace_dir<NS, 2>(lo, hi, vlo[2], vhi[2], ld, QM, QP, dtdx);
}

template <int NS, int D>
void compute_flux_dir(const int* lo, const int* hi, Fab QL, Fab QR, Fab FX, Fab QI, Fab QG, Fab QA)
{
    launch_box("compute_flux", lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NQS = Dims<NS>::NQS, NVAR = Dims<NS>::NVAR, QVAR = Dims<NS>::QVAR;
        double ql[NQS], qr[NQS], flx[NVAR], qg[NGDNV], qint[QVAR];
        load_state<NS>(QL, i, j, k, ql);
        load_state<NS>(QR, i, j, k, qr);
        constexpr int ex = D == 0, ey = D == 1, ez = D == 2;
        riemann_cgf<NS, D>(ql, qr, QA(i - ex, j - ey, k - ez, QGAMC), QA(i, j, k, QGAMC),
                           QA(i - ex, j - ey, k - ez, QC), QA(i, j, k, QC), flx, qg, qint);
#pragma unroll
        for (int n = 0; n < NVAR; ++n) FX(i, j, k, n) = flx[n];
#pragma unroll
        for (int n = 0; n < NGDNV; ++n) QG(i, j, k, n) = qg[n];
#pragma unroll
        for (int n = 0; n < QVAR; ++n)
            if (n != QTEMP) QI(i, j, k, n) = qint[n];
    });
}

template <int NS>
void compute_flux_impl(const int* lo, const int* hi, Fab QL, Fab QR, Fab FX, Fab QI, Fab QG, Fab QA, int idir)
{
    if (idir == 0) compute_flux_dir<NS, 0>(lo, hi, QL, QR, FX, QI, QG, QA);
    else if (idir == 1) compute_flux_dir<NS, 1>(lo, hi, QL, QR, FX, QI, QG, QA);
    else compute_flux_dir<NS, 2>(lo, hi, QL, QR, FX, QI, QG, QA);
}

template <int NS>
void trans1_impl(const int* lo, const int* hi, int idir1, int idir2, Fab Q2M, Fab Q2MO, Fab Q2P, Fab Q2PO,
                 Fab QA, Fab F1, Fab Q1, double cdtdx)
{
    launch_box("trans1", lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF;
        const int e1x = idir1 == 0, e1y = idir1 == 1, e1z = idir1 == 2;
        const int e2x = idir2 == 0, e2y = idir2 == 1, e2z = idir2 == 2;
#pragma unroll
        for (int d = -1; d <= 0; ++d) {
            int il = i + d * e2x, jl = j + d * e2y, kl = k + d * e2z;
            int ir = il + e1x, jr = jl + e1y, kr = kl + e1z;
            double lq[NQS], lqo[NQS], fr[NTF], fl[NTF];
            if (d == -1) load_state<NS>(Q2M, i, j, k, lq);
            else load_state<NS>(Q2P, i, j, k, lq);
            load_tflux<NS>(F1, Q1, ir, jr, kr, idir1, fr);
            load_tflux<NS>(F1, Q1, il, jl, kl, idir1, fl);
            bool reset = trans1_state<NS>(lq, fr, fl, QA(il, jl, kl, QGAMC), cdtdx, lqo);
            const Fab& O = (d == -1) ? Q2MO : Q2PO;
            const Fab& I = (d == -1) ? Q2M : Q2P;
            store_state<NS>(O, i, j, k, lqo);
            if (reset) O(i, j, k, QGAME) = I(i, j, k, QGAME);
        }
    });
}

template <int NS>
void trans2_impl(const int* lo, const int* hi, int idir1, int idir2, int idir3, Fab QM, Fab QMO, Fab QP, Fab QPO,
                 Fab QA, Fab F2, Fab F3, Fab G2, Fab G3, double cdtdx2, double cdtdx3)
{
    launch_box("trans2", lo, hi, [=] __device__(int i, int j, int k) {
        constexpr int NQS = Dims<NS>::NQS, NTF = Dims<NS>::NTF;
        const int e1x = idir1 == 0, e1y = idir1 == 1, e1z = idir1 == 2;
        const int e2x = idir2 == 0, e2y = idir2 == 1, e2z = idir2 == 2;
        const int e3x = idir3 == 0, e3y = idir3 == 1, e3z = idir3 == 2;
#pragma unroll
        for (int d = -1; d <= 0; ++d) {
            // zone the state comes from (il1 = il2 = il3 of trans.F90:332-380)
            int il = i + d * e1x, jl = j + d * e1y, kl = k + d * e1z;
            double lq[NQS], lqo[NQS], f2r[NTF], f2l[NTF], f3r[NTF], f3l[NTF];
            if (d == -1) load_state<NS>(QM, i, j, k, lq);
            else load_state<NS>(QP, i, j, k, lq);
            load_tflux<NS>(F2, G2, il + e2x, jl + e2y, kl + e2z, idir2, f2r);
            load_tflux<NS>(F2, G2, il, jl, kl, idir2, f2l);
            load_tflux<NS>(F3, G3, il + e3x, jl + e3y, kl + e3z, idir3, f3r);
            load_tflux<NS>(F3, G3, il, jl, kl, idir3, f3l);
            bool reset = trans2_state<NS>(lq, f2r, f2l, f3r, f3l, QA(il, jl, kl, QGAMC), cdtdx2, cdtdx3, lqo);
            const Fab& O = (d == -1) ? QMO : QPO;
            const Fab& I = (d == -1) ? QM : QP;
            store_state<NS>(O, i, j, k, lqo);
            if (reset) O(i, j, k, QGAME) = I(i, j, k, QGAME);
        }
    });
}

template <int NS>
void apply_av_impl(const int* lo, const int* hi, int idir, double dxd, Fab DIV, Fab U, Fab FX)
{
    launch_box("apply_av", lo, hi, [=] __device__(int i, int j, int k) {
        double ds;
        if (idir == 0) ds = DIV(i, j, k, 0) + DIV(i, j + 1, k, 0) + DIV(i, j, k + 1, 0) + DIV(i, j + 1, k, 0);
        else if (idir == 1) ds = DIV(i, j, k, 0) + DIV(i + 1, j, k, 0) + DIV(i, j, k + 1, 0) + DIV(i + 1, j, k, 0);
        else ds = DIV(i, j, k, 0) + DIV(i + 1, j, k, 0) + DIV(i, j + 1, k, 0) + DIV(i + 1, j + 1, k, 0);
        const int ex = idir == 0, ey = idir == 1, ez = idir == 2;
#pragma unroll
        for (int n = 0; n < Dims<NS>::NVAR; ++n) {
            if (n == UTEMP) continue;
            double div1 = av_term(ds, U(i, j, k, n) - U(i - ex, j - ey, k - ez, n));
            FX(i, j, k, n) = FX(i, j, k, n) + dxd * div1;
        }
    });
}

template <int NS>
void normalize_species_fluxes_impl(const int* lo, const int* hi, Fab FX)
{
    launch_box("normalize_species_fluxes", lo, hi, [=] __device__(int i, int j, int k) {
        double sum = 0.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) sum = sum + FX(i, j, k, UFS + n);
        double fac = (sum != 0.0) ? FX(i, j, k, URHO) / sum : 1.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) FX(i, j, k, UFS + n) = FX(i, j, k, UFS + n) * fac;
    });
}

template <int NS>
void store_flux_impl(const int* lo, const int* hi, Fab FO, Fab FI, Fab A, double dt)
{
    launch_box("store_flux", lo, hi, [=] __device__(int i, int j, int k) {
#pragma unroll
        for (int n = 0; n < Dims<NS>::NVAR; ++n) FO(i, j, k, n) = dt * FI(i, j, k, n) * A(i, j, k, 0);
    });
}

template <int NS>
void fill_hydro_source_impl(const int* lo, const int* hi, Fab SRC, Fab F0, Fab F1, Fab F2, Fab Q0, Fab Q1, Fab Q2,
                            Fab A0, Fab A1, Fab A2, Fab V, double dx0, double dx1, double dx2)
{
    launch_box("fill_hydro_source", lo, hi, [=] __device__(int i, int j, int k) {
        for (int n = 0; n < Dims<NS>::NVAR; ++n) {
            double volinv = 1.0 / V(i, j, k, 0);
            SRC(i, j, k, n) = SRC(i, j, k, n) +
                (F0(i, j, k, n) * A0(i, j, k, 0) - F0(i + 1, j, k, n) * A0(i + 1, j, k, 0)
               + F1(i, j, k, n) * A1(i, j, k, 0) - F1(i, j + 1, k, n) * A1(i, j + 1, k, 0)
               + F2(i, j, k, n) * A2(i, j, k, 0) - F2(i, j, k + 1, n) * A2(i, j, k + 1, 0)) * volinv;
            if (n == UEINT) {
                double pdivu = 0.5 * (Q0(i + 1, j, k, GDPRES) + Q0(i, j, k, GDPRES)) *
                                   (Q0(i + 1, j, k, GDU) - Q0(i, j, k, GDU)) / dx0 +
                               0.5 * (Q1(i, j + 1, k, GDPRES) + Q1(i, j, k, GDPRES)) *
                                   (Q1(i, j + 1, k, GDV) - Q1(i, j, k, GDV)) / dx1 +
                               0.5 * (Q2(i, j, k + 1, GDPRES) + Q2(i, j, k, GDPRES)) *
                                   (Q2(i, j, k + 1, GDW) - Q2(i, j, k, GDW)) / dx2;
                SRC(i, j, k, n) = SRC(i, j, k, n) - pdivu;
            }
        }
    });
}

template <int NS>
void divu_impl(const int* lo, const int* hi, Fab Q, Fab DIV, double dx0, double dx1, double dx2)
{
    launch_box("divu", lo, hi, [=] __device__(int i, int j, int k) {
        double dxinv = 1.0 / dx0, dyinv = 1.0 / dx1, dzinv = 1.0 / dx2;
        double ux = 0.25 * (+Q(i, j, k, QU) - Q(i - 1, j, k, QU)
                            + Q(i, j, k - 1, QU) - Q(i - 1, j, k - 1, QU)
                            + Q(i, j - 1, k, QU) - Q(i - 1, j - 1, k, QU)
                            + Q(i, j - 1, k - 1, QU) - Q(i - 1, j - 1, k - 1, QU)) * dxinv;
        double vy = 0.25 * (+Q(i, j, k, QV) - Q(i, j - 1, k, QV)
                            + Q(i, j, k - 1, QV) - Q(i, j - 1, k - 1, QV)
                            + Q(i - 1, j, k, QV) - Q(i - 1, j - 1, k, QV)
                            + Q(i - 1, j, k - 1, QV) - Q(i - 1, j - 1, k - 1, QV)) * dyinv;
        double wz = 0.25 * (+Q(i, j, k, QW) - Q(i, j, k - 1, QW)
                            + Q(i, j - 1, k, QW) - Q(i, j - 1, k - 1, QW)
                            + Q(i - 1, j, k, QW) - Q(i - 1, j, k - 1, QW)
                            + Q(i - 1, j - 1, k, QW) - Q(i - 1, j - 1, k - 1, QW)) * dzinv;
        DIV(i, j, k, 0) = ux + vy + wz;
    });
}

}  // namespace

// problem constants set by castro_set_problem (castro_host.cu)
namespace castro { const castro_problem& problem(); }

namespace {

struct SpeciesX { double x[MAX_SPEC]; };

// the ambient internal energy of initdata, Prob.F90:51-59, into *d_e (one
// EOS call; a single-thread kernel keeps it on the device EOS)
template <int NS, bool COUL>
void ambient_energy(double* d_e, SpeciesX xs, int from_T, double rho_a, double T_a, double p_a)
{
    const int one[3] = {0, 0, 0};
    launch_box<32>("initdata(ambient)", one, one, [=] __device__(int, int, int) {
        double s1 = 0.0, s2 = 0.0;
        for (int n = 0; n < NS; ++n) s1 = s1 + xs.x[n] * c_net.aion_inv[n];
        for (int n = 0; n < NS; ++n) s2 = s2 + xs.x[n] * c_net.zion[n] * c_net.aion_inv[n];
        EosResult r;
        if (from_T) {
            double abar = 1.0 / s1;
            r = eos_solve<EOS_RT, COUL>(rho_a, T_a, 0.0, abar, abar * s2);
        } else {
            r = eos_solve<EOS_RP, COUL>(rho_a, 1.e4, p_a, c_net.aion[0], c_net.zion[0]);
        }
        *d_e = r.e;
    });
}

template <int NS>
void initdata_impl(const int* lo, const int* hi, Fab U, const double* dx, const double* problo, const double* probhi)
{
    const castro_problem P = castro::problem();
    double* d_e = nullptr;
    if (cudaMallocAsync(&d_e, sizeof(double), stream()) != cudaSuccess) { set_error(1, "initdata: alloc"); return; }
    SpeciesX xs;
    for (int n = 0; n < MAX_SPEC; ++n) xs.x[n] = P.X[n];
    const int from_T = P.ambient_from_T;
    const double rho_a = P.dens_ambient, p_a = P.p_ambient, T_a = P.T_ambient;
    if (coulomb_on()) ambient_energy<NS, true>(d_e, xs, from_T, rho_a, T_a, p_a);
    else ambient_energy<NS, false>(d_e, xs, from_T, rho_a, T_a, p_a);
    const double r_init = P.r_init;
    const double vctr = (4.0 / 3.0) * 3.14159265358979323846 * (r_init * r_init * r_init);
    const double e_exp = P.exp_energy / vctr / P.dens_ambient;
    const double c0 = (problo[0] + probhi[0]) / 2.e0, c1 = (problo[1] + probhi[1]) / 2.e0, c2 = (problo[2] + probhi[2]) / 2.e0;
    const double pl0 = problo[0], pl1 = problo[1], pl2 = problo[2];
    const double dx0 = dx[0], dx1 = dx[1], dx2 = dx[2];
    const int nsub = P.nsub;
    const double T_init = P.T_init, pert_amp = P.pert_amp;
    Fab PERT{};
    const bool has_pert = P.pert != nullptr;
    if (has_pert) PERT = make_fab(P.pert, P.pert_lo, P.pert_hi);
    launch_box("initdata", lo, hi, [=] __device__(int i, int j, int k) {
        double e_ambient = *d_e;
        double xmin = pl0 + dx0 * (double)i;
        double ymin = pl1 + dx1 * (double)j;
        double zmin = pl2 + dx2 * (double)k;
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
        double eint = ((double)npert * e_exp + (double)nambient * e_ambient) / (double)(nsub * nsub * nsub);
        double rho = rho_a;
        if (has_pert) rho = rho_a * (1.0 + pert_amp * PERT(i, j, k, 0));
        U(i, j, k, URHO) = rho;
        U(i, j, k, UMX) = 0.e0;
        U(i, j, k, UMY) = 0.e0;
        U(i, j, k, UMZ) = 0.e0;
        U(i, j, k, UTEMP) = T_init;
        U(i, j, k, UEDEN) = U(i, j, k, URHO) * eint;
        U(i, j, k, UEINT) = U(i, j, k, URHO) * eint;
#pragma unroll
        for (int n = 0; n < NS; ++n) U(i, j, k, UFS + n) = xs.x[n] * U(i, j, k, URHO);
    });
    cudaFreeAsync(d_e, stream());
}

template <int NS>
__global__ void k_blast(BoxRange r, Fab U, double pl0, double pl1, double pl2, double dx0, double dx1, double dx2,
                        double c0, double c1, double c2, double max_density, double* bm, double* br)
{
    __shared__ double sm[2][32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0, rr = 0.0;
    if (t < r.n) {
        int i = r.lx + (int)(t % r.nx);
        long long t2 = t / r.nx;
        int j = r.ly + (int)(t2 % r.ny);
        int k = r.lz + (int)(t2 / r.ny);
        double x = pl0 + (i + 0.5) * dx0 - c0;
        double y = pl1 + (j + 0.5) * dx1 - c1;
        double z = pl2 + (k + 0.5) * dx2 - c2;
        double rho = U(i, j, k, URHO);
        if (fabs(rho - max_density) / max_density <= 0.1) {
            m = rho;
            rr = rho * sqrt(x * x + y * y + z * z);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        m += __shfl_xor_sync(0xffffffffu, m, o);
        rr += __shfl_xor_sync(0xffffffffu, rr, o);
    }
    if ((threadIdx.x & 31) == 0) { sm[0][threadIdx.x >> 5] = m; sm[1][threadIdx.x >> 5] = rr; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += sm[0][w]; b += sm[1][w]; }
        atomicAdd(bm, a);
        atomicAdd(br, b);
    }
}

}  // namespace

namespace {
template <int NS> void emd_impl(const int* lo, const int* hi, Fab U) { clean_impl<NS, 0>("enforce_minimum_density", lo, hi, U); }
template <int NS> void nsp_impl(const int* lo, const int* hi, Fab U) { clean_impl<NS, 1>("normalize_species", lo, hi, U); }
template <int NS> void rie_impl(const int* lo, const int* hi, Fab U) { clean_impl<NS, 2>("reset_internal_e", lo, hi, U); }
template <int NS> void ctp_impl(const int* lo, const int* hi, Fab U) { clean_impl<NS, 3>("compute_temp", lo, hi, U); }
template <int NS> void cls_impl(const int* lo, const int* hi, Fab U) { clean_impl<NS, 4>("castro_clean_state", lo, hi, U); }

template <int NS>
void blast_impl(const int* lo, const int* hi, Fab U, const double* dx, const double* problo, const double* probhi,
                double* bm, double* br, double max_density)
{
    BoxRange r = make_range(lo, hi);
    if (r.n == 0) return;
    const int B = 128;
    // center of Source/Castro_nd.F90:377 (probhi - problo)/2, as written there
    k_blast<NS><<<(unsigned)((r.n + B - 1) / B), B, 0, stream()>>>(
        r, U, problo[0], problo[1], problo[2], dx[0], dx[1], dx[2],
        (probhi[0] - problo[0]) / 2.0, (probhi[1] - problo[1]) / 2.0, (probhi[2] - problo[2]) / 2.0,
        max_density, bm, br);
    check_launch("calculate_blast_radius");
}

__global__ void k_denerror(BoxRange r, Fab D, int8_t* tag, int tlx, int tly, int tlz, int tnx, int tny,
                           int8_t tagval)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= r.n) return;
    int i = r.lx + (int)(t % r.nx);
    long long t2 = t / r.nx;
    int j = r.ly + (int)(t2 % r.ny);
    int k = r.lz + (int)(t2 / r.ny);
    double c = D(i, j, k, 0);
    double ax = fabs(D(i + 1, j, k, 0) - c);
    double ay = fabs(D(i, j + 1, k, 0) - c);
    double az = fabs(D(i, j, k + 1, 0) - c);
    ax = DMAX(ax, fabs(c - D(i - 1, j, k, 0)));
    ay = DMAX(ay, fabs(c - D(i, j - 1, k, 0)));
    az = DMAX(az, fabs(c - D(i, j, k - 1, 0)));
    if (DMAX(DMAX(ax, ay), az) >= fabs(0.25 * c))
        tag[(long long)(i - tlx) + (long long)tnx * ((long long)(j - tly) + (long long)tny * (k - tlz))] = tagval;
}
}  // namespace

// ===========================================================================
// extern "C" entry points, Source/Castro_F.H:19-161
// ===========================================================================
extern "C" {

void ctoprim(const int* lo, const int* hi, const double* u, const int* u_lo, const int* u_hi,
             const double* q, const int* q_lo, const int* q_hi, const double* qaux, const int* qa_lo, const int* qa_hi)
{
    CASTRO_DISPATCH_NS(ctoprim_impl, lo, hi, make_fab(u, u_lo, u_hi), make_fab(q, q_lo, q_hi),
                       make_fab(qaux, qa_lo, qa_hi));
}

void enforce_minimum_density(const int* lo, const int* hi, double* s, const int* s_lo, const int* s_hi)
{
    CASTRO_DISPATCH_NS(emd_impl, lo, hi, make_fab(s, s_lo, s_hi));
}

void normalize_species(const int* lo, const int* hi, double* s, const int* s_lo, const int* s_hi)
{
    CASTRO_DISPATCH_NS(nsp_impl, lo, hi, make_fab(s, s_lo, s_hi));
}

void reset_internal_e(const int* lo, const int* hi, double* s, const int* s_lo, const int* s_hi)
{
    CASTRO_DISPATCH_NS(rie_impl, lo, hi, make_fab(s, s_lo, s_hi));
}

void compute_temp(const int* lo, const int* hi, double* s, const int* s_lo, const int* s_hi)
{
    CASTRO_DISPATCH_NS(ctp_impl, lo, hi, make_fab(s, s_lo, s_hi));
}

void castro_clean_state(const int* lo, const int* hi, double* s, const int* s_lo, const int* s_hi)
{
    CASTRO_DISPATCH_NS(cls_impl, lo, hi, make_fab(s, s_lo, s_hi));
}

void estdt(const int* lo, const int* hi, const double* s, const int* s_lo, const int* s_hi, const double* dx, double* dt)
{
    CASTRO_DISPATCH_NS(estdt_impl, lo, hi, make_fab(s, s_lo, s_hi), dx, dt);
}

// MultiFab::Saxpy of Source/Castro_advance.cpp:74 (U_new = U_old + dt * source)
// on n contiguous doubles of one FAB
__global__ void k_saxpy_host_dt(double* u, const double* src, long long n, double dt)
{
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m < n) u[m] = u[m] + dt * src[m];
}

// ---------------------------------------------------------------------------
// The AMR pieces of Castro.cpp (Castro::reflux, Source/Castro.cpp:451-483;
// Castro::avgDown, :486-504), which the reference delegates to AMReX's
// FluxRegister and amrex::average_down: the register of one side of a fine
// patch on the coarse faces it covers, and the conservative average of fine
// zones onto the coarse zones beneath them.  Fluxes are in store_flux's form,
// dt * F * A, on face boxes (node-centred in the normal direction).
// ---------------------------------------------------------------------------
}  // extern "C"

namespace {
// [lo, hi] inside [alo, ahi] (an empty box is inside anything)
bool box_inside(const int* lo, const int* hi, const int* alo, const int* ahi)
{
    for (int d = 0; d < 3; ++d)
        if (lo[d] <= hi[d] && (lo[d] < alo[d] || hi[d] > ahi[d])) return false;
    return true;
}
// the fine cells or faces under coarse [lo, hi] refined by r (faces: not refined along dir, dir < 0 for cells)
void refine_box(const int* lo, const int* hi, int r, int dir, int* flo, int* fhi)
{
    for (int d = 0; d < 3; ++d) {
        flo[d] = lo[d] * r;
        fhi[d] = d == dir ? hi[d] * r : hi[d] * r + r - 1;
    }
}
bool amr_args_ok(const char* who, bool ok)
{
    if (!ok) {
        char msg[160];
        snprintf(msg, sizeof msg, "%s: a box the call reads or writes lies outside its array", who);
        set_error(CASTRO_ERR_ARG, msg);
    }
    return ok;
}
}  // namespace

extern "C" {

void castro_flux_register_crse_init(const int* flo, const int* fhi, double* reg, const int* r_lo, const int* r_hi,
                                    const double* crse_flux, const int* c_lo, const int* c_hi, int ncomp)
{
    if (!amr_args_ok("castro_flux_register_crse_init",
                     ncomp > 0 && box_inside(flo, fhi, r_lo, r_hi) && box_inside(flo, fhi, c_lo, c_hi)))
        return;
    Fab R = make_fab(reg, r_lo, r_hi), F = make_fab(crse_flux, c_lo, c_hi);
    launch_box("castro_flux_register_crse_init", flo, fhi, [=] __device__(int i, int j, int k) {
        for (int n = 0; n < ncomp; ++n) R(i, j, k, n) = -F(i, j, k, n);
    });
}

void castro_flux_register_fine_add(const int* flo, const int* fhi, int dir, double* reg, const int* r_lo,
                                   const int* r_hi, const double* fine_flux, const int* f_lo, const int* f_hi,
                                   int ncomp, int ratio)
{
    if (dir < 0 || dir > 2 || ratio < 1) {
        set_error(CASTRO_ERR_ARG, "castro_flux_register_fine_add: dir 0..2, ratio >= 1");
        return;
    }
    int ffl[3], ffh[3];
    refine_box(flo, fhi, ratio, dir, ffl, ffh);
    if (!amr_args_ok("castro_flux_register_fine_add",
                     ncomp > 0 && box_inside(flo, fhi, r_lo, r_hi) && box_inside(ffl, ffh, f_lo, f_hi)))
        return;
    Fab R = make_fab(reg, r_lo, r_hi), F = make_fab(fine_flux, f_lo, f_hi);
    launch_box("castro_flux_register_fine_add", flo, fhi, [=] __device__(int i, int j, int k) {
        // the ratio^2 fine faces on coarse face (i,j,k): the same plane, ratio x ratio across it
        const int fi = i * ratio, fj = j * ratio, fk = k * ratio;
        const int na = dir == 0 ? 1 : ratio, nb = dir == 1 ? 1 : ratio, nc = dir == 2 ? 1 : ratio;
        for (int n = 0; n < ncomp; ++n) {
            double s = 0.0;
            for (int c = 0; c < nc; ++c)
                for (int b = 0; b < nb; ++b)
                    for (int a = 0; a < na; ++a) s = s + F(fi + a, fj + b, fk + c, n);
            R(i, j, k, n) = R(i, j, k, n) + s;
        }
    });
}

void castro_flux_register_reflux(const int* flo, const int* fhi, int dir, int side, double* state, const int* s_lo,
                                 const int* s_hi, const double* reg, const int* r_lo, const int* r_hi, int ncomp,
                                 double volume)
{
    if (dir < 0 || dir > 2 || (side != 0 && side != 1) || !(volume > 0.0)) {
        set_error(CASTRO_ERR_ARG, "castro_flux_register_reflux: dir 0..2, side 0/1, volume > 0");
        return;
    }
    int zlo[3] = {flo[0], flo[1], flo[2]}, zhi[3] = {fhi[0], fhi[1], fhi[2]};
    if (side == 0) { zlo[dir] -= 1; zhi[dir] -= 1; }
    if (!amr_args_ok("castro_flux_register_reflux",
                     ncomp > 0 && box_inside(flo, fhi, r_lo, r_hi) && box_inside(zlo, zhi, s_lo, s_hi)))
        return;
    Fab S = make_fab(state, s_lo, s_hi), R = make_fab(reg, r_lo, r_hi);
    const double scale = (side == 0 ? -1.0 : 1.0) / volume;
    launch_box("castro_flux_register_reflux", flo, fhi, [=] __device__(int i, int j, int k) {
        // side 0: the coarse zone is below the face (the fine patch above), side 1: above it
        const int zi = i - (side == 0 && dir == 0), zj = j - (side == 0 && dir == 1), zk = k - (side == 0 && dir == 2);
        for (int n = 0; n < ncomp; ++n) S(zi, zj, zk, n) = S(zi, zj, zk, n) + scale * R(i, j, k, n);
    });
}

void castro_average_down(const int* clo, const int* chi, double* crse, const int* c_lo, const int* c_hi,
                         const double* fine, const int* f_lo, const int* f_hi, int ncomp, int ratio)
{
    if (ratio < 1) {
        set_error(CASTRO_ERR_ARG, "castro_average_down: ratio >= 1");
        return;
    }
    int fl[3], fh[3];
    refine_box(clo, chi, ratio, -1, fl, fh);
    if (!amr_args_ok("castro_average_down",
                     ncomp > 0 && box_inside(clo, chi, c_lo, c_hi) && box_inside(fl, fh, f_lo, f_hi)))
        return;
    Fab C = make_fab(crse, c_lo, c_hi), F = make_fab(fine, f_lo, f_hi);
    const double inv = 1.0 / ((double)ratio * ratio * ratio);
    launch_box("castro_average_down", clo, chi, [=] __device__(int i, int j, int k) {
        for (int n = 0; n < ncomp; ++n) {
            double s = 0.0;
            for (int c = 0; c < ratio; ++c)
                for (int b = 0; b < ratio; ++b)
                    for (int a = 0; a < ratio; ++a) s = s + F(i * ratio + a, j * ratio + b, k * ratio + c, n);
            C(i, j, k, n) = s * inv;
        }
    });
}

void castro_saxpy(double* u, const double* src, long long n, double dt)
{
    if (n <= 0) return;
    k_saxpy_host_dt<<<(unsigned)((n + 255) / 256), 256, 0, stream()>>>(u, src, n, dt);
    check_launch("castro_saxpy");
}

void store_flux(const int* lo, const int* hi, double* fo, const int* fo_lo, const int* fo_hi,
                double* fi, const int* fi_lo, const int* fi_hi, double* a, const int* a_lo, const int* a_hi,
                const double dt)
{
    CASTRO_DISPATCH_NS(store_flux_impl, lo, hi, make_fab(fo, fo_lo, fo_hi), make_fab(fi, fi_lo, fi_hi),
                       make_fab(a, a_lo, a_hi), dt);
}

void fill_hydro_source(const int* lo, const int* hi,
                       const double* state, const int* s_lo, const int* s_hi,
                       const double* q, const int* q_lo, const int* q_hi,
                       double* source, const int* sr_lo, const int* sr_hi,
                       const double* flux0, const int* f0_lo, const int* f0_hi,
                       const double* flux1, const int* f1_lo, const int* f1_hi,
                       const double* flux2, const int* f2_lo, const int* f2_hi,
                       const double* qe0, const int* qe0_lo, const int* qe0_hi,
                       const double* qe1, const int* qe1_lo, const int* qe1_hi,
                       const double* qe2, const int* qe2_lo, const int* qe2_hi,
                       const double* area0, const int* a0_lo, const int* a0_hi,
                       const double* area1, const int* a1_lo, const int* a1_hi,
                       const double* area2, const int* a2_lo, const int* a2_hi,
                       const double* volume, const int* v_lo, const int* v_hi,
                       const double* dx, const double dt)
{
    (void)state; (void)s_lo; (void)s_hi; (void)q; (void)q_lo; (void)q_hi; (void)dt;
    CASTRO_DISPATCH_NS(fill_hydro_source_impl, lo, hi, make_fab(source, sr_lo, sr_hi),
                       make_fab(flux0, f0_lo, f0_hi), make_fab(flux1, f1_lo, f1_hi), make_fab(flux2, f2_lo, f2_hi),
                       make_fab(qe0, qe0_lo, qe0_hi), make_fab(qe1, qe1_lo, qe1_hi), make_fab(qe2, qe2_lo, qe2_hi),
                       make_fab(area0, a0_lo, a0_hi), make_fab(area1, a1_lo, a1_hi), make_fab(area2, a2_lo, a2_hi),
                       make_fab(volume, v_lo, v_hi), dx[0], dx[1], dx[2]);
}

void normalize_species_fluxes(const int* lo, const int* hi, double* flux, const int* f_lo, const int* f_hi)
{
    CASTRO_DISPATCH_NS(normalize_species_fluxes_impl, lo, hi, make_fab(flux, f_lo, f_hi));
}

void apply_av(const int* lo, const int* hi, const int idir, const double* dx,
              double* div, const int* d_lo, const int* d_hi, double* sb, const int* s_lo, const int* s_hi,
              double* flux, const int* f_lo, const int* f_hi)
{
    if (idir < 1 || idir > 3) { set_error(CASTRO_ERR_ARG, "apply_av: idir"); return; }
    CASTRO_DISPATCH_NS(apply_av_impl, lo, hi, idir - 1, dx[idir - 1], make_fab(div, d_lo, d_hi),
                       make_fab(sb, s_lo, s_hi), make_fab(flux, f_lo, f_hi));
}

void trans1(const int* lo, const int* hi, const int idir1, const int idir2,
            const double* q2m, const int* q2m_lo, const int* q2m_hi,
            double* q2mo, const int* q2mo_lo, const int* q2mo_hi,
            const double* q2p, const int* q2p_lo, const int* q2p_hi,
            double* q2po, const int* q2po_lo, const int* q2po_hi,
            const double* qaux, const int* qa_lo, const int* qa_hi,
            const double* f1, const int* f1_lo, const int* f1_hi,
            const double* q1, const int* q1_lo, const int* q1_hi, const double cdtdx)
{
    if (idir1 < 1 || idir1 > 3 || idir2 < 1 || idir2 > 3 || idir1 == idir2) { set_error(CASTRO_ERR_ARG, "trans1: idir"); return; }
    CASTRO_DISPATCH_NS(trans1_impl, lo, hi, idir1 - 1, idir2 - 1,
                       make_fab(q2m, q2m_lo, q2m_hi), make_fab(q2mo, q2mo_lo, q2mo_hi),
                       make_fab(q2p, q2p_lo, q2p_hi), make_fab(q2po, q2po_lo, q2po_hi),
                       make_fab(qaux, qa_lo, qa_hi), make_fab(f1, f1_lo, f1_hi), make_fab(q1, q1_lo, q1_hi), cdtdx);
}

void trans2(const int* lo, const int* hi, const int idir1, const int idir2, const int idir3,
            const double* qm, const int* qm_lo, const int* qm_hi,
            double* qmo, const int* qmo_lo, const int* qmo_hi,
            const double* qp, const int* qp_lo, const int* qp_hi,
            double* qpo, const int* qpo_lo, const int* qpo_hi,
            const double* qaux, const int* qa_lo, const int* qa_hi,
            const double* fyz, const int* fyz_lo, const int* fyz_hi,
            const double* fzy, const int* fzy_lo, const int* fzy_hi,
            const double* qy, const int* qy_lo, const int* qy_hi,
            const double* qz, const int* qz_lo, const int* qz_hi,
            const double hdtdx, const double cdtdy, const double cdtdz)
{
    (void)hdtdx;
    if (idir1 < 1 || idir1 > 3 || idir2 < 1 || idir2 > 3 || idir3 < 1 || idir3 > 3) { set_error(CASTRO_ERR_ARG, "trans2: idir"); return; }
    CASTRO_DISPATCH_NS(trans2_impl, lo, hi, idir1 - 1, idir2 - 1, idir3 - 1,
                       make_fab(qm, qm_lo, qm_hi), make_fab(qmo, qmo_lo, qmo_hi),
                       make_fab(qp, qp_lo, qp_hi), make_fab(qpo, qpo_lo, qpo_hi), make_fab(qaux, qa_lo, qa_hi),
                       make_fab(fyz, fyz_lo, fyz_hi), make_fab(fzy, fzy_lo, fzy_hi),
                       make_fab(qy, qy_lo, qy_hi), make_fab(qz, qz_lo, qz_hi), cdtdy, cdtdz);
}

void compute_flux(const int* lo, const int* hi,
                  const double* ql, const int* ql_lo, const int* ql_hi,
                  const double* qr, const int* qr_lo, const int* qr_hi,
                  double* flux, const int* fx_lo, const int* fx_hi,
                  double* q_int, const int* qi_lo, const int* qi_hi,
                  double* qe, const int* qe_lo, const int* qe_hi,
                  const double* qaux, const int* qa_lo, const int* qa_hi, const int idir)
{
    if (idir < 1 || idir > 3) { set_error(CASTRO_ERR_ARG, "compute_flux: idir"); return; }
    CASTRO_DISPATCH_NS(compute_flux_impl, lo, hi, make_fab(ql, ql_lo, ql_hi), make_fab(qr, qr_lo, qr_hi),
                       make_fab(flux, fx_lo, fx_hi), make_fab(q_int, qi_lo, qi_hi), make_fab(qe, qe_lo, qe_hi),
                       make_fab(qaux, qa_lo, qa_hi), idir - 1);
}

void divu(const int* lo, const int* hi, double* q, const int* q_lo, const int* q_hi,
          const double* dx, double* div, const int* d_lo, const int* d_hi)
{
    CASTRO_DISPATCH_NS(divu_impl, lo, hi, make_fab(q, q_lo, q_hi), make_fab(div, d_lo, d_hi), dx[0], dx[1], dx[2]);
}

void trace_ppm(const int* lo, const int* hi, const int* vlo, const int* vhi, const int idir,
               const double* q, const int* q_lo, const int* q_hi,
               const double* qaux, const int* qa_lo, const int* qa_hi,
               double* qm, const int* qm_lo, const int* qm_hi,
               double* qp, const int* qp_lo, const int* qp_hi,
               const int* domlo, const int* domhi, const double* dx, const double dt)
{
    (void)domlo; (void)domhi;
    if (idir < 1 || idir > 3) { set_error(CASTRO_ERR_ARG, "trace_ppm: idir"); return; }
    CASTRO_DISPATCH_NS(trace_impl, lo, hi, vlo, vhi, idir - 1, make_fab(q, q_lo, q_hi), make_fab(qaux, qa_lo, qa_hi),
                       make_fab(qm, qm_lo, qm_hi), make_fab(qp, qp_lo, qp_hi), dt / dx[idir - 1]);
}

void initdata(const int* lo, const int* hi, double* s, const int* s_lo, const int* s_hi,
              const double* dx, const double* problo, const double* probhi)
{
    CASTRO_DISPATCH_NS(initdata_impl, lo, hi, make_fab(s, s_lo, s_hi), dx, problo, probhi);
}

void denerror(const int* lo, const int* hi, int8_t* tag, const int* tag_lo, const int* tag_hi,
              const double* den, const int* den_lo, const int* den_hi, const int8_t tagval, const int8_t clearval)
{
    (void)clearval;
    BoxRange r = make_range(lo, hi);
    if (r.n == 0) return;
    const int B = 128;
    k_denerror<<<(unsigned)((r.n + B - 1) / B), B, 0, stream()>>>(
        r, make_fab(den, den_lo, den_hi), tag, tag_lo[0], tag_lo[1], tag_lo[2],
        tag_hi[0] - tag_lo[0] + 1, tag_hi[1] - tag_lo[1] + 1, tagval);
    check_launch("denerror");
}

void calculate_blast_radius(const int* lo, const int* hi, double* s, const int* s_lo, const int* s_hi,
                            const double* dx, const double* problo, const double* probhi,
                            double* blast_mass, double* blast_radius, const double max_density)
{
    CASTRO_DISPATCH_NS(blast_impl, lo, hi, make_fab(s, s_lo, s_hi), dx, problo, probhi, blast_mass, blast_radius,
                       max_density);
}

}  // extern "C"

namespace castro {
void upload_constants_abi(const EosTableDev& e, const NetworkDev& n)
{
    cudaMemcpyToSymbol(c_eos, &e, sizeof e);
    cudaMemcpyToSymbol(c_net, &n, sizeof n);
}
}  // namespace castro
