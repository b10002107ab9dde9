// castro_device.cuh -- per-zone and per-face device stages of the CTU hydro
// advance (Helmholtz EOS, state cleaning, conserved->primitive, PPM trace,
// CGF Riemann, transverse corrections), shared by the per-routine C-ABI
// kernels (castro_abi.cu), the fused batched pipeline (castro_sim.cu) and the
// reverse-mode stages (castro_adjoint.cuh).
//
// FP64 throughout.  Statement order follows the reference Fortran so that a
// build with -DCASTRO_EXACT --fmad=false reproduces a non-contracting CPU build
// bit for bit; the default build contracts to FMA and factors the biquintic
// table interpolation (see eos_eval), which changes results only by rounding.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

// Stages that are plain arithmetic are callable from host code as well, so the
// reverse-mode stages built on them can be checked on a CPU.
#define CASTRO_HD __host__ __device__ __forceinline__

namespace castro {

// ---- index maps, Source/Castro_nd.F90:14-57 (0-based) ----
constexpr int URHO = 0, UMX = 1, UMY = 2, UMZ = 3, UEDEN = 4, UEINT = 5, UTEMP = 6, UFS = 7;
constexpr int QRHO = 0, QU = 1, QV = 2, QW = 3, QGAME = 4, QPRES = 5, QREINT = 6, QTEMP = 7, QFS = 8;
constexpr int QGAMC = 0, QC = 1, QDPDR = 2, QDPDE = 3, NQAUX = 4;
constexpr int GDRHO = 0, GDU = 1, GDV = 2, GDW = 3, GDPRES = 4, GDGAME = 5, NGDNV = 6;

// Compact primitive "state" used on faces: absolute velocities, no QGAME/QTEMP
// (neither is ever read from an interface state by the reference).
constexpr int SRHO = 0, SU = 1, SV = 2, SW = 3, SPRES = 4, SREI = 5, SX = 6;

template <int NS>
struct Dims {
    static constexpr int NVAR = 7 + NS;
    static constexpr int QVAR = 8 + NS;
    static constexpr int NQS = 6 + NS;   // compact face state
    static constexpr int NTF = 7 + NS;   // transverse flux record: URHO,UMX,UMY,UMZ,UEDEN,species,GDPRES,GDU_n
};
constexpr int MAX_SPEC = 13;

// ---- physical floors, Source/Castro_nd.F90:59-65 ----
constexpr double small_dens = 1.0e-12;
constexpr double small_temp = 1.0e3;
constexpr double small_pres = 1.e-200;
constexpr double smallu = 1.e-12;
constexpr double small = 1.e-8;
constexpr double dual_energy_eta1 = 1.e0;
constexpr double dual_energy_eta2 = 1.e-4;   // Source/Castro_nd.F90:180
constexpr double cfl = 0.5;
constexpr double SIXTH = 1.0 / 6.0;
constexpr double TWO3RD = 2.0 / 3.0;

// ---- EOS table layout on the device ----
constexpr int IMAX = 541, JMAX = 201;
constexpr int NODE_STRIDE = 16;   // doubles per (i,j) node record (128 B)
// node record slots: the f family in "(density order a, temperature order b)"
// order, then the dp/dd family
enum { N_F = 0, N_FT, N_FTT, N_FD, N_FDD, N_FDT, N_FDDT, N_FDTT, N_FDDTT,
       N_DPDF, N_DPDFT, N_DPDFD, N_DPDFDT };
// per-row records: t/d, dt/dd, dt2/dd2, dti/ddi, dt2i/dd2i
constexpr int ROW_STRIDE = 8;
// slot of a temperature / density row record holding the next node's value
// (the cell's upper bound); the record is one 64-byte line
constexpr int ROW_NEXT = 5;

struct EosTableDev {
    const double* node;   // [JMAX][IMAX][NODE_STRIDE]
    const double* trow;   // [JMAX][ROW_STRIDE]
    const double* drow;   // [IMAX][ROW_STRIDE]
    double tlo, dlo, tstpi, dstpi, mintemp;
    double asoli3, kergavo, avo_eos, sioncon, kerg;
    // incremented when a Newton inversion ends unconverged after 100
    // iterations (the reference continues silently, eos.F90:193-554)
    unsigned long long* fail_count;
};

struct NetworkDev {
    int nspec;
    double aion[MAX_SPEC], zion[MAX_SPEC], aion_inv[MAX_SPEC];
    // 1: the interface pressure in the normal momentum flux, as full Castro has
    // it in Cartesian geometry (castro_set_momentum_flux_pressure); 0, the
    // default: the reference's compute_flux, whose momentum flux is rho u u
    // alone (Source/riemann.F90:306-308)
    int mom_flux_p;
    // 1: the EOS with Coulomb corrections (castro_set_coulomb_corrections); 0,
    // the default: the reference's eos.F90, which has none
    int coulomb;
};

// Each translation unit holds its own copy; castro_upload_constants_<tu>()
// fills it (see castro_host.cu).
static __constant__ EosTableDev c_eos;
static __constant__ NetworkDev c_net;

// the library's Coulomb setting (castro_set_coulomb_corrections), read by the
// host code that launches the EOS kernels to pick their instantiation
bool coulomb_on();

CASTRO_HD double fmaxf_(double a, double b) { return (a > b) ? a : b; }
CASTRO_HD double fminf_(double a, double b) { return (a < b) ? a : b; }
#define DMAX(a, b) ::castro::fmaxf_((a), (b))
#define DMIN(a, b) ::castro::fminf_((a), (b))

// ---------------------------------------------------------------------------
// Helmholtz EOS, Source/eos.F90:141-576
// ---------------------------------------------------------------------------
// quintic Hermite basis, eos.F90:740-911
CASTRO_HD double psi0(double z)   { return z * z * z * (z * (-6.0 * z + 15.0) - 10.0) + 1.0; }
CASTRO_HD double dpsi0(double z)  { return z * z * (z * (-30.0 * z + 60.0) - 30.0); }
CASTRO_HD double ddpsi0(double z) { return z * (z * (-120.0 * z + 180.0) - 60.0); }
CASTRO_HD double psi1(double z)   { return z * (z * z * (z * (-3.0 * z + 8.0) - 6.0) + 1.0); }
CASTRO_HD double dpsi1(double z)  { return z * z * (z * (-15.0 * z + 32.0) - 18.0) + 1.0; }
CASTRO_HD double ddpsi1(double z) { return z * (z * (-60.0 * z + 96.0) - 36.0); }
CASTRO_HD double psi2(double z)   { return 0.5 * z * z * (z * (z * (-z + 3.0) - 3.0) + 1.0); }
CASTRO_HD double dpsi2(double z)  { return 0.5 * z * (z * (z * (-5.0 * z + 12.0) - 9.0) + 2.0); }
CASTRO_HD double ddpsi2(double z) { return 0.5 * (z * (z * (-20.0 * z + 36.0) - 18.0) + 2.0); }
// cubic Hermite basis, eos.F90:955-1031
CASTRO_HD double xpsi0(double z)  { return z * z * (2.0 * z - 3.0) + 1.0; }
CASTRO_HD double xpsi1(double z)  { return z * (z * (z - 2.0) + 1.0); }

// Fortran INT() of a table coordinate, with the overflow/NaN guard the
// conversion needs in C.
CASTRO_HD int table_trunc(double x)
{
    if (!(x < 1.0e6)) x = 1.0e6;
    if (x < -1.0e6) x = -1.0e6;
    return (int)x;
}

// Weights of one table axis: w[a][0] at the lower node, w[a][1] at the upper
// node, a = value / first / second derivative order.
struct Basis6 { double w[3][2]; };
struct Basis4 { double w[2][2]; };

// density-direction weights (si*d, dsi*d) and cubic weights; depend only on
// din, so they are formed once per EOS call.
struct DensityBasis {
    int iat;
    Basis6 si, dsi;
    Basis4 xsi;
};

// log10 of a table coordinate, good to ~1e-5 of a cell (single-precision
// hardware log2; every argument here is a positive temperature or density far
// inside float range, and NaN stays NaN): the cell it selects is settled
// against the node values right after, so the cell -- and every result -- is
// the one a double-precision log10 leads to.
CASTRO_HD double table_log10(double x)
{
#ifdef __CUDA_ARCH__
    return (double)__log2f((float)x) * 0.30102999566398119521;
#else
    return log10(x);   // host builds of the stages (the adjoint self-test)
#endif
}

__device__ __forceinline__ void density_basis(double din, DensityBasis& B)
{
    int iat = table_trunc((table_log10(din) - c_eos.dlo) * c_eos.dstpi);   // eos.F90:244-245
    iat = iat > IMAX - 2 ? IMAX - 2 : iat;
    iat = iat < 0 ? 0 : iat;
    // Near a node the rounding of the logarithm decides the cell (the last bit
    // of a double log10, or the ~1e-5 cell of table_log10): the estimate is
    // settled against the node values, so that the cell is the one whose nodes
    // bracket the argument, whatever the logarithm returned.
    const double* dr = c_eos.drow + (size_t)iat * ROW_STRIDE;
    double d0 = __ldg(dr + 0), dd = __ldg(dr + 1), dd2 = __ldg(dr + 2), ddi = __ldg(dr + 3);
    const double d1 = __ldg(dr + ROW_NEXT);
    if ((iat > 0 && din < d0) || (iat < IMAX - 2 && din >= d1)) {
        iat += din < d0 ? -1 : 1;
        dr = c_eos.drow + (size_t)iat * ROW_STRIDE;
        d0 = __ldg(dr + 0); dd = __ldg(dr + 1); dd2 = __ldg(dr + 2); ddi = __ldg(dr + 3);
    }
    B.iat = iat;
    double xd = DMAX((din - d0) * ddi, 0.0);                         // eos.F90:287
    double mxd = 1.0 - xd;
    B.si.w[0][0] = psi0(xd);
    B.si.w[1][0] = psi1(xd) * dd;
    B.si.w[2][0] = psi2(xd) * dd2;
    B.si.w[0][1] = psi0(mxd);
    B.si.w[1][1] = -psi1(mxd) * dd;
    B.si.w[2][1] = psi2(mxd) * dd2;
    B.dsi.w[0][0] = dpsi0(xd) * ddi;
    B.dsi.w[1][0] = dpsi1(xd);
    B.dsi.w[2][0] = dpsi2(xd) * dd;
    B.dsi.w[0][1] = -dpsi0(mxd) * ddi;
    B.dsi.w[1][1] = dpsi1(mxd);
    B.dsi.w[2][1] = -dpsi2(mxd) * dd;
    B.xsi.w[0][0] = xpsi0(xd);
    B.xsi.w[1][0] = xpsi1(xd) * dd;
    B.xsi.w[0][1] = xpsi0(mxd);
    B.xsi.w[1][1] = -xpsi1(mxd) * dd;
}

// Quantities of one EOS evaluation at (rho, T) that the hydro path consumes.
struct EosEval {
    double p, e, dpdT, dpdr, dedT, dedr, gam1;
};

struct EosConst {   // per-call constants of the Newton loop
    double den, deni, ytot1, ye, din, zbar;
};

// Coulomb corrections of an ion plasma in a uniform electron background (off
// by default: the reference's eos.F90 has none; its 2017 runs had them on,
// scaling/summitdev_20171020/1.out:14).  The fits of Yakovlev & Shalybkov
// (1989) as the Helmholtz EOS applies them (Timmes & Swesty 2000): with n_i =
// N_A rho / abar, the ion-sphere radius a = (3 / (4 pi n_i))^(1/3) and the
// coupling Gamma = zbar^2 q_e^2 / (a k T), the excess energy per ion in kT is
// a1 Gamma + b1 Gamma^(1/4) + c1 Gamma^(-1/4) + d1 for Gamma >= 1 and
// -3 c2 Gamma^(3/2) + a2 Gamma^b2 below (c2 = 1 / (2 sqrt 3), Debye-Hueckel),
// the excess pressure a third of the excess energy density; Gamma goes as
// rho^(1/3) / T.  Operation for operation the oracle's coulomb(), whose cube
// root and power are the host libm's: the two agree to an ulp, not bit for bit.
namespace coul {
constexpr double QE = 4.80320427e-10;   // electron charge, esu
constexpr double A1 = -0.898004, B1 = 0.96786, C1 = 0.220703, D1 = -0.86097;
constexpr double A2 = 0.29561, B2 = 1.9885, C2 = 0.288675;
constexpr double FOUR_PI = 4.0 * 3.14159265358979323846;
}  // namespace coul

struct CoulombTerms {
    double p, e, dedt, dpdd, dpdt, dedd;
};

__device__ __forceinline__ void coulomb_terms(double den, double temp, double ytot1, double zbar, double pion,
                                              double dpiondd, double dpiondt, CoulombTerms& c)
{
    double xni = c_eos.avo_eos * ytot1 * den;
    double a_ion = cbrt(3.0 / (coul::FOUR_PI * xni));
    double gam = zbar * zbar * coul::QE * coul::QE / (a_ion * c_eos.kerg * temp);
    double gdd = gam / (3.0 * den);
    double gdt = -gam / temp;
    double y = c_eos.kergavo * ytot1;
    if (gam >= 1.0) {
        double x = sqrt(sqrt(gam));
        double u = coul::A1 * gam + coul::B1 * x + coul::C1 / x + coul::D1;
        double du = coul::A1 + 0.25 * (coul::B1 * x - coul::C1 / x) / gam;
        c.e = y * temp * u;
        c.dedd = y * temp * du * gdd;
        c.dedt = y * u + y * temp * du * gdt;
        c.p = den * c.e / 3.0;
        c.dpdd = (c.e + den * c.dedd) / 3.0;
        c.dpdt = den * c.dedt / 3.0;
    } else {
        double sg = sqrt(gam);
        double g32 = gam * sg;
        double gb = pow(gam, coul::B2);
        double z = coul::C2 * g32 - coul::A2 * gb / 3.0;
        double dz = 1.5 * coul::C2 * sg - coul::A2 * coul::B2 * gb / (3.0 * gam);
        c.p = -pion * z;
        c.dpdd = -(dpiondd * z + pion * dz * gdd);
        c.dpdt = -(dpiondt * z + pion * dz * gdt);
        c.e = 3.0 * c.p / den;
        c.dedd = 3.0 * c.dpdd / den - 3.0 * c.p / (den * den);
        c.dedt = 3.0 * c.dpdt / den;
    }
}

// The electron-positron part plus radiation and ions at temperature temp,
// eos.F90:195-518 (entropy, eta and xne are not formed: no hydro consumer).
// ENERGY_ONLY forms r.e and r.dedT alone -- all that a Newton iteration on e
// (EOS_RE) reads -- skipping the density derivatives, the pressure-derivative
// table and gamma_1; every quantity it does form is the full evaluation's,
// operation for operation.
// COUL adds the Coulomb corrections (full evaluations only).
enum { EVAL_FULL = 0, EVAL_ENERGY_ONLY = 1 };
template <int WHAT, bool COUL = false>
__device__ __forceinline__ void eos_eval_part(double temp, const EosConst& K, const DensityBasis& B, EosEval& r)
{
    constexpr bool FULL = WHAT == EVAL_FULL;
    const double den = K.den, deni = K.deni, ytot1 = K.ytot1, ye = K.ye, din = K.din;
    // radiation, :207-213
    double prad = c_eos.asoli3 * temp * temp * temp * temp;
    double dpraddd = 0.0;
#ifdef CASTRO_EXACT
    double tempi = 1.0 / temp;
    double dpraddt = 4.0 * prad * tempi;
#else
    // 4 a T^3 / 3 without the division by T (the production build's rounding)
    double dpraddt = 4.0 * (c_eos.asoli3 * temp * temp * temp);
#endif
    double erad = 3.0 * prad * deni;
    double deraddd = FULL ? -erad * deni : 0.0;
    double deraddt = 3.0 * dpraddt * deni;
    // ions, :220-226
    double pion = c_eos.kergavo * ytot1 * den * temp;
    double dpiondd = FULL ? c_eos.kergavo * ytot1 * temp : 0.0;
    double dpiondt = c_eos.kergavo * ytot1 * den;
    double eion = 1.5 * pion * deni;
    double deiondd = FULL ? (1.5 * dpiondd - eion) * deni : 0.0;
    double deiondt = 1.5 * dpiondt * deni;

    // temperature cell, :242-243
    int jat = table_trunc((table_log10(temp) - c_eos.tlo) * c_eos.tstpi);
    jat = jat > JMAX - 2 ? JMAX - 2 : jat;
    jat = jat < 0 ? 0 : jat;
    // settled against the node temperatures, as the density cell in
    // density_basis: a row record holds its cell's lower and upper nodes
    const double* tr = c_eos.trow + (size_t)jat * ROW_STRIDE;
    double t0 = __ldg(tr + 0), dt = __ldg(tr + 1), dt2 = __ldg(tr + 2), dti = __ldg(tr + 3), dt2i = __ldg(tr + 4);
    const double t1 = __ldg(tr + ROW_NEXT);
    if ((jat > 0 && temp < t0) || (jat < JMAX - 2 && temp >= t1)) {
        jat += temp < t0 ? -1 : 1;
        tr = c_eos.trow + (size_t)jat * ROW_STRIDE;
        t0 = __ldg(tr + 0); dt = __ldg(tr + 1); dt2 = __ldg(tr + 2); dti = __ldg(tr + 3); dt2i = __ldg(tr + 4);
    }
    double xt = DMAX((temp - t0) * dti, 0.0);                          // :286
    double mxt = 1.0 - xt;

    Basis6 st, dst, ddst;                                              // :292-332
    st.w[0][0] = psi0(xt);
    st.w[1][0] = psi1(xt) * dt;
    st.w[2][0] = psi2(xt) * dt2;
    st.w[0][1] = psi0(mxt);
    st.w[1][1] = -psi1(mxt) * dt;
    st.w[2][1] = psi2(mxt) * dt2;
    dst.w[0][0] = dpsi0(xt) * dti;
    dst.w[1][0] = dpsi1(xt);
    dst.w[2][0] = dpsi2(xt) * dt;
    dst.w[0][1] = -dpsi0(mxt) * dti;
    dst.w[1][1] = dpsi1(mxt);
    dst.w[2][1] = -dpsi2(mxt) * dt;
    ddst.w[0][0] = ddpsi0(xt) * dt2i;
    ddst.w[1][0] = ddpsi1(xt) * dti;
    ddst.w[2][0] = ddpsi2(xt);
    ddst.w[0][1] = ddpsi0(mxt) * dt2i;
    ddst.w[1][1] = -ddpsi1(mxt) * dti;
    ddst.w[2][1] = ddpsi2(mxt);

    // node records of the cell corners: c = di + 2*dj
    const double* nb = c_eos.node + ((size_t)jat * IMAX + B.iat) * NODE_STRIDE;
    const double* nc[4] = {nb, nb + NODE_STRIDE, nb + (size_t)IMAX * NODE_STRIDE,
                           nb + (size_t)IMAX * NODE_STRIDE + NODE_STRIDE};
    // table slot of (density order a, temperature order b)
    const int slot[3][3] = {{N_F, N_FT, N_FTT}, {N_FD, N_FDT, N_FDTT}, {N_FDD, N_FDDT, N_FDDTT}};

    double free_e, df_d, df_t, df_tt, df_dt;
#ifdef CASTRO_EXACT
    // h5 of eos.F90:915-950, term order as written there
    double fi[36];
    {
        const int tabs[9] = {N_F, N_FT, N_FTT, N_FD, N_FDD, N_FDT, N_FDDT, N_FDTT, N_FDDTT};
#pragma unroll
        for (int m = 0; m < 9; ++m)
#pragma unroll
            for (int c = 0; c < 4; ++c) fi[4 * m + c] = __ldg(nc[c] + tabs[m]);
    }
    auto h5 = [&](const Basis6& T, const Basis6& D) {
        const double w0t = T.w[0][0], w1t = T.w[1][0], w2t = T.w[2][0];
        const double w0mt = T.w[0][1], w1mt = T.w[1][1], w2mt = T.w[2][1];
        const double w0d = D.w[0][0], w1d = D.w[1][0], w2d = D.w[2][0];
        const double w0md = D.w[0][1], w1md = D.w[1][1], w2md = D.w[2][1];
        return fi[0] * w0d * w0t + fi[1] * w0md * w0t
             + fi[2] * w0d * w0mt + fi[3] * w0md * w0mt
             + fi[4] * w0d * w1t + fi[5] * w0md * w1t
             + fi[6] * w0d * w1mt + fi[7] * w0md * w1mt
             + fi[8] * w0d * w2t + fi[9] * w0md * w2t
             + fi[10] * w0d * w2mt + fi[11] * w0md * w2mt
             + fi[12] * w1d * w0t + fi[13] * w1md * w0t
             + fi[14] * w1d * w0mt + fi[15] * w1md * w0mt
             + fi[16] * w2d * w0t + fi[17] * w2md * w0t
             + fi[18] * w2d * w0mt + fi[19] * w2md * w0mt
             + fi[20] * w1d * w1t + fi[21] * w1md * w1t
             + fi[22] * w1d * w1mt + fi[23] * w1md * w1mt
             + fi[24] * w2d * w1t + fi[25] * w2md * w1t
             + fi[26] * w2d * w1mt + fi[27] * w2md * w1mt
             + fi[28] * w1d * w2t + fi[29] * w1md * w2t
             + fi[30] * w1d * w2mt + fi[31] * w1md * w2mt
             + fi[32] * w2d * w2t + fi[33] * w2md * w2t
             + fi[34] * w2d * w2mt + fi[35] * w2md * w2mt;
    };
    free_e = h5(st, B.si);
    df_d = FULL ? h5(st, B.dsi) : 0.0;
    df_t = h5(dst, B.si);
    df_tt = h5(ddst, B.si);
    df_dt = FULL ? h5(dst, B.dsi) : 0.0;
    (void)slot;
#else
    // Factored biquintic: contract the temperature direction first for each of
    // the three temperature weight sets, then the density direction.
    // 138 multiply-adds instead of the 540 operations of five h5 calls.
    double g0[3][2], g1[3][2], g2[3][2];   // [density order a][density node di]
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int dj = 0; dj < 2; ++dj) {
                    double v = __ldg(nc[di + 2 * dj] + slot[a][b]);
                    s0 = fma(v, st.w[b][dj], s0);
                    s1 = fma(v, dst.w[b][dj], s1);
                    s2 = fma(v, ddst.w[b][dj], s2);
                }
            g0[a][di] = s0; g1[a][di] = s1; g2[a][di] = s2;
        }
    free_e = 0.0; df_d = 0.0; df_t = 0.0; df_tt = 0.0; df_dt = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int di = 0; di < 2; ++di) {
            free_e = fma(g0[a][di], B.si.w[a][di], free_e);
            if (FULL) df_d = fma(g0[a][di], B.dsi.w[a][di], df_d);
            df_t = fma(g1[a][di], B.si.w[a][di], df_t);
            df_tt = fma(g2[a][di], B.si.w[a][di], df_tt);
            if (FULL) df_dt = fma(g1[a][di], B.dsi.w[a][di], df_dt);
        }
#endif
    if constexpr (!FULL) {
        // :468-472, :476-478 for e and de/dT
        double sele = -df_t * ye;
        double dsepdt = -df_tt * ye;
        double eele = ye * free_e + temp * sele;
        double deepdt = temp * dsepdt;
        r.e = erad + eion + eele;
        r.dedT = deraddt + deiondt + deepdt;
        return;
    }

    // cubic pressure-derivative interpolation, :362-409
    double xs0t = xpsi0(xt), xs1t = xpsi1(xt) * dt, xs0mt = xpsi0(mxt), xs1mt = -xpsi1(mxt) * dt;
    double dpepdd;
    {
        double f1 = __ldg(nc[0] + N_DPDF), f2 = __ldg(nc[1] + N_DPDF), f3 = __ldg(nc[2] + N_DPDF), f4 = __ldg(nc[3] + N_DPDF);
        double f5 = __ldg(nc[0] + N_DPDFT), f6 = __ldg(nc[1] + N_DPDFT), f7 = __ldg(nc[2] + N_DPDFT), f8 = __ldg(nc[3] + N_DPDFT);
        double f9 = __ldg(nc[0] + N_DPDFD), f10 = __ldg(nc[1] + N_DPDFD), f11 = __ldg(nc[2] + N_DPDFD), f12 = __ldg(nc[3] + N_DPDFD);
        double f13 = __ldg(nc[0] + N_DPDFDT), f14 = __ldg(nc[1] + N_DPDFDT), f15 = __ldg(nc[2] + N_DPDFDT), f16 = __ldg(nc[3] + N_DPDFDT);
        const double w0d = B.xsi.w[0][0], w1d = B.xsi.w[1][0], w0md = B.xsi.w[0][1], w1md = B.xsi.w[1][1];
        // h3, eos.F90:1034-1059
        dpepdd = f1 * w0d * xs0t + f2 * w0md * xs0t
               + f3 * w0d * xs0mt + f4 * w0md * xs0mt
               + f5 * w0d * xs1t + f6 * w0md * xs1t
               + f7 * w0d * xs1mt + f8 * w0md * xs1mt
               + f9 * w1d * xs0t + f10 * w1md * xs0t
               + f11 * w1d * xs0mt + f12 * w1md * xs0mt
               + f13 * w1d * xs1t + f14 * w1md * xs1t
               + f15 * w1d * xs1mt + f16 * w1md * xs1mt;
    }
    dpepdd = DMAX(ye * dpepdd, 0.0);

    // :464-489
    double x = din * din;
    double pele = x * df_d;
    double dpepdt = x * df_dt;
    x = ye * ye;
    double sele = -df_t * ye;
    double dsepdt = -df_tt * ye;
    double dsepdd = -df_dt * x;
    double eele = ye * free_e + temp * sele;
    double deepdt = temp * dsepdt;
    double deepdd = x * df_d + temp * dsepdd;

    double pres = prad + pion + pele;
    double ener = erad + eion + eele;
    double dpresdd = dpraddd + dpiondd + dpepdd;
    double dpresdt = dpraddt + dpiondt + dpepdt;
    double denerdd = deraddd + deiondd + deepdd;
    double denerdt = deraddt + deiondt + deepdt;
    if constexpr (COUL) {
        static_assert(FULL, "the Coulomb corrections enter full evaluations");
        CoulombTerms c;
        coulomb_terms(den, temp, ytot1, K.zbar, pion, dpiondd, dpiondt, c);
        if (pres + c.p > 0.0 && ener + c.e > 0.0) {   // kept only while the totals stay positive
            pres = pres + c.p;
            ener = ener + c.e;
            dpresdd = dpresdd + c.dpdd;
            dpresdt = dpresdt + c.dpdt;
            denerdd = denerdd + c.dedd;
            denerdt = denerdt + c.dedt;
        }
    }

    // :491-507
    double zz = pres * deni;
    double zzi = den / pres;
    double chit = temp / pres * dpresdt;
    double chid = dpresdd * zzi;
    double cv = denerdt;
    r.gam1 = chit * zz * chit / (temp * cv) + chid;
    r.p = pres;
    r.e = ener;
    r.dpdT = dpresdt;
    r.dpdr = dpresdd;
    r.dedT = denerdt;
    r.dedr = denerdd;
}

template <bool COUL = false>
__device__ __forceinline__ void eos_eval(double temp, const EosConst& K, const DensityBasis& B, EosEval& r)
{
    eos_eval_part<EVAL_FULL, COUL>(temp, K, B, r);
}

struct EosResult {
    double T, p, e, gam1, cs, dedT, dpdT, dpde, dpdr_e;
};

enum { EOS_RT = 1, EOS_RE = 2, EOS_RP = 3 };   // eos.F90:11-13

// eos(input, state): the Newton inversion of eos.F90:181-574.  v_want is e for
// EOS_RE and p for EOS_RP (ignored for EOS_RT).  OUTPUTS = false when the
// caller reads only T (and the input e or p back): the evaluation after
// convergence, which only forms the other outputs, is then not made.  COUL:
// with the Coulomb corrections -- a compile-time choice, so that the kernels
// instantiated without them (the default) carry none of their code; every
// kernel that calls the EOS is instantiated both ways and its launch picks
// the instantiation from the library's setting (coulomb_on()).
template <int MODE, bool COUL, bool OUTPUTS = true>
__device__ __forceinline__ EosResult eos_solve(double rho, double T, double v_want, double abar, double zbar)
{
    EosConst K;
    K.den = rho;
    K.ytot1 = 1.0 / abar;
    K.ye = zbar / abar;
    K.din = K.ye * rho;
    K.deni = 1.0 / rho;
    K.zbar = zbar;
    DensityBasis B;
    density_basis(K.din, B);

    bool converged = (MODE == EOS_RT);
    EosEval r;
    // The reference evaluates the full EOS at the top of every iteration and
    // leaves the loop right after the evaluation that follows convergence
    // (eos.F90:520-552), so only that last evaluation's outputs are used; for
    // EOS_RE the iterations before it form only e and de/dT.
    static_assert(OUTPUTS || MODE != EOS_RT, "an EOS_RT call exists for its outputs");
    bool full = false;
    double temp_last = T;
    for (int iter = 1; iter <= 100; ++iter) {
        double temp = T;
        if (converged) {
            if (OUTPUTS) {
                eos_eval<COUL>(temp, K, B, r);
                full = true;
            }
            break;
        }
        temp_last = temp;
        // (with the Coulomb corrections, every iteration's evaluation is the
        // full one: its e and de/dT are the light one's plus the corrections)
        if (MODE == EOS_RE && !COUL) eos_eval_part<EVAL_ENERGY_ONLY>(temp, K, B, r);
        else eos_eval<COUL>(temp, K, B, r);
        double temp_old = temp;
        double v = (MODE == EOS_RE) ? r.e : r.p;
        double dvdx = (MODE == EOS_RE) ? r.dedT : r.dpdT;
        temp = temp - (v - v_want) / dvdx;
        temp = DMAX(0.5 * temp_old, DMIN(temp, 2.0 * temp_old));
        temp = DMAX(c_eos.mintemp, temp);
        T = temp;
#ifdef CASTRO_EXACT
        double error = fabs((temp - temp_old) / temp_old);
        if (error < 1.e-8) converged = true;
#else
        // |dT / T_old| < 1e-8 without the division
        if (fabs(temp - temp_old) < 1.e-8 * fabs(temp_old)) converged = true;
#endif
    }
    // ended by the iteration limit: the reference's outputs are those of the
    // last iteration's evaluation, here a light one
    if (OUTPUTS && MODE == EOS_RE && !full) eos_eval<COUL>(temp_last, K, B, r);
    if (!converged && c_eos.fail_count) atomicAdd(c_eos.fail_count, 1ULL);
    EosResult o;
    o.T = T;
    if (!OUTPUTS) {
        o.e = v_want;
        o.p = o.gam1 = o.cs = o.dedT = o.dpdT = o.dpde = o.dpdr_e = 0.0;
        return o;
    }
    o.p = (MODE == EOS_RP) ? v_want : r.p;
    o.e = (MODE == EOS_RE) ? v_want : r.e;
    o.gam1 = r.gam1;
    o.cs = sqrt(r.gam1 * r.p / rho);                                   // :556
    o.dedT = r.dedT;
    o.dpdT = r.dpdT;
    o.dpde = r.dpdT / r.dedT;                                          // :502-503
    o.dpdr_e = r.dpdr - r.dpdT * r.dedr / r.dedT;
    return o;
}

// abar, zbar from rho*X as the state kernels form them (Castro_nd.F90:285-286)
template <int NS>
__device__ __forceinline__ void abar_zbar_cons(const double* u, double rhoInv, double& abar, double& zbar)
{
    double s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int n = 0; n < NS; ++n) s1 = s1 + u[UFS + n] * c_net.aion_inv[n];
#pragma unroll
    for (int n = 0; n < NS; ++n) s2 = s2 + u[UFS + n] * c_net.zion[n] * c_net.aion_inv[n];
    abar = 1.0 / (s1 * rhoInv);
    zbar = abar * (s2 * rhoInv);
}

// ---------------------------------------------------------------------------
// State cleaning on one zone, Source/Castro_nd.F90:69-297
// ---------------------------------------------------------------------------
template <int NS, bool COUL>
__device__ __forceinline__ void enforce_minimum_density_pt(double* u)
{
    if (u[URHO] < small_dens) {                                        // :95-119
#pragma unroll
        for (int n = 0; n < NS; ++n) u[UFS + n] = u[UFS + n] * (small_dens / u[URHO]);
        double s1 = 0.0, s2 = 0.0;
#pragma unroll
        for (int n = 0; n < NS; ++n) s1 = s1 + u[UFS + n] * c_net.aion_inv[n];
#pragma unroll
        for (int n = 0; n < NS; ++n) s2 = s2 + u[UFS + n] * c_net.zion[n] * c_net.aion_inv[n];
        double abar = 1.0 / (s1 / small_dens);
        double zbar = abar * (s2 / small_dens);
        EosResult r = eos_solve<EOS_RT, COUL>(small_dens, small_temp, 0.0, abar, zbar);
        u[URHO] = small_dens;
        u[UTEMP] = r.T;
        u[UMX] = 0.0;
        u[UMY] = 0.0;
        u[UMZ] = 0.0;
        u[UEINT] = small_dens * r.e;
        u[UEDEN] = u[UEINT];
    }
}

template <int NS>
__device__ __forceinline__ void normalize_species_pt(double* u)
{
    double rho = u[URHO];                                              // :152-154
#pragma unroll
    for (int n = 0; n < NS; ++n) u[UFS + n] = DMAX(1.0e-30 * rho, DMIN(rho, u[UFS + n]));
    double sum = 0.0;
#pragma unroll
    for (int n = 0; n < NS; ++n) sum = sum + u[UFS + n];
#pragma unroll
    for (int n = 0; n < NS; ++n) u[UFS + n] = u[UFS + n] / sum;
}

template <int NS, bool COUL>
__device__ __forceinline__ void reset_internal_e_pt(double* u)
{
    double rhoInv = 1.0 / u[URHO];                                     // :196-244
    double Up = u[UMX] * rhoInv;
    double Vp = u[UMY] * rhoInv;
    double Wp = u[UMZ] * rhoInv;
    double ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp);
    if (u[UEDEN] < 0.0) {
        if (u[UEINT] < 0.0) {
            double abar, zbar;
            abar_zbar_cons<NS>(u, rhoInv, abar, zbar);
            EosResult r = eos_solve<EOS_RT, COUL>(u[URHO], small_temp, 0.0, abar, zbar);
            u[UEINT] = u[URHO] * r.e;
        }
        u[UEDEN] = u[UEINT] + u[URHO] * ke;
    } else {
        double rho_eint = u[UEDEN] - u[URHO] * ke;
        if (rho_eint > 0.0 && rho_eint / u[UEDEN] > dual_energy_eta2) {
            u[UEINT] = rho_eint;
        } else if (u[UEINT] <= 0.0) {
            double abar, zbar;
            abar_zbar_cons<NS>(u, rhoInv, abar, zbar);
            EosResult r = eos_solve<EOS_RT, COUL>(u[URHO], small_temp, 0.0, abar, zbar);
            u[UEINT] = u[URHO] * r.e;
        }
    }
}

template <int NS, bool COUL>
__device__ __forceinline__ void compute_temp_pt(double* u)
{
    double rhoInv = 1.0 / u[URHO];                                     // :280-291
    double abar, zbar;
    abar_zbar_cons<NS>(u, rhoInv, abar, zbar);
    EosResult r = eos_solve<EOS_RE, COUL, false>(u[URHO], u[UTEMP], u[UEINT] * rhoInv, abar, zbar);   // reads T only
    u[UTEMP] = r.T;
    u[UEINT] = u[URHO] * r.e;
}

// Castro::clean_state on one zone (Source/Castro.cpp:563-591)
template <int NS, bool COUL>
__device__ __forceinline__ void clean_state_pt(double* u)
{
    enforce_minimum_density_pt<NS, COUL>(u);
    normalize_species_pt<NS>(u);
    reset_internal_e_pt<NS, COUL>(u);
    compute_temp_pt<NS, COUL>(u);
}

// estdt on one zone, Source/timestep.F90:446-468: min over directions of dx/(c+|u|)
template <int NS, bool COUL>
__device__ __forceinline__ double estdt_pt(const double* u, double dx0, double dx1, double dx2)
{
    double rhoInv = 1.0 / u[URHO];
    double abar, zbar;
    abar_zbar_cons<NS>(u, rhoInv, abar, zbar);
    EosResult r = eos_solve<EOS_RE, COUL>(u[URHO], u[UTEMP], u[UEINT] * rhoInv, abar, zbar);
    double ux = u[UMX] * rhoInv;
    double uy = u[UMY] * rhoInv;
    double uz = u[UMZ] * rhoInv;
    double c = r.cs;
    double dt1 = dx0 / (c + fabs(ux));
    double dt2 = dx1 / (c + fabs(uy));
    double dt3 = dx2 / (c + fabs(uz));
    return DMIN(DMIN(dt1, dt2), dt3);
}

// ctoprim on one zone, Source/Castro_hydro_nd.F90:115-164.  q is the full
// QVAR record, qaux the NQAUX record.
template <int NS, bool COUL>
__device__ __forceinline__ void ctoprim_pt(const double* u, double* q, double* qaux)
{
    q[QRHO] = u[URHO];
    double rhoinv = 1.0 / q[QRHO];
    q[QU] = u[UMX] * rhoinv;
    q[QV] = u[UMY] * rhoinv;
    q[QW] = u[UMZ] * rhoinv;
    double kineng = 0.5 * q[QRHO] * (q[QU] * q[QU] + q[QV] * q[QV] + q[QW] * q[QW]);
    if ((u[UEDEN] - kineng) / u[UEDEN] > dual_energy_eta1)
        q[QREINT] = (u[UEDEN] - kineng) * rhoinv;
    else
        q[QREINT] = u[UEINT] * rhoinv;
    q[QTEMP] = u[UTEMP];
#pragma unroll
    for (int n = 0; n < NS; ++n) q[QFS + n] = u[UFS + n] * rhoinv;
    double s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int n = 0; n < NS; ++n) s1 = s1 + q[QFS + n] * c_net.aion_inv[n];
#pragma unroll
    for (int n = 0; n < NS; ++n) s2 = s2 + q[QFS + n] * c_net.zion[n] * c_net.aion_inv[n];
    double abar = 1.0 / s1;
    double zbar = abar * s2;
    EosResult r = eos_solve<EOS_RE, COUL>(q[QRHO], q[QTEMP], q[QREINT], abar, zbar);
    q[QTEMP] = r.T;
    q[QREINT] = r.e * q[QRHO];
    q[QPRES] = r.p;
    q[QGAME] = q[QPRES] / q[QREINT] + 1.0;
    qaux[QDPDR] = r.dpdr_e;
    qaux[QDPDE] = r.dpde;
    qaux[QGAMC] = r.gam1;
    qaux[QC] = r.cs;
}

// ---------------------------------------------------------------------------
// PPM, Source/ppm.F90
// ---------------------------------------------------------------------------
// Loader concept: q(i,j,k,n) returns q component n (full QVAR numbering, only
// QRHO,QU,QV,QW,QPRES,QREINT,QFS.. are requested) and gamc(i,j,k) / c(i,j,k)
// the auxiliary values.

// uflatten, Source/ppm.F90:11-128
template <class L>
CASTRO_HD double uflatten(const L& ld, int i, int j, int k)
{
    const double shktst = 0.33, zcut1 = 0.75, zcut2 = 0.85;
    const double dzcut = 1.0 / (zcut2 - zcut1);
    double flatn = 1.0;
#pragma unroll
    for (int idir = 0; idir < 3; ++idir) {
        const int ex = idir == 0, ey = idir == 1, ez = idir == 2;
        const int qun = QU + idir;
        double pr = ld.q(i + ex, j + ey, k + ez, QPRES);
        double pl = ld.q(i - ex, j - ey, k - ez, QPRES);
        double dp2 = ld.q(i + 2 * ex, j + 2 * ey, k + 2 * ez, QPRES) - ld.q(i - 2 * ex, j - 2 * ey, k - 2 * ez, QPRES);
        double du = ld.q(i + ex, j + ey, k + ez, qun) - ld.q(i - ex, j - ey, k - ez, qun);
        double dp = pr - pl;
        int s = (dp > 0.0) ? -1 : 1;   // s = -ishft
        double denom = DMAX(small_pres, fabs(dp2));
        double denominv = 1.0 / denom;
        double zeta = fabs(dp) * denominv;
        double z = DMIN(1.0, DMAX(0.0, dzcut * (zeta - zcut1)));
        double tst = (du <= 0.0) ? 1.0 : 0.0;
        double tmp = DMIN(pr, pl);
        double chi = (fabs(dp) > shktst * tmp) ? tst : 0.0;

        pr = ld.q(i + (1 + s) * ex, j + (1 + s) * ey, k + (1 + s) * ez, QPRES);
        pl = ld.q(i + (s - 1) * ex, j + (s - 1) * ey, k + (s - 1) * ez, QPRES);
        dp2 = ld.q(i + (2 + s) * ex, j + (2 + s) * ey, k + (2 + s) * ez, QPRES)
            - ld.q(i + (s - 2) * ex, j + (s - 2) * ey, k + (s - 2) * ez, QPRES);
        du = ld.q(i + (1 + s) * ex, j + (1 + s) * ey, k + (1 + s) * ez, qun)
           - ld.q(i + (s - 1) * ex, j + (s - 1) * ey, k + (s - 1) * ez, qun);
        dp = pr - pl;
        denom = DMAX(small_pres, fabs(dp2));
        denominv = 1.0 / denom;
        zeta = fabs(dp) * denominv;
        double z2 = DMIN(1.0, DMAX(0.0, dzcut * (zeta - zcut1)));
        tst = (du <= 0.0) ? 1.0 : 0.0;
        tmp = DMIN(pr, pl);
        double chi2 = (fabs(dp) > shktst * tmp) ? tst : 0.0;
        flatn = DMIN(flatn, 1.0 - DMAX(chi2 * z2, chi * z));
    }
    return flatn;
}

// van Leer limited slope of ppm.F90:153-169
CASTRO_HD double vl_slope(double sm1, double s0, double sp1)
{
    double dsl = 2.0 * (s0 - sm1);
    double dsr = 2.0 * (sp1 - s0);
    if (dsl * dsr > 0.0) {
        double dsc = 0.5 * (sp1 - sm1);
        return copysign(1.0, dsc) * DMIN(DMIN(fabs(dsc), fabs(dsl)), fabs(dsr));
    }
    return 0.0;
}

// Interface value between a zone with value a and its right neighbour with
// value b, from their van Leer slopes da, db (ppm.F90:171-180 for sm, :193-202
// for sp).  The minus edge of a zone and the plus edge of its left neighbour
// are this same expression on the same operands in the same order.
CASTRO_HD double ppm_edge(double a, double b, double da, double db)
{
    double e = 0.5 * (b + a) - SIXTH * (db - da);
    e = DMAX(e, DMIN(b, a));
    return DMIN(e, DMAX(b, a));
}

// Flattening and monotonicity limiting of the edges of a zone with value s0,
// ppm.F90:204-236
CASTRO_HD void ppm_limit(double s0, double flatn, double& sm, double& sp)
{
    sm = flatn * sm + (1.0 - flatn) * s0;
    sp = flatn * sp + (1.0 - flatn) * s0;
    if ((sp - s0) * (s0 - sm) <= 0.0) {
        sp = s0;
        sm = s0;
    } else if (fabs(sp - s0) >= 2.0 * fabs(sm - s0)) {
        sp = 3.0 * s0 - 2.0 * sm;
    } else if (fabs(sm - s0) >= 2.0 * fabs(sp - s0)) {
        sm = 3.0 * s0 - 2.0 * sp;
    }
}

// ppm_reconstruct, Source/ppm.F90:132-236; s[0..4] = s(-2..2)
CASTRO_HD void ppm_reconstruct(const double* s, double flatn, double& smo, double& spo)
{
    double dsvl_l = vl_slope(s[0], s[1], s[2]);
    double dsvl_c = vl_slope(s[1], s[2], s[3]);
    double dsvl_r = vl_slope(s[2], s[3], s[4]);   // ppm.F90:184-191 repeats :162-169 for the centre slope
    double sm = ppm_edge(s[1], s[2], dsvl_l, dsvl_c);
    double sp = ppm_edge(s[2], s[3], dsvl_c, dsvl_r);
    ppm_limit(s[2], flatn, sm, sp);
    smo = sm;
    spo = sp;
}

// ppm_int_profile for one wave speed, Source/ppm.F90:260-303
CASTRO_HD void ppm_int_wave(double sm, double sp, double s6, double speed, double dtdx,
                                             double& Ip, double& Im)
{
    double sigma = fabs(speed) * dtdx;
    if (speed <= 0.0) {
        Ip = sp;
        Im = sm + 0.5 * sigma * (sp - sm + (1.0 - TWO3RD * sigma) * s6);
    } else {
        Ip = sp - 0.5 * sigma * (sp - sm - (1.0 - TWO3RD * sigma) * s6);
        Im = sm;
    }
}

// Characteristic projection of trace_ppm (ppm.F90:537-623 for the plus state,
// :637-734 for the minus state).  I[w][v] are the wave integrals of rho, un, p,
// rhoe (v = 0..3) for waves w = u-c, u, u+c; gam is the gamc integral of the
// reference wave.  'plus' selects the plus (right) state of face i.
CASTRO_HD void trace_project(const double I[3][4], double gam_g_ref, double un, double cc,
                                              bool plus, double& rho_o, double& un_o, double& rhoe_o, double& p_o)
{
    const int wr = plus ? 0 : 2;   // reference wave: fastest toward the interface
    double rho_ref = I[wr][0];
    double un_ref = I[wr][1];
    double p_ref = I[wr][2];
    double rhoe_g_ref = I[wr][3];
    rho_ref = DMAX(rho_ref, small_dens);
    double rho_ref_inv = 1.0 / rho_ref;
    p_ref = DMAX(p_ref, small_pres);
    double csq_ref = gam_g_ref * p_ref * rho_ref_inv;
    double cc_ref = sqrt(csq_ref);
    double cc_ref_inv = 1.0 / cc_ref;
    double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv;
    double dum = un_ref - I[0][1];
    double dptotm = p_ref - I[0][2];
    double drho = rho_ref - I[1][0];
    double dptot = p_ref - I[1][2];
    double drhoe_g = rhoe_g_ref - I[1][3];
    double dup = un_ref - I[2][1];
    double dptotp = p_ref - I[2][2];
    double alpham = 0.5 * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
    double alphap = 0.5 * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
    double alpha0r = drho - dptot / csq_ref;
    double alpha0e_g = drhoe_g - dptot * h_g_ref / csq_ref;
    if (plus) {
        alpham = (un - cc > 0.0) ? 0.0 : -alpham;
        alphap = (un + cc > 0.0) ? 0.0 : -alphap;
        alpha0r = (un > 0.0) ? 0.0 : -alpha0r;
        alpha0e_g = (un > 0.0) ? 0.0 : -alpha0e_g;
    } else {
        alpham = (un - cc > 0.0) ? -alpham : 0.0;
        alphap = (un + cc > 0.0) ? -alphap : 0.0;
        alpha0r = (un > 0.0) ? -alpha0r : 0.0;
        alpha0e_g = (un > 0.0) ? -alpha0e_g : 0.0;
    }
    rho_o = DMAX(small_dens, rho_ref + alphap + alpham + alpha0r);
    un_o = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
    rhoe_o = rhoe_g_ref + (alphap + alpham) * h_g_ref + alpha0e_g;
    p_o = DMAX(small_pres, p_ref + (alphap + alpham) * csq_ref);
}

// trace_ppm for one zone and one direction D (Source/ppm.F90:437-737): the
// plus state on face i (left face of the zone) and the minus state on face
// i+1, in compact face-state layout.  flatn is uflatten of the zone.
template <int NS, int D, class L>
CASTRO_HD void trace_zone(const L& ld, int i, int j, int k, double dtdx, double flatn,
                                           double* qplus, double* qminus)
{
    constexpr int ex = D == 0, ey = D == 1, ez = D == 2;
    constexpr int qun = QU + D;
    constexpr int qut = QU + (D == 0 ? 1 : D == 1 ? 2 : 0);
    constexpr int qutt = QU + (D == 0 ? 2 : D == 1 ? 0 : 1);
    double cc = ld.c(i, j, k);
    double un = ld.q(i, j, k, qun);
    // rho, un, p, rhoe feed the characteristic projection
    double Ip[3][4], Im[3][4];
    constexpr int vars[4] = {QRHO, qun, QPRES, QREINT};
    double s[5], sm, sp;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
#pragma unroll
        for (int m = -2; m <= 2; ++m) s[m + 2] = ld.q(i + m * ex, j + m * ey, k + m * ez, vars[v]);
        ppm_reconstruct(s, flatn, sm, sp);
        double s6 = 6.0 * s[2] - 3.0 * (sm + sp);
        ppm_int_wave(sm, sp, s6, un - cc, dtdx, Ip[0][v], Im[0][v]);
        ppm_int_wave(sm, sp, s6, un, dtdx, Ip[1][v], Im[1][v]);
        ppm_int_wave(sm, sp, s6, un + cc, dtdx, Ip[2][v], Im[2][v]);
    }
    // transverse velocities: only the u wave
    double Ipt, Imt, Iptt, Imtt;
    {
#pragma unroll
        for (int m = -2; m <= 2; ++m) s[m + 2] = ld.q(i + m * ex, j + m * ey, k + m * ez, qut);
        ppm_reconstruct(s, flatn, sm, sp);
        double s6 = 6.0 * s[2] - 3.0 * (sm + sp);
        ppm_int_wave(sm, sp, s6, un, dtdx, Ipt, Imt);
#pragma unroll
        for (int m = -2; m <= 2; ++m) s[m + 2] = ld.q(i + m * ex, j + m * ey, k + m * ez, qutt);
        ppm_reconstruct(s, flatn, sm, sp);
        s6 = 6.0 * s[2] - 3.0 * (sm + sp);
        ppm_int_wave(sm, sp, s6, un, dtdx, Iptt, Imtt);
    }
    // gamma_c: waves u-c (plus state) and u+c (minus state)
    double gp0, gm0, gp2, gm2;
    {
#pragma unroll
        for (int m = -2; m <= 2; ++m) s[m + 2] = ld.gamc(i + m * ex, j + m * ey, k + m * ez);
        ppm_reconstruct(s, flatn, sm, sp);
        double s6 = 6.0 * s[2] - 3.0 * (sm + sp);
        ppm_int_wave(sm, sp, s6, un - cc, dtdx, gp0, gm0);
        ppm_int_wave(sm, sp, s6, un + cc, dtdx, gp2, gm2);
    }
#pragma unroll
    for (int n = 0; n < NS; ++n) {
#pragma unroll
        for (int m = -2; m <= 2; ++m) s[m + 2] = ld.q(i + m * ex, j + m * ey, k + m * ez, QFS + n);
        ppm_reconstruct(s, flatn, sm, sp);
        double s6 = 6.0 * s[2] - 3.0 * (sm + sp);
        double ipx, imx;
        ppm_int_wave(sm, sp, s6, un, dtdx, ipx, imx);
        qplus[SX + n] = imx;
        qminus[SX + n] = ipx;
    }
    {
        double r, u, re, p;
        trace_project(Im, gm0, un, cc, true, r, u, re, p);
        qplus[SRHO] = r;
        qplus[SU + D] = u;
        qplus[SREI] = re;
        qplus[SPRES] = p;
        qplus[qut - QU + SU] = Imt;
        qplus[qutt - QU + SU] = Imtt;
    }
    {
        double r, u, re, p;
        trace_project(Ip, gp2, un, cc, false, r, u, re, p);
        qminus[SRHO] = r;
        qminus[SU + D] = u;
        qminus[SREI] = re;
        qminus[SPRES] = p;
        qminus[qut - QU + SU] = Ipt;
        qminus[qutt - QU + SU] = Iptt;
    }
}

// ---------------------------------------------------------------------------
// CGF Riemann solver on one face, Source/riemann.F90:114-325
// ---------------------------------------------------------------------------
// D is the direction normal to the face.  ql/qr: compact face states;
// gamcl/cl of the left zone, gamcr/cr of the right zone.  Outputs: flx (NVAR, conserved order), qg (NGDNV) and, when
// qint is non-null, the interface state in full QVAR numbering (QRHO, velocities,
// QPRES, QGAME, QREINT, species).
template <int NS, int D>
CASTRO_HD void riemann_cgf(const double* ql, const double* qr, double gamcl, double gamcr,
                                            double cl, double cr, double* flx, double* qg, double* qint)
{
    constexpr int iu = SU + D;
    constexpr int iv1 = SU + (D == 0 ? 1 : 0);
    constexpr int iv2 = SU + (D == 2 ? 1 : 2);
    constexpr int im1 = UMX + D;
    constexpr int im2 = UMX + (D == 0 ? 1 : 0);
    constexpr int im3 = UMX + (D == 2 ? 1 : 2);

    double rl = DMAX(ql[SRHO], small_dens);
    double ul = ql[iu], v1l = ql[iv1], v2l = ql[iv2];
    double pl = DMAX(ql[SPRES], small_pres);
    double rel = ql[SREI];
    double rr = DMAX(qr[SRHO], small_dens);
    double ur = qr[iu], v1r = qr[iv1], v2r = qr[iv2];
    double pr = DMAX(qr[SPRES], small_pres);
    double rer = qr[SREI];

    double csmall = DMAX(small, small * DMAX(cr, cl));
    double cavg = 0.5 * (cr + cl);
    double wsmall = small_dens * csmall;
    double wl = DMAX(wsmall, sqrt(fabs(gamcl * pl * rl)));
    double wr = DMAX(wsmall, sqrt(fabs(gamcr * pr * rr)));
    double wwinv = 1.0 / (wl + wr);
    double pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) * wwinv;
    double ustar = ((wl * ul + wr * ur) + (pl - pr)) * wwinv;
    pstar = DMAX(pstar, small_pres);
    if (fabs(ustar) < smallu * 0.5 * (fabs(ul) + fabs(ur))) ustar = 0.0;

    double sgnm = copysign(1.0, ustar);
    if (ustar == 0.0) sgnm = 0.0;
    double fp = 0.5 * (1.0 + sgnm);
    double fm = 0.5 * (1.0 - sgnm);
    double ro = fp * rl + fm * rr;
    double uo = fp * ul + fm * ur;
    double po = fp * pl + fm * pr;
    double reo = fp * rel + fm * rer;
    double gamco = fp * gamcl + fm * gamcr;
    ro = DMAX(small_dens, ro);
    double roinv = 1.0 / ro;
    double co = sqrt(fabs(gamco * po * roinv));
    co = DMAX(csmall, co);
    double co2inv = 1.0 / (co * co);
    double qv1 = fp * v1l + fm * v1r;
    double qv2 = fp * v2l + fm * v2r;

    double drho = (pstar - po) * co2inv;
    double rstar = ro + drho;
    rstar = DMAX(small_dens, rstar);
    double rstarinv = 1.0 / rstar;
    double entho = (reo + po) * roinv * co2inv;
    double estar = reo + (pstar - po) * entho;
    double cstar = sqrt(fabs(gamco * pstar * rstarinv));
    cstar = DMAX(cstar, csmall);

    sgnm = copysign(1.0, ustar);                                       // riemann.F90:225 (no zero guard)
    double spout = co - sgnm * uo;
    double spin = cstar - sgnm * ustar;
    double ushock = 0.5 * (spin + spout);
    if (pstar - po > 0.0) { spin = ushock; spout = ushock; }
    double scr = (spout - spin == 0.0) ? small * cavg : spout - spin;
    double scrinv = 1.0 / scr;
    double frac = (1.0 + (spout + spin) * scrinv) * 0.5;
    frac = DMAX(0.0, DMIN(1.0, frac));

    double qrho = frac * rstar + (1.0 - frac) * ro;
    double qu = frac * ustar + (1.0 - frac) * uo;
    double qp = frac * pstar + (1.0 - frac) * po;
    double regdnv = frac * estar + (1.0 - frac) * reo;
    if (spout < 0.0) { qrho = ro; qu = uo; qp = po; regdnv = reo; }
    if (spin >= 0.0) { qrho = rstar; qu = ustar; qp = pstar; regdnv = estar; }
    double regdnvinv = 1.0 / regdnv;
    double qgame = qp * regdnvinv + 1.0;
    qp = DMAX(qp, small_pres);

    double vel[3];
    vel[D] = qu;
    vel[iv1 - SU] = qv1;
    vel[iv2 - SU] = qv2;
    qg[GDRHO] = qrho;
    qg[GDU] = vel[0];
    qg[GDV] = vel[1];
    qg[GDW] = vel[2];
    qg[GDPRES] = qp;
    qg[GDGAME] = qgame;

    double u_adv = qu;
    double rhoeint = regdnv;
    flx[URHO] = qrho * u_adv;
    flx[im1] = flx[URHO] * qu;
#ifdef __CUDA_ARCH__
    if (c_net.mom_flux_p) flx[im1] = flx[im1] + qp;
#endif
    flx[im2] = flx[URHO] * qv1;
    flx[im3] = flx[URHO] * qv2;
    double rhoetot = rhoeint + 0.5 * qrho * (qu * qu + qv1 * qv1 + qv2 * qv2);
    flx[UEDEN] = u_adv * (rhoetot + qp);
    flx[UEINT] = u_adv * rhoeint;
    flx[UTEMP] = 0.0;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        double x = fp * ql[SX + n] + fm * qr[SX + n];
        flx[UFS + n] = flx[URHO] * x;
        if (qint) qint[QFS + n] = x;
    }
    if (qint) {
        qint[QRHO] = qrho;
        qint[QU] = vel[0];
        qint[QV] = vel[1];
        qint[QW] = vel[2];
        qint[QPRES] = qp;
        qint[QGAME] = qgame;
        qint[QREINT] = regdnv;
    }
}

// ---------------------------------------------------------------------------
// Transverse corrections, Source/trans.F90
// ---------------------------------------------------------------------------
// Flux record used by the corrections: F_URHO, F_UMX, F_UMY, F_UMZ, F_UEDEN,
// F_species (NS), then Godunov GDPRES and the Godunov velocity normal to the
// flux face.  Indices into that record:
template <int NS>
struct TF {
    static constexpr int RHO = 0, MX = 1, MY = 2, MZ = 3, ED = 4, X = 5, PG = 5 + NS, UG = 6 + NS, N = 7 + NS;
};

// trans1 on one face state (trans.F90:151-229): lq is the state normal to
// direction 2, fr/fl the flux records of direction 1 on the right/left faces,
// gamc the left zone's gamma_1.  Returns true when the density reset fired.
template <int NS>
CASTRO_HD bool trans1_state(const double* lq, const double* fr, const double* fl, double gamc,
                                             double cdtdx, double* lqo)
{
    using R = TF<NS>;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        double rrnew = lq[SRHO] - cdtdx * (fr[R::RHO] - fl[R::RHO]);
        double compu = lq[SRHO] * lq[SX + n] - cdtdx * (fr[R::X + n] - fl[R::X + n]);
        lqo[SX + n] = compu / rrnew;
    }
    double pgp = fr[R::PG], pgm = fl[R::PG];
    double ugp = fr[R::UG], ugm = fl[R::UG];
    double dup = pgp * ugp - pgm * ugm;
    double du = ugp - ugm;
    double pav = 0.5 * (pgp + pgm);

    double rrl2 = lq[SRHO];
    double rul2 = rrl2 * lq[SU];
    double rvl2 = rrl2 * lq[SV];
    double rwl2 = rrl2 * lq[SW];
    double ekenl2 = 0.5 * rrl2 * (lq[SU] * lq[SU] + lq[SV] * lq[SV] + lq[SW] * lq[SW]);
    double rel2 = lq[SREI] + ekenl2;
    double rrnewl2 = rrl2 - cdtdx * (fr[R::RHO] - fl[R::RHO]);
    double runewl2 = rul2 - cdtdx * (fr[R::MX] - fl[R::MX]);
    double rvnewl2 = rvl2 - cdtdx * (fr[R::MY] - fl[R::MY]);
    double rwnewl2 = rwl2 - cdtdx * (fr[R::MZ] - fl[R::MZ]);
    double renewl2 = rel2 - cdtdx * (fr[R::ED] - fl[R::ED]);
    bool reset_state = false;
    if (rrnewl2 < 0.0) {
        rrnewl2 = rrl2; runewl2 = rul2; rvnewl2 = rvl2; rwnewl2 = rwl2; renewl2 = rel2;
        reset_state = true;
    }
    lqo[SRHO] = rrnewl2;
    double rhoinv = 1.0 / rrnewl2;
    lqo[SU] = runewl2 * rhoinv;
    lqo[SV] = rvnewl2 * rhoinv;
    lqo[SW] = rwnewl2 * rhoinv;
    double rhoekenl2 = 0.5 * (runewl2 * runewl2 + rvnewl2 * rvnewl2 + rwnewl2 * rwnewl2) * rhoinv;
    lqo[SREI] = renewl2 - rhoekenl2;
    if (!reset_state) {
        double pnewl2 = lq[SPRES] - cdtdx * (dup + pav * du * (gamc - 1.0));
        lqo[SPRES] = DMAX(pnewl2, small_pres);
    } else {
        lqo[SPRES] = lq[SPRES];
    }
    return reset_state;
}

// trans2 on one face state (trans.F90:393-491): f2r/f2l and f3r/f3l are the
// flux records of the two transverse directions, gamc the gamma_1 of the zone
// the state comes from.
template <int NS>
CASTRO_HD bool trans2_state(const double* lq, const double* f2r, const double* f2l,
                                             const double* f3r, const double* f3l, double gamc,
                                             double cdtdx2, double cdtdx3, double* lqo)
{
    using R = TF<NS>;
#pragma unroll
    for (int n = 0; n < NS; ++n) {
        double rrr = lq[SRHO];
        double compr = rrr * lq[SX + n];
        double rrnewr = rrr - cdtdx2 * (f2r[R::RHO] - f2l[R::RHO]) - cdtdx3 * (f3r[R::RHO] - f3l[R::RHO]);
        double compnr = compr - cdtdx2 * (f2r[R::X + n] - f2l[R::X + n]) - cdtdx3 * (f3r[R::X + n] - f3l[R::X + n]);
        lqo[SX + n] = compnr / rrnewr;
    }
    double pg2p = f2r[R::PG], pg2m = f2l[R::PG], ug2p = f2r[R::UG], ug2m = f2l[R::UG];
    double du2p = pg2p * ug2p - pg2m * ug2m;
    double p2av = 0.5 * (pg2p + pg2m);
    double du2 = ug2p - ug2m;
    double p2new = cdtdx2 * (du2p + p2av * du2 * (gamc - 1.0));
    double pg3p = f3r[R::PG], pg3m = f3l[R::PG], ug3p = f3r[R::UG], ug3m = f3l[R::UG];
    double du3p = pg3p * ug3p - pg3m * ug3m;
    double p3av = 0.5 * (pg3p + pg3m);
    double du3 = ug3p - ug3m;
    double p3new = cdtdx3 * (du3p + p3av * du3 * (gamc - 1.0));

    double rrr = lq[SRHO];
    double rur = rrr * lq[SU];
    double rvr = rrr * lq[SV];
    double rwr = rrr * lq[SW];
    double ekenr = 0.5 * rrr * (lq[SU] * lq[SU] + lq[SV] * lq[SV] + lq[SW] * lq[SW]);
    double rer = lq[SREI] + ekenr;
    double rrnewr = rrr - cdtdx2 * (f2r[R::RHO] - f2l[R::RHO]) - cdtdx3 * (f3r[R::RHO] - f3l[R::RHO]);
    double runewr = rur - cdtdx2 * (f2r[R::MX] - f2l[R::MX]) - cdtdx3 * (f3r[R::MX] - f3l[R::MX]);
    double rvnewr = rvr - cdtdx2 * (f2r[R::MY] - f2l[R::MY]) - cdtdx3 * (f3r[R::MY] - f3l[R::MY]);
    double rwnewr = rwr - cdtdx2 * (f2r[R::MZ] - f2l[R::MZ]) - cdtdx3 * (f3r[R::MZ] - f3l[R::MZ]);
    double renewr = rer - cdtdx2 * (f2r[R::ED] - f2l[R::ED]) - cdtdx3 * (f3r[R::ED] - f3l[R::ED]);
    bool reset_state = false;
    if (rrnewr < 0.0) {
        rrnewr = rrr; runewr = rur; rvnewr = rvr; rwnewr = rwr; renewr = rer;
        reset_state = true;
    }
    lqo[SRHO] = rrnewr;
    lqo[SU] = runewr / rrnewr;
    lqo[SV] = rvnewr / rrnewr;
    lqo[SW] = rwnewr / rrnewr;
    double rhoekenr = 0.5 * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
    lqo[SREI] = renewr - rhoekenr;
    lqo[SPRES] = reset_state ? lq[SPRES] : lq[SPRES] - p2new - p3new;
    lqo[SPRES] = DMAX(lqo[SPRES], small_pres);
    return reset_state;
}

// artificial viscosity of one face component (Castro_hydro_nd.F90:214-237):
// divsum is the four-node sum exactly as the reference forms it.
CASTRO_HD double av_term(double divsum, double du)
{
    double div1 = 0.25 * divsum;
    div1 = 0.1 * DMIN(0.0, div1);
    return div1 * du;
}

}  // namespace castro
