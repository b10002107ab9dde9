// adjoint_selftest.cu -- host-side check of the reverse-mode stages of
// castro_adjoint.cuh against central finite differences of their forward
// stages (castro_device.cuh / castro_adjoint.cuh), on seeded random inputs.
//
//   castro_adjoint_selftest <helm_table.dat> [ncase]
//
// For each stage y = f(x): random output weights w and input direction v,
// compare <J^T w, v> from the adjoint with (w.f(x+hv) - w.f(x-hv)) / 2h.
// Prints one line per stage with the worst relative mismatch and exits
// non-zero when a stage exceeds its tolerance.  Runs on the CPU only.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <functional>
#include <random>
#include <vector>

#include "castro_adjoint.cuh"
#include "castro_table.h"

using namespace castro;

namespace {

std::mt19937_64 rng(20240611);
double urand(double a, double b) { return std::uniform_real_distribution<double>(a, b)(rng); }
double nrand() { return std::normal_distribution<double>(0.0, 1.0)(rng); }

NetworkDev net2()
{
    NetworkDev n{};
    n.nspec = 2;
    n.aion[0] = 4.0; n.zion[0] = 2.0;
    n.aion[1] = 16.0; n.zion[1] = 8.0;
    for (int k = 0; k < 2; ++k) n.aion_inv[k] = 1.0 / n.aion[k];
    return n;
}

struct Stat {
    const char* name;
    double worst = 0.0;
    int n = 0, skipped = 0;
    double tol;
    void add(double ad, double fd, double scale)
    {
        double den = fmax(fmax(fabs(ad), fabs(fd)), scale);
        double e = den > 0 ? fabs(ad - fd) / den : 0.0;
        if (e > worst) worst = e;
        ++n;
    }
    bool report() const
    {
        bool ok = worst <= tol;
        printf("%-24s cases %4d  worst rel %.3e  tol %.1e  %s\n", name, n, worst, tol, ok ? "ok" : "FAIL");
        return ok;
    }
};

// directional FD of s(x) = w.f(x) along v with per-component step h*scale_i
double fd1(const std::function<double(const std::vector<double>&)>& s, const std::vector<double>& x,
           const std::vector<double>& v, double h)
{
    std::vector<double> xp(x), xm(x);
    for (size_t i = 0; i < x.size(); ++i) { xp[i] += h * v[i]; xm[i] -= h * v[i]; }
    return (s(xp) - s(xm)) / (2.0 * h);
}

// FD estimate at steps h, 10h and h/10, returned as the one closest to the
// adjoint value 'ad': a branch switch inside the stencil of one step, or
// rounding noise at the smallest step, spoils at most some of the three, while
// a wrong adjoint agrees with none of them
double fd_best(const std::function<double(const std::vector<double>&)>& s, const std::vector<double>& x,
               const std::vector<double>& v, double h, double ad)
{
    double a = fd1(s, x, v, h), b = fd1(s, x, v, 10.0 * h), c = fd1(s, x, v, 0.1 * h);
    double best = a;
    if (fabs(b - ad) < fabs(best - ad)) best = b;
    if (fabs(c - ad) < fabs(best - ad)) best = c;
    return best;
}

double dot(const std::vector<double>& a, const std::vector<double>& b)
{
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

constexpr int NS = 2;
using DM = Dims<NS>;
// Correct adjoints agree with the best of the three FD steps to ~2e-6 relative
// (FD cancellation noise); a wrong branch derivative shows as 1e-2 .. 1.
constexpr double TOL = 1e-5;

// a random compact face state around a Sedov-like flow
void rand_state(double* s, double rho0, double p0)
{
    s[SRHO] = rho0 * urand(0.5, 2.0);
    double c = sqrt(1.5 * p0 / rho0);
    s[SU] = c * urand(-1.5, 1.5);
    s[SV] = c * urand(-1.0, 1.0);
    s[SW] = c * urand(-1.0, 1.0);
    s[SPRES] = p0 * urand(0.3, 3.0);
    s[SREI] = s[SPRES] * urand(1.3, 2.0);
    s[SX] = urand(0.2, 0.8) / s[SRHO];
    s[SX + 1] = urand(0.2, 0.8) / s[SRHO];
}

// ---------------------------------------------------------------- Riemann
template <int D>
void test_riemann(Stat& st, int ncase)
{
    const int NQ = DM::NQS, NV = DM::NVAR;
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x(2 * NQ + 4);
        rand_state(&x[0], 1.0, 1.0e15);
        rand_state(&x[NQ], 1.0, 1.0e15 * (c % 3 == 0 ? 30.0 : 1.0));
        x[2 * NQ + 0] = urand(1.3, 1.67);
        x[2 * NQ + 1] = urand(1.3, 1.67);
        x[2 * NQ + 2] = sqrt(x[2 * NQ + 0] * x[SPRES] / x[SRHO]);
        x[2 * NQ + 3] = sqrt(x[2 * NQ + 1] * x[NQ + SPRES] / x[NQ + SRHO]);
        std::vector<double> w(NV + NGDNV);
        for (auto& a : w) a = nrand();
        w[UTEMP] = 0.0;
        auto f = [&](const std::vector<double>& y) {
            double flx[NV], qg[NGDNV];
            riemann_cgf<NS, D>(&y[0], &y[NQ], y[2 * NQ], y[2 * NQ + 1], y[2 * NQ + 2], y[2 * NQ + 3], flx, qg, nullptr);
            double s = 0.0;
            for (int n = 0; n < NV; ++n) s += w[n] * flx[n];
            for (int n = 0; n < NGDNV; ++n) s += w[NV + n] * qg[n];
            return s;
        };
        std::vector<double> xb(x.size(), 0.0);
        riemann_cgf_adj<NS, D>(&x[0], &x[NQ], x[2 * NQ], x[2 * NQ + 1], x[2 * NQ + 2], x[2 * NQ + 3], &w[0], &w[NV],
                               &xb[0], &xb[NQ], xb[2 * NQ], xb[2 * NQ + 1], xb[2 * NQ + 2], xb[2 * NQ + 3]);
        std::vector<double> v(x.size());
        for (size_t i = 0; i < x.size(); ++i) v[i] = nrand() * fabs(x[i]);
        double ad = dot(xb, v);
        st.add(ad, fd_best(f, x, v, 1e-7, ad), 0.0);
    }
}

// ---------------------------------------------------------------- trans1/trans2
void rand_tflux(double* r, double scale)
{
    using R = TF<NS>;
    for (int n = 0; n < R::N; ++n) r[n] = scale * urand(-1.0, 1.0);
    r[R::PG] = 1.0e15 * urand(0.5, 2.0);
    r[R::UG] = 3.0e7 * urand(-1.0, 1.0);
}

void test_trans1(Stat& st, int ncase)
{
    const int NQ = DM::NQS, NT = DM::NTF;
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x(NQ + 2 * NT + 2);
        rand_state(&x[0], 1.0, 1.0e15);
        rand_tflux(&x[NQ], 3.0e7);
        rand_tflux(&x[NQ + NT], 3.0e7);
        // energy-like fluxes scaled to the state
        x[NQ + TF<NS>::ED] *= 1.0e15; x[NQ + NT + TF<NS>::ED] *= 1.0e15;
        for (int m = 0; m < 3; ++m) { x[NQ + TF<NS>::MX + m] *= 3.0e7; x[NQ + NT + TF<NS>::MX + m] *= 3.0e7; }
        x[NQ + 2 * NT] = urand(1.3, 1.67);
        x[NQ + 2 * NT + 1] = urand(0.001, 0.01) * 1.0e-7;
        std::vector<double> w(NQ);
        for (auto& a : w) a = nrand();
        auto f = [&](const std::vector<double>& y) {
            double o[NQ];
            trans1_state<NS>(&y[0], &y[NQ], &y[NQ + NT], y[NQ + 2 * NT], y[NQ + 2 * NT + 1], o);
            double s = 0.0;
            for (int n = 0; n < NQ; ++n) s += w[n] * o[n];
            return s;
        };
        std::vector<double> xb(x.size(), 0.0);
        trans1_state_adj<NS>(&x[0], &x[NQ], &x[NQ + NT], x[NQ + 2 * NT], x[NQ + 2 * NT + 1], &w[0], &xb[0], &xb[NQ],
                             &xb[NQ + NT], xb[NQ + 2 * NT], xb[NQ + 2 * NT + 1]);
        std::vector<double> v(x.size());
        for (size_t i = 0; i < x.size(); ++i) v[i] = nrand() * fabs(x[i]);
        { double ad = dot(xb, v); st.add(ad, fd_best(f, x, v, 1e-7, ad), 0.0); }
    }
}

void test_trans2(Stat& st, int ncase)
{
    const int NQ = DM::NQS, NT = DM::NTF;
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x(NQ + 4 * NT + 3);
        rand_state(&x[0], 1.0, 1.0e15);
        for (int f = 0; f < 4; ++f) {
            rand_tflux(&x[NQ + f * NT], 3.0e7);
            x[NQ + f * NT + TF<NS>::ED] *= 1.0e15;
            for (int m = 0; m < 3; ++m) x[NQ + f * NT + TF<NS>::MX + m] *= 3.0e7;
        }
        const int o = NQ + 4 * NT;
        x[o] = urand(1.3, 1.67);
        x[o + 1] = urand(0.001, 0.01) * 1.0e-7;
        x[o + 2] = urand(0.001, 0.01) * 1.0e-7;
        std::vector<double> w(NQ);
        for (auto& a : w) a = nrand();
        auto f = [&](const std::vector<double>& y) {
            double out[NQ];
            trans2_state<NS>(&y[0], &y[NQ], &y[NQ + NT], &y[NQ + 2 * NT], &y[NQ + 3 * NT], y[o], y[o + 1], y[o + 2], out);
            double s = 0.0;
            for (int n = 0; n < NQ; ++n) s += w[n] * out[n];
            return s;
        };
        std::vector<double> xb(x.size(), 0.0);
        trans2_state_adj<NS>(&x[0], &x[NQ], &x[NQ + NT], &x[NQ + 2 * NT], &x[NQ + 3 * NT], x[o], x[o + 1], x[o + 2],
                             &w[0], &xb[0], &xb[NQ], &xb[NQ + NT], &xb[NQ + 2 * NT], &xb[NQ + 3 * NT], xb[o],
                             xb[o + 1], xb[o + 2]);
        std::vector<double> v(x.size());
        for (size_t i = 0; i < x.size(); ++i) v[i] = nrand() * fabs(x[i]);
        { double ad = dot(xb, v); st.add(ad, fd_best(f, x, v, 1e-7, ad), 0.0); }
    }
}

// ---------------------------------------------------------------- trace + flatten
constexpr int G = 9;   // 9^3 zones, centre at (4,4,4)
struct HostLoader {
    const double* qd;   // QVAR comps
    const double* qa;   // NQAUX comps
    CASTRO_HD double q(int i, int j, int k, int n) const { return qd[((n * G + k) * G + j) * G + i]; }
    CASTRO_HD double gamc(int i, int j, int k) const { return qa[((QGAMC * G + k) * G + j) * G + i]; }
    CASTRO_HD double c(int i, int j, int k) const { return qa[((QC * G + k) * G + j) * G + i]; }
};
struct HostSink {
    double* qb;
    double* qab;
    CASTRO_HD void q(int i, int j, int k, int n, double v) const { qb[((n * G + k) * G + j) * G + i] += v; }
    CASTRO_HD void gamc(int i, int j, int k, double v) const { qab[((QGAMC * G + k) * G + j) * G + i] += v; }
    CASTRO_HD void c(int i, int j, int k, double v) const { qab[((QC * G + k) * G + j) * G + i] += v; }
};

template <int D>
void test_trace(Stat& st, int ncase, bool with_flatten)
{
    const int QV = DM::QVAR, NQ = DM::NQS;
    const int nq = QV * G * G * G, na = NQAUX * G * G * G;
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x(nq + na);
        // smooth-ish random fields with a pressure jump so flattening is active in some cases
        double jump = (c % 2) ? 8.0 : 1.3;
        for (int k = 0; k < G; ++k)
            for (int j = 0; j < G; ++j)
                for (int i = 0; i < G; ++i) {
                    int id = (k * G + j) * G + i;
                    int ic = D == 0 ? i : D == 1 ? j : k;
                    double rho = urand(0.8, 1.2);
                    double p = 1.0e15 * urand(0.8, 1.2) * (ic >= 5 ? jump : 1.0);
                    x[QRHO * G * G * G + id] = rho;
                    x[QU * G * G * G + id] = 3.0e7 * urand(-1, 1) - (ic >= 5 ? 2.0e7 : 0.0);
                    x[QV * G * G * G + id] = 3.0e7 * urand(-1, 1);
                    x[QW * G * G * G + id] = 3.0e7 * urand(-1, 1);
                    x[QGAME * G * G * G + id] = 1.6;
                    x[QPRES * G * G * G + id] = p;
                    x[QREINT * G * G * G + id] = p * urand(1.4, 1.6);
                    x[QTEMP * G * G * G + id] = 1.0e6;
                    x[QFS * G * G * G + id] = urand(0.3, 0.7) / rho;
                    x[(QFS + 1) * G * G * G + id] = urand(0.3, 0.7) / rho;
                    double g = urand(1.4, 1.67);
                    x[nq + QGAMC * G * G * G + id] = g;
                    x[nq + QC * G * G * G + id] = sqrt(g * p / rho);
                    x[nq + QDPDR * G * G * G + id] = 0.0;
                    x[nq + QDPDE * G * G * G + id] = 0.0;
                }
        const double dtdx = urand(0.5, 1.0) * 1.0e-7 / 1.0;
        std::vector<double> wp(NQ), wm(NQ);
        for (auto& a : wp) a = nrand();
        for (auto& a : wm) a = nrand();
        const int ci = 4, cj = 4, ck = 4;
        auto f = [&](const std::vector<double>& y) {
            HostLoader ld{&y[0], &y[nq]};
            double flatn = with_flatten ? uflatten(ld, ci, cj, ck) : 0.7;
            double qp[NQ], qm[NQ];
            trace_zone<NS, D>(ld, ci, cj, ck, y.back(), flatn, qp, qm);
            double s = 0.0;
            for (int n = 0; n < NQ; ++n) s += wp[n] * qp[n] + wm[n] * qm[n];
            return s;
        };
        x.push_back(dtdx);
        std::vector<double> xb(x.size(), 0.0);
        HostLoader ld{&x[0], &x[nq]};
        HostSink sk{&xb[0], &xb[nq]};
        double flatn = with_flatten ? uflatten(ld, ci, cj, ck) : 0.7;
        double dtdxb = 0.0;
        double flatnb = trace_zone_adj<NS, D>(ld, sk, ci, cj, ck, dtdx, flatn, &wp[0], &wm[0], dtdxb);
        if (with_flatten) uflatten_adj(ld, sk, ci, cj, ck, flatnb);
        xb.back() = dtdxb;
        std::vector<double> v(x.size());
        for (size_t i = 0; i < x.size(); ++i) v[i] = nrand() * fabs(x[i]);
        { double ad = dot(xb, v); st.add(ad, fd_best(f, x, v, 1e-7, ad), 0.0); }
    }
}

// ---------------------------------------------------------------- EOS-based stages
void rand_cons(double* u, const NetworkDev& net)
{
    (void)net;
    double rho = urand(0.5, 2.0);
    double T = pow(10.0, urand(5.5, 9.0));
    (void)T;
    u[URHO] = rho;
    double vel = 1.0e7 * urand(-1, 1);
    u[UMX] = rho * vel;
    u[UMY] = rho * 1.0e7 * urand(-1, 1);
    u[UMZ] = rho * 1.0e7 * urand(-1, 1);
    double e = pow(10.0, urand(13.0, 17.0));
    u[UEINT] = rho * e;
    u[UEDEN] = u[UEINT] + 0.5 * (u[UMX] * u[UMX] + u[UMY] * u[UMY] + u[UMZ] * u[UMZ]) / rho * urand(1.0, 1.001);
    u[UTEMP] = 1.0e6;
    u[UFS] = urand(0.3, 0.7);
    u[UFS + 1] = urand(0.3, 0.7);
}

void test_ctoprim(Stat& st, const EosTableDev& tb, const NetworkDev& net, int ncase)
{
    const int NV = DM::NVAR, QV = DM::QVAR;
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x(NV);
        rand_cons(&x[0], net);
        // a realistic T guess
        {
            double q[QV], qa[NQAUX];
            ctoprim_pt_t<NS>(tb, net, &x[0], q, qa);
            x[UTEMP] = q[QTEMP];
        }
        std::vector<double> w(QV + NQAUX);
        for (auto& a : w) a = nrand();
        auto f = [&](const std::vector<double>& y) {
            double q[QV], qa[NQAUX];
            ctoprim_pt_t<NS>(tb, net, &y[0], q, qa);
            double s = 0.0;
            for (int n = 0; n < QV; ++n) s += w[n] * q[n];
            for (int n = 0; n < NQAUX; ++n) s += w[QV + n] * qa[n];
            return s;
        };
        std::vector<double> xb(NV, 0.0);
        ctoprim_pt_adj<NS>(tb, net, &x[0], &w[0], &w[QV], &xb[0]);
        std::vector<double> v(NV);
        for (int i = 0; i < NV; ++i) v[i] = nrand() * fabs(x[i]);
        v[UTEMP] = 0.0;   // the initial guess
        { double ad = dot(xb, v); st.add(ad, fd_best(f, x, v, 1e-5, ad), 0.0); }
    }
}

void test_clean(Stat& st, const EosTableDev& tb, const NetworkDev& net, int ncase, int which)
{
    const int NV = DM::NVAR;
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x(NV);
        rand_cons(&x[0], net);
        if (which == 1) {   // E < 0 branch with a positive internal energy
            x[UEDEN] = -fabs(x[UEDEN]) * 0.1;
        } else if (which == 2) {   // dual-energy branch not taken: e from the state
            x[UEDEN] = x[UEINT] * 1.00001 + 0.5 * (x[UMX] * x[UMX] + x[UMY] * x[UMY] + x[UMZ] * x[UMZ]) / x[URHO];
            x[UMX] *= 1e-3;
        } else if (which == 3) {   // clamped species
            x[UFS] = 2.5 * x[URHO];
        }
        std::vector<double> w(NV);
        for (auto& a : w) a = nrand();
        w[UTEMP] = 0.0;
        auto f = [&](const std::vector<double>& y) {
            double u[NV];
            for (int n = 0; n < NV; ++n) u[n] = y[n];
            clean_state_pt_t<NS>(tb, net, u);
            double s = 0.0;
            for (int n = 0; n < NV; ++n) s += w[n] * u[n];
            return s;
        };
        std::vector<double> xb(w);
        clean_state_pt_adj<NS>(tb, net, &x[0], &xb[0]);
        std::vector<double> v(NV);
        for (int i = 0; i < NV; ++i) v[i] = nrand() * fabs(x[i]);
        v[UTEMP] = 0.0;
        // E - rho*ke cancels strongly in some cases: a wider step keeps FD rounding below 1e-7
        double a = dot(xb, v), b = fd_best(f, x, v, 1e-5, a);
        if (getenv("SELFTEST_VERBOSE") && fabs(a - b) > 1e-6 * fabs(b))
            printf("  clean %d case %d: ad %.6e fd %.6e fd(1e-7) %.6e\n", which, c, a, b, fd1(f, x, v, 1e-7));
        st.add(a, b, 0.0);
    }
}

void test_estdt(Stat& st, const EosTableDev& tb, const NetworkDev& net, int ncase)
{
    const int NV = DM::NVAR;
    const double dx[3] = {1.0 / 64, 1.0 / 64, 1.0 / 64};
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x(NV);
        rand_cons(&x[0], net);
        auto f = [&](const std::vector<double>& y) { return estdt_pt_t<NS>(tb, net, &y[0], dx); };
        std::vector<double> xb(NV, 0.0);
        estdt_pt_adj<NS>(tb, net, &x[0], dx, 1.0, &xb[0]);
        std::vector<double> v(NV);
        for (int i = 0; i < NV; ++i) v[i] = nrand() * fabs(x[i]);
        v[UTEMP] = 0.0;
        double a = dot(xb, v), b = fd_best(f, x, v, 1e-5, a);
        if (getenv("SELFTEST_VERBOSE") && fabs(a - b) > 1e-6 * fabs(b))
            printf("  estdt case %d: ad %.6e fd %.6e fd(1e-7) %.6e  rho %.3e ei %.3e\n", c, a, b, fd1(f, x, v, 1e-7), x[URHO], x[UEINT]);
        st.add(a, b, 0.0);
    }
}

void test_eos_rt(Stat& st, const EosTableDev& tb, int ncase)
{
    for (int c = 0; c < ncase; ++c) {
        std::vector<double> x = {pow(10.0, urand(-3.0, 6.0)), pow(10.0, urand(4.0, 9.5)), urand(4.0, 16.0), 0.0};
        x[3] = x[2] * urand(0.4, 0.5);
        EosBar ob{0.0, nrand(), nrand(), nrand(), nrand(), nrand(), nrand()};
        auto f = [&](const std::vector<double>& y) {
            EosOutT<double> r;
            eos_solve_t<EOS_RT>(tb, y[0], y[1], 0.0, y[2], y[3], r);
            double cs = sqrt(r.gam1 * r.p / y[0]);
            return ob.p * r.p + ob.e * r.e + ob.gam1 * r.gam1 + ob.cs * cs + ob.dpde * (r.dpdT / r.dedT) +
                   ob.dpdr_e * (r.dpdr - r.dpdT * r.dedr / r.dedT);
        };
        std::vector<double> xb(4, 0.0);
        eos_vjp<EOS_RT>(tb, x[0], x[1], x[2], x[3], ob, xb[0], xb[1], xb[2], xb[3]);
        std::vector<double> v(4);
        for (int i = 0; i < 4; ++i) v[i] = nrand() * fabs(x[i]);
        { double ad = dot(xb, v); st.add(ad, fd_best(f, x, v, 1e-5, ad), 0.0); }
    }
}

void test_eos_re(Stat& st, const EosTableDev& tb, int ncase)
{
    for (int c = 0; c < ncase; ++c) {
        double rho = pow(10.0, urand(-3.0, 6.0)), T = pow(10.0, urand(4.0, 9.5)), abar = urand(4.0, 16.0);
        double zbar = abar * urand(0.4, 0.5);
        EosOutT<double> r0;
        eos_solve_t<EOS_RT>(tb, rho, T, 0.0, abar, zbar, r0);
        std::vector<double> x = {rho, r0.e, abar, zbar};
        EosBar ob{nrand(), nrand(), 0.0, nrand(), nrand(), nrand(), nrand()};
        auto f = [&](const std::vector<double>& y) {
            EosOutT<double> r;
            double Tc = eos_solve_t<EOS_RE>(tb, y[0], T, y[1], y[2], y[3], r);
            double cs = sqrt(r.gam1 * r.p / y[0]);
            return ob.T * Tc + ob.p * r.p + ob.gam1 * r.gam1 + ob.cs * cs + ob.dpde * (r.dpdT / r.dedT) +
                   ob.dpdr_e * (r.dpdr - r.dpdT * r.dedr / r.dedT);
        };
        EosOutT<double> r;
        double Tc = eos_solve_t<EOS_RE>(tb, x[0], T, x[1], x[2], x[3], r);
        std::vector<double> xb(4, 0.0);
        eos_vjp<EOS_RE>(tb, x[0], Tc, x[2], x[3], ob, xb[0], xb[1], xb[2], xb[3]);
        std::vector<double> v(4);
        for (int i = 0; i < 4; ++i) v[i] = nrand() * fabs(x[i]);
        { double ad = dot(xb, v); st.add(ad, fd_best(f, x, v, 1e-5, ad), 0.0); }
    }
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s helm_table.dat [ncase]\n", argv[0]);
        return 2;
    }
    const int ncase = argc > 2 ? atoi(argv[2]) : 200;
    HostTable T;
    if (read_helm_table(argv[1], T) != 0) {
        fprintf(stderr, "cannot read %s\n", argv[1]);
        return 2;
    }
    EosTableDev tb = T.consts;
    tb.node = T.node.data();
    tb.trow = T.trow.data();
    tb.drow = T.drow.data();
    NetworkDev net = net2();

    bool ok = true;
    {
        Stat s{"riemann_cgf x", 0, 0, 0, TOL}; test_riemann<0>(s, ncase); ok &= s.report();
        Stat s1{"riemann_cgf y", 0, 0, 0, TOL}; test_riemann<1>(s1, ncase); ok &= s1.report();
        Stat s2{"riemann_cgf z", 0, 0, 0, TOL}; test_riemann<2>(s2, ncase); ok &= s2.report();
    }
    { Stat s{"trans1_state", 0, 0, 0, TOL}; test_trans1(s, ncase); ok &= s.report(); }
    { Stat s{"trans2_state", 0, 0, 0, TOL}; test_trans2(s, ncase); ok &= s.report(); }
    {
        Stat s{"trace_zone x", 0, 0, 0, TOL}; test_trace<0>(s, ncase / 4 + 1, false); ok &= s.report();
        Stat s1{"trace_zone y", 0, 0, 0, TOL}; test_trace<1>(s1, ncase / 4 + 1, false); ok &= s1.report();
        Stat s2{"trace_zone z", 0, 0, 0, TOL}; test_trace<2>(s2, ncase / 4 + 1, false); ok &= s2.report();
        Stat s3{"trace+uflatten x", 0, 0, 0, TOL}; test_trace<0>(s3, ncase / 4 + 1, true); ok &= s3.report();
        Stat s4{"trace+uflatten z", 0, 0, 0, TOL}; test_trace<2>(s4, ncase / 4 + 1, true); ok &= s4.report();
    }
    { Stat s{"eos_vjp rt", 0, 0, 0, TOL}; test_eos_rt(s, tb, ncase); ok &= s.report(); }
    { Stat s{"eos_vjp re", 0, 0, 0, TOL}; test_eos_re(s, tb, ncase); ok &= s.report(); }
    { Stat s{"ctoprim", 0, 0, 0, TOL}; test_ctoprim(s, tb, net, ncase); ok &= s.report(); }
    {
        Stat s{"clean_state", 0, 0, 0, TOL}; test_clean(s, tb, net, ncase, 0); ok &= s.report();
        Stat s1{"clean_state E<0", 0, 0, 0, TOL}; test_clean(s1, tb, net, ncase / 4 + 1, 1); ok &= s1.report();
        Stat s2{"clean_state keep ei", 0, 0, 0, TOL}; test_clean(s2, tb, net, ncase / 4 + 1, 2); ok &= s2.report();
        Stat s3{"clean_state X clamp", 0, 0, 0, TOL}; test_clean(s3, tb, net, ncase / 4 + 1, 3); ok &= s3.report();
    }
    { Stat s{"estdt", 0, 0, 0, TOL}; test_estdt(s, tb, net, ncase); ok &= s.report(); }
    printf("%s\n", ok ? "ALL OK" : "FAILURES");
    return ok ? 0 : 1;
}
