/*
 * castro_oracle.c -- CPU oracle for mini-Castro's CTU hydro advance.
 *
 * TEST INFRASTRUCTURE ONLY (see castro_oracle.h).  This is a plain-C
 * restatement of the reference's Fortran, following it statement by statement
 * so that floating-point operation order matches a non-contracting build
 * (gfortran on x86-64: no FMA, left-to-right evaluation, integer powers as
 * repeated multiplies).  Build with -ffp-contract=off.
 *
 * PARITY UNPINNED: no Fortran compiler exists in this image and the reference
 * ships no golden vectors; see castro_oracle.h.
 *
 * Reference files are cited as Source/<file>:<line>.
 */
#include "castro_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* the interface pressure in the normal momentum flux: off, as in the reference
 * (see oracle_set_momentum_flux_pressure) */
static int g_mom_flux_p = 0;
/* Coulomb corrections in the EOS: off, as in the reference (see
 * oracle_set_coulomb_corrections) */
static int g_coulomb = 0;

/* ------------------------------------------------------------------------ */
/* Index maps, Source/Castro_nd.F90:14-57 (0-based)                          */
/* ------------------------------------------------------------------------ */
enum { URHO = 0, UMX = 1, UMY = 2, UMZ = 3, UEDEN = 4, UEINT = 5, UTEMP = 6, UFS = 7 };
enum { QRHO = 0, QU = 1, QV = 2, QW = 3, QGAME = 4, QPRES = 5, QREINT = 6, QTEMP = 7, QFS = 8 };
#define QTHERM 8
enum { QGAMC = 0, QC = 1, QDPDR = 2, QDPDE = 3 };
#define NQAUX 4
enum { GDRHO = 0, GDU = 1, GDV = 2, GDW = 3, GDPRES = 4, GDGAME = 5 };
#define NGDNV 6

/* Source/Castro_nd.F90:59-65 */
static const double small_dens = 1.0e-12;
static const double small_temp = 1.0e3;
static const double small_pres = 1.e-200;
static const double smallu = 1.e-12;
static const double small = 1.e-8;
static const double dual_energy_eta1 = 1.e0;
static const double cfl = 0.5;

/* amrex_constants_module values used by the reference */
#define ZERO 0.0
#define HALF 0.5
#define ONE 1.0
#define TWO 2.0
#define THREE 3.0
#define SIX 6.0
#define FOURTH 0.25
static double SIXTH, TWO3RD, FOUR3RD;

/* ------------------------------------------------------------------------ */
/* Network, Source/network.F90:7-19 (nspec is a run-time choice here)        */
/* ------------------------------------------------------------------------ */
static int nspec = 13;
static double aion[ORACLE_MAX_SPEC] = {4., 12., 16., 20., 24., 28., 32., 36., 40., 44., 48., 52., 56.};
static double zion[ORACLE_MAX_SPEC] = {2., 6., 8., 10., 12., 14., 16., 18., 20., 22., 24., 26., 28.};
static double aion_inv[ORACLE_MAX_SPEC];
static int NVAR = 20, QVAR = 21;

static void init_constants(void)
{
    SIXTH = 1.0 / 6.0;
    TWO3RD = 2.0 / 3.0;
    FOUR3RD = 4.0 / 3.0;
    for (int n = 0; n < nspec; ++n) aion_inv[n] = 1.0 / aion[n];
    NVAR = 7 + nspec;
    QVAR = 8 + nspec;
}

int oracle_network_init(int ns, const double* a, const double* z)
{
    if (ns < 1 || ns > ORACLE_MAX_SPEC) return -1;
    nspec = ns;
    for (int n = 0; n < ns; ++n) { aion[n] = a[n]; zion[n] = z[n]; }
    init_constants();
    return 0;
}

int oracle_nspec(void) { return nspec; }

/* Fortran MAX/MIN of two reals */
static inline double fmx(double a, double b) { return (a > b) ? a : b; }
static inline double fmn(double a, double b) { return (a < b) ? a : b; }

/* ------------------------------------------------------------------------ */
/* FAB accessor (BL_FORT_FAB_ARG_3D, Fortran order)                          */
/* ------------------------------------------------------------------------ */
typedef struct { double* p; int lo[3]; long nx, ny, nz; } fab_t;

static inline fab_t mkfab(const double* p, const int* lo, const int* hi)
{
    fab_t f;
    f.p = (double*)p;
    f.lo[0] = lo[0]; f.lo[1] = lo[1]; f.lo[2] = lo[2];
    f.nx = hi[0] - lo[0] + 1; f.ny = hi[1] - lo[1] + 1; f.nz = hi[2] - lo[2] + 1;
    return f;
}
#define AT(f, i, j, k, n) ((f).p[((long)(i) - (f).lo[0]) + (f).nx * (((long)(j) - (f).lo[1]) + \
                            (f).ny * (((long)(k) - (f).lo[2]) + (f).nz * (long)(n)))])

/* ------------------------------------------------------------------------ */
/* Helmholtz EOS, Source/eos.F90                                             */
/* ------------------------------------------------------------------------ */
#define IMAX 541
#define JMAX 201
static const double tlo = 3.0, thi = 13.0, dlo = -12.0, dhi = 15.0;   /* eos.F90:62-63 */
static double tstp, tstpi, dstp, dstpi, mintemp;
static const double ttol = 1.e-8;                                      /* eos.F90:74 */
#define MAX_NEWTON 100                                                 /* eos.F90:126 */

/* eos.F90:129-137 */
static const double h_planck = 6.6260689633e-27;
static const double avo_eos = 6.0221417930e23;
static const double clight = 2.99792458e10;
static const double kerg = 1.380650424e-16;
static const double amu = 1.66053878283e-24;
static double asol, sioncon, kergavo, asoli3;

static double tab_d[IMAX], tab_t[JMAX];
static double tab_dt[JMAX], tab_dt2[JMAX], tab_dti[JMAX], tab_dt2i[JMAX];
static double tab_dd[IMAX], tab_dd2[IMAX], tab_ddi[IMAX], tab_dd2i[IMAX];
/* the 21 tables, (i,j) at [i + IMAX*j], i density index, j temperature index */
static double* tf; static double* tfd; static double* tft; static double* tfdd; static double* tftt;
static double* tfdt; static double* tfddt; static double* tfdtt; static double* tfddtt;
static double* tdpdf; static double* tdpdfd; static double* tdpdft; static double* tdpdfdt;
static double* tef; static double* tefd; static double* teft; static double* tefdt;
static double* txf; static double* txfd; static double* txft; static double* txfdt;
static int eos_ready = 0;

#define TB(a, i, j) ((a)[(i) + IMAX * (j)])

/* One list-directed READ of n values: starts a new record, may continue onto
 * following records, discards the rest of the last record consumed. */
static int read_record(FILE* fp, double* v, int n)
{
    char line[4096];
    int got = 0;
    while (got < n) {
        if (!fgets(line, sizeof line, fp)) return -1;
        for (char* c = line; *c; ++c) if (*c == 'D' || *c == 'd') *c = 'E';
        char* s = line;
        while (got < n) {
            char* e;
            double x = strtod(s, &e);
            if (e == s) break;
            v[got++] = x;
            s = e;
            while (*s == ',' || *s == ' ' || *s == '\t') ++s;
        }
    }
    return 0;
}

static void eos_constants(void)
{
    init_constants();
    tstp = (thi - tlo) / (double)(float)(JMAX - 1);   /* eos.F90:65 */
    tstpi = 1.0 / tstp;
    dstp = (dhi - dlo) / (double)(float)(IMAX - 1);   /* eos.F90:68 */
    dstpi = 1.0 / dstp;
    mintemp = pow(10.0, tlo);                          /* eos.F90:71 */
    asol = 4.0 * 5.67051e-5 / clight;
    sioncon = (2.0 * M_PI * amu * kerg) / (h_planck * h_planck);
    kergavo = kerg * avo_eos;
    asoli3 = asol / 3.0;
}

/* eos_init, Source/eos.F90:580-734 */
int oracle_eos_init(const char* path)
{
    eos_constants();
    for (int j = 0; j < JMAX; ++j) tab_t[j] = pow(10.0, tlo + j * tstp);   /* eos.F90:626-628 */
    for (int i = 0; i < IMAX; ++i) tab_d[i] = pow(10.0, dlo + i * dstp);   /* eos.F90:630-632 */

    double** tabs[21] = {&tf, &tfd, &tft, &tfdd, &tftt, &tfdt, &tfddt, &tfdtt, &tfddtt,
                         &tdpdf, &tdpdfd, &tdpdft, &tdpdfdt,
                         &tef, &tefd, &teft, &tefdt,
                         &txf, &txfd, &txft, &txfdt};
    for (int m = 0; m < 21; ++m) {
        free(*tabs[m]);
        *tabs[m] = (double*)calloc((size_t)IMAX * JMAX, sizeof(double));
    }
    FILE* fp = fopen(path ? path : "helm_table.dat", "r");
    if (!fp) return -1;
    double v[9];
    /* eos.F90:644-649 */
    for (int j = 0; j < JMAX; ++j)
        for (int i = 0; i < IMAX; ++i) {
            if (read_record(fp, v, 9)) { fclose(fp); return -2; }
            TB(tf, i, j) = v[0]; TB(tfd, i, j) = v[1]; TB(tft, i, j) = v[2];
            TB(tfdd, i, j) = v[3]; TB(tftt, i, j) = v[4]; TB(tfdt, i, j) = v[5];
            TB(tfddt, i, j) = v[6]; TB(tfdtt, i, j) = v[7]; TB(tfddtt, i, j) = v[8];
        }
    /* eos.F90:652-656 */
    for (int j = 0; j < JMAX; ++j)
        for (int i = 0; i < IMAX; ++i) {
            if (read_record(fp, v, 4)) { fclose(fp); return -3; }
            TB(tdpdf, i, j) = v[0]; TB(tdpdfd, i, j) = v[1]; TB(tdpdft, i, j) = v[2]; TB(tdpdfdt, i, j) = v[3];
        }
    /* eos.F90:659-663 */
    for (int j = 0; j < JMAX; ++j)
        for (int i = 0; i < IMAX; ++i) {
            if (read_record(fp, v, 4)) { fclose(fp); return -4; }
            TB(tef, i, j) = v[0]; TB(tefd, i, j) = v[1]; TB(teft, i, j) = v[2]; TB(tefdt, i, j) = v[3];
        }
    /* eos.F90:666-670 */
    for (int j = 0; j < JMAX; ++j)
        for (int i = 0; i < IMAX; ++i) {
            if (read_record(fp, v, 4)) { fclose(fp); return -5; }
            TB(txf, i, j) = v[0]; TB(txfd, i, j) = v[1]; TB(txft, i, j) = v[2]; TB(txfdt, i, j) = v[3];
        }
    fclose(fp);
    /* eos.F90:700-712 */
    for (int j = 0; j < JMAX - 1; ++j) {
        tab_dt[j] = tab_t[j + 1] - tab_t[j];
        tab_dt2[j] = tab_dt[j] * tab_dt[j];
        tab_dti[j] = 1.0 / tab_dt[j];
        tab_dt2i[j] = 1.0 / tab_dt2[j];
    }
    for (int i = 0; i < IMAX - 1; ++i) {
        tab_dd[i] = tab_d[i + 1] - tab_d[i];
        tab_dd2[i] = tab_dd[i] * tab_dd[i];
        tab_ddi[i] = 1.0 / tab_dd[i];
        tab_dd2i[i] = 1.0 / tab_dd2[i];
    }
    eos_ready = 1;
    return 0;
}

void oracle_eos_finalize(void)
{
    double** tabs[21] = {&tf, &tfd, &tft, &tfdd, &tftt, &tfdt, &tfddt, &tfdtt, &tfddtt,
                         &tdpdf, &tdpdfd, &tdpdft, &tdpdfdt,
                         &tef, &tefd, &teft, &tefdt,
                         &txf, &txfd, &txft, &txfdt};
    for (int m = 0; m < 21; ++m) { free(*tabs[m]); *tabs[m] = NULL; }
    eos_ready = 0;
}

/* quintic Hermite basis, eos.F90:740-911 */
static inline double psi0(double z)   { return z * z * z * (z * (-6.0 * z + 15.0) - 10.0) + 1.0; }
static inline double dpsi0(double z)  { return z * z * (z * (-30.0 * z + 60.0) - 30.0); }
static inline double ddpsi0(double z) { return z * (z * (-120.0 * z + 180.0) - 60.0); }
static inline double psi1(double z)   { return z * (z * z * (z * (-3.0 * z + 8.0) - 6.0) + 1.0); }
static inline double dpsi1(double z)  { return z * z * (z * (-15.0 * z + 32.0) - 18.0) + 1.0; }
static inline double ddpsi1(double z) { return z * (z * (-60.0 * z + 96.0) - 36.0); }
static inline double psi2(double z)   { return 0.5 * z * z * (z * (z * (-z + 3.0) - 3.0) + 1.0); }
static inline double dpsi2(double z)  { return 0.5 * z * (z * (z * (-5.0 * z + 12.0) - 9.0) + 2.0); }
static inline double ddpsi2(double z) { return 0.5 * (z * (z * (-20.0 * z + 36.0) - 18.0) + 2.0); }

/* biquintic Hermite, eos.F90:915-950 */
static inline double h5(const double* fi, double w0t, double w1t, double w2t, double w0mt, double w1mt, double w2mt,
                        double w0d, double w1d, double w2d, double w0md, double w1md, double w2md)
{
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
}

/* cubic Hermite basis, eos.F90:955-1031 */
static inline double xpsi0(double z)  { return z * z * (2.0 * z - 3.0) + 1.0; }
static inline double xdpsi0(double z) { return z * (6.0 * z - 6.0); }
static inline double xpsi1(double z)  { return z * (z * (z - 2.0) + 1.0); }
static inline double xdpsi1(double z) { return z * (3.0 * z - 4.0) + 1.0; }

/* bicubic Hermite, eos.F90:1034-1059 */
static inline double h3(const double* fi, double w0t, double w1t, double w0mt, double w1mt,
                        double w0d, double w1d, double w0md, double w1md)
{
    return fi[0] * w0d * w0t + fi[1] * w0md * w0t
         + fi[2] * w0d * w0mt + fi[3] * w0md * w0mt
         + fi[4] * w0d * w1t + fi[5] * w0md * w1t
         + fi[6] * w0d * w1mt + fi[7] * w0md * w1mt
         + fi[8] * w1d * w0t + fi[9] * w1md * w0t
         + fi[10] * w1d * w0mt + fi[11] * w1md * w0mt
         + fi[12] * w1d * w1t + fi[13] * w1md * w1t
         + fi[14] * w1d * w1mt + fi[15] * w1md * w1mt;
}

/* Fortran INT() of a table coordinate, guarded against overflow */
static inline int ftrunc(double x)
{
    if (!(x < 1.0e6)) x = 1.0e6;        /* also maps NaN high */
    if (x < -1.0e6) x = -1.0e6;
    return (int)x;
}

static inline void fill4(double* fi, const double* a, int iat, int jat)
{
    fi[0] = TB(a, iat, jat);
    fi[1] = TB(a, iat + 1, jat);
    fi[2] = TB(a, iat, jat + 1);
    fi[3] = TB(a, iat + 1, jat + 1);
}

/* Coulomb corrections of an ion plasma in a uniform electron background
 * (absent from the reference's eos.F90; the 2017 runs of the reference had
 * them on): the fits of Yakovlev & Shalybkov (1989, Sov. Sci. Rev. E Astrophys.
 * Space Phys. 7, 311), as the Helmholtz EOS (Timmes & Swesty 2000, ApJS 126,
 * 501) applies them.  With n_i = N_A rho / abar the ion density, a =
 * (3 / (4 pi n_i))^(1/3) the ion-sphere radius and Gamma = zbar^2 q_e^2 / (a k T)
 * the coupling parameter, the excess internal energy per ion in kT is
 *   Gamma >= 1:  u = a1 Gamma + b1 Gamma^(1/4) + c1 Gamma^(-1/4) + d1
 *   Gamma <  1:  u = -3 c2 Gamma^(3/2) + a2 Gamma^b2   (c2 = 1/(2 sqrt 3): Debye-Hueckel)
 * and, the excess pressure of a Coulomb system being a third of its energy
 * density, p = rho e / 3.  The entropy is u - f with f the excess free energy
 * (f' = u / Gamma), the strong branch's integration constant -e1.  Gamma goes
 * as rho^(1/3) / T, which gives the derivatives. */
static const double COUL_QE = 4.80320427e-10;                      /* electron charge, esu */
static const double COUL_A1 = -0.898004, COUL_B1 = 0.96786, COUL_C1 = 0.220703, COUL_D1 = -0.86097,
                    COUL_E1 = 2.5269, COUL_A2 = 0.29561, COUL_B2 = 1.9885, COUL_C2 = 0.288675;

typedef struct { double p, dpdd, dpdt, e, dedd, dedt, s, dsdd, dsdt; } coulomb_t;

static void coulomb(double den, double temp, double ytot1, double zbar, double pion, double dpiondd,
                    double dpiondt, coulomb_t* c)
{
    double xni = avo_eos * ytot1 * den;
    double a_ion = cbrt(3.0 / (4.0 * M_PI * xni));
    double gam = zbar * zbar * COUL_QE * COUL_QE / (a_ion * kerg * temp);
    double gdd = gam / (3.0 * den);                 /* dGamma/drho */
    double gdt = -gam / temp;                       /* dGamma/dT */
    double y = kergavo * ytot1;                     /* k N_A / abar */
    if (gam >= 1.0) {
        double x = sqrt(sqrt(gam));
        double u = COUL_A1 * gam + COUL_B1 * x + COUL_C1 / x + COUL_D1;
        double du = COUL_A1 + 0.25 * (COUL_B1 * x - COUL_C1 / x) / gam;
        c->e = y * temp * u;
        c->dedd = y * temp * du * gdd;
        c->dedt = y * u + y * temp * du * gdt;
        c->p = den * c->e / 3.0;
        c->dpdd = (c->e + den * c->dedd) / 3.0;
        c->dpdt = den * c->dedt / 3.0;
        double sv = 3.0 * COUL_B1 * x - 5.0 * COUL_C1 / x + COUL_D1 * (log(gam) - 1.0) - COUL_E1;
        double dsv = (0.75 * COUL_B1 * x + 1.25 * COUL_C1 / x + COUL_D1) / gam;
        c->s = -y * sv;
        c->dsdd = -y * dsv * gdd;
        c->dsdt = -y * dsv * gdt;
    } else {
        double g32 = gam * sqrt(gam);
        double gb = pow(gam, COUL_B2);
        double z = COUL_C2 * g32 - COUL_A2 * gb / 3.0;
        double dz = 1.5 * COUL_C2 * sqrt(gam) - COUL_A2 * COUL_B2 * gb / (3.0 * gam);
        c->p = -pion * z;
        c->dpdd = -(dpiondd * z + pion * dz * gdd);
        c->dpdt = -(dpiondt * z + pion * dz * gdt);
        c->e = 3.0 * c->p / den;
        c->dedd = 3.0 * c->dpdd / den - 3.0 * c->p / (den * den);
        c->dedt = 3.0 * c->dpdt / den;
        double sv = COUL_C2 * g32 - COUL_A2 * (COUL_B2 - 1.0) / COUL_B2 * gb;
        double dsv = 1.5 * COUL_C2 * sqrt(gam) - COUL_A2 * (COUL_B2 - 1.0) * gb / gam;
        c->s = -y * sv;
        c->dsdd = -y * dsv * gdd;
        c->dsdt = -y * dsv * gdt;
    }
}

/* eos, Source/eos.F90:141-576 */
void oracle_eos(int input, oracle_eos_t* state)
{
    int converged;
    double v_want = 0.0, v, dvdx, error, temp_old;
    double temp, den, din, deni, tempi, ytot1, ye;
    double pres, ener, entr, dpresdd, dpresdt, denerdd, denerdt, dentrdd, dentrdt;
    double pele, dpepdt, dpepdd, eele, deepdt, deepdd, sele, dsepdd, dsepdt;
    double prad, dpraddd, dpraddt, erad, deraddd, deraddt, srad, dsraddd, dsraddt;
    double pion, dpiondd, dpiondt, eion, deiondd, deiondt, sion, dsiondd, dsiondt;
    double s, x, y, z, zz, zzi, chit, chid;
    int iat, jat;
    double free_e, df_d, df_t, df_tt, df_dt;
    double xt, xd, mxt, mxd;
    double fi[36];
    double si0t, si1t, si2t, si0mt, si1mt, si2mt;
    double si0d, si1d, si2d, si0md, si1md, si2md;
    double dsi0t, dsi1t, dsi2t, dsi0mt, dsi1mt, dsi2mt;
    double dsi0d, dsi1d, dsi2d, dsi0md, dsi1md, dsi2md;
    double ddsi0t, ddsi1t, ddsi2t, ddsi0mt, ddsi1mt, ddsi2mt;

    converged = (input == ORACLE_EOS_INPUT_RT);                        /* :181-185 */
    if (input == ORACLE_EOS_INPUT_RE) v_want = state->e;               /* :187-191 */
    else if (input == ORACLE_EOS_INPUT_RP) v_want = state->p;

    for (int iter = 1; iter <= MAX_NEWTON; ++iter) {                   /* :193 */
        temp = state->T;
        den = state->rho;

        ytot1 = 1.0 / state->abar;
        ye = state->zbar / state->abar;
        din = ye * den;

        deni = 1.0 / den;
        tempi = 1.0 / temp;

        /* radiation, :206-217 */
        prad = asoli3 * temp * temp * temp * temp;
        dpraddd = 0.0;
        dpraddt = 4.0 * prad * tempi;
        erad = 3.0 * prad * deni;
        deraddd = -erad * deni;
        deraddt = 3.0 * dpraddt * deni;
        srad = (prad * deni + erad) * tempi;
        dsraddd = (dpraddd * deni - prad * deni * deni + deraddd) * tempi;
        dsraddt = (dpraddt * deni + deraddt - srad) * tempi;

        /* ions, :219-237 */
        pion = kergavo * ytot1 * den * temp;
        dpiondd = kergavo * ytot1 * temp;
        dpiondt = kergavo * ytot1 * den;
        eion = 1.5 * pion * deni;
        deiondd = (1.5 * dpiondd - eion) * deni;
        deiondt = 1.5 * dpiondt * deni;
        x = state->abar * state->abar * sqrt(state->abar) * deni / avo_eos;
        s = sioncon * temp;
        z = x * s * sqrt(s);
        y = log(z);
        sion = (pion * deni + eion) * tempi + kergavo * ytot1 * y;
        dsiondd = (dpiondd * deni - pion * deni * deni + deiondd) * tempi - kergavo * deni * ytot1;
        dsiondt = (dpiondt * deni + deiondt) * tempi - (pion * deni + eion) * tempi * tempi
                + 1.5 * kergavo * tempi * ytot1;

        /* hash locate, :242-245 (0-based).  Within an ulp of a node the last
         * bit of log10 decides the cell, and two faithful log10s (this host's
         * libm, a GPU's) can decide differently: the estimate is settled against
         * the node values, so that the cell is the one whose nodes bracket the
         * argument whatever log10 returned. */
        jat = ftrunc((log10(temp) - tlo) * tstpi);
        if (jat > JMAX - 2) jat = JMAX - 2;
        if (jat < 0) jat = 0;
        if (jat > 0 && temp < tab_t[jat]) --jat;
        else if (jat < JMAX - 2 && temp >= tab_t[jat + 1]) ++jat;
        iat = ftrunc((log10(din) - dlo) * dstpi);
        if (iat > IMAX - 2) iat = IMAX - 2;
        if (iat < 0) iat = 0;
        if (iat > 0 && din < tab_d[iat]) --iat;
        else if (iat < IMAX - 2 && din >= tab_d[iat + 1]) ++iat;

        /* :248-283 */
        fill4(fi + 0, tf, iat, jat);
        fill4(fi + 4, tft, iat, jat);
        fill4(fi + 8, tftt, iat, jat);
        fill4(fi + 12, tfd, iat, jat);
        fill4(fi + 16, tfdd, iat, jat);
        fill4(fi + 20, tfdt, iat, jat);
        fill4(fi + 24, tfddt, iat, jat);
        fill4(fi + 28, tfdtt, iat, jat);
        fill4(fi + 32, tfddtt, iat, jat);

        /* :286-289 */
        xt = fmx((temp - tab_t[jat]) * tab_dti[jat], 0.0);
        xd = fmx((din - tab_d[iat]) * tab_ddi[iat], 0.0);
        mxt = 1.0 - xt;
        mxd = 1.0 - xd;

        /* :292-306 */
        si0t = psi0(xt);
        si1t = psi1(xt) * tab_dt[jat];
        si2t = psi2(xt) * tab_dt2[jat];
        si0mt = psi0(mxt);
        si1mt = -psi1(mxt) * tab_dt[jat];
        si2mt = psi2(mxt) * tab_dt2[jat];
        si0d = psi0(xd);
        si1d = psi1(xd) * tab_dd[iat];
        si2d = psi2(xd) * tab_dd2[iat];
        si0md = psi0(mxd);
        si1md = -psi1(mxd) * tab_dd[iat];
        si2md = psi2(mxd) * tab_dd2[iat];

        /* :309-323 */
        dsi0t = dpsi0(xt) * tab_dti[jat];
        dsi1t = dpsi1(xt);
        dsi2t = dpsi2(xt) * tab_dt[jat];
        dsi0mt = -dpsi0(mxt) * tab_dti[jat];
        dsi1mt = dpsi1(mxt);
        dsi2mt = -dpsi2(mxt) * tab_dt[jat];
        dsi0d = dpsi0(xd) * tab_ddi[iat];
        dsi1d = dpsi1(xd);
        dsi2d = dpsi2(xd) * tab_dd[iat];
        dsi0md = -dpsi0(mxd) * tab_ddi[iat];
        dsi1md = dpsi1(mxd);
        dsi2md = -dpsi2(mxd) * tab_dd[iat];

        /* :326-332 */
        ddsi0t = ddpsi0(xt) * tab_dt2i[jat];
        ddsi1t = ddpsi1(xt) * tab_dti[jat];
        ddsi2t = ddpsi2(xt);
        ddsi0mt = ddpsi0(mxt) * tab_dt2i[jat];
        ddsi1mt = -ddpsi1(mxt) * tab_dti[jat];
        ddsi2mt = ddpsi2(mxt);

        /* :335-357 */
#ifndef ORACLE_FACTORED_EOS
        free_e = h5(fi, si0t, si1t, si2t, si0mt, si1mt, si2mt, si0d, si1d, si2d, si0md, si1md, si2md);
        df_d = h5(fi, si0t, si1t, si2t, si0mt, si1mt, si2mt, dsi0d, dsi1d, dsi2d, dsi0md, dsi1md, dsi2md);
        df_t = h5(fi, dsi0t, dsi1t, dsi2t, dsi0mt, dsi1mt, dsi2mt, si0d, si1d, si2d, si0md, si1md, si2md);
        df_tt = h5(fi, ddsi0t, ddsi1t, ddsi2t, ddsi0mt, ddsi1mt, ddsi2mt, si0d, si1d, si2d, si0md, si1md, si2md);
        df_dt = h5(fi, dsi0t, dsi1t, dsi2t, dsi0mt, dsi1mt, dsi2mt, dsi0d, dsi1d, dsi2d, dsi0md, dsi1md, dsi2md);
#else
        /* The same 36-term sums factored the way the production GPU build
         * forms them (temperature direction first for each density order and
         * density node, then the density direction, in fused multiply-adds):
         * a reordering of the interpolation's arithmetic, not of its
         * algorithm.  Only the timing build uses it; the parity build keeps
         * eos.F90's term order. */
        {
            /* fi[4*m + c]: table m in (f, ft, ftt, fd, fdd, fdt, fddt, fdtt, fddtt), corner
             * c = di + 2*dj; slot of (density order a, temperature order b) */
            static const int mslot[3][3] = {{0, 1, 2}, {3, 5, 7}, {4, 6, 8}};
            const double tw[3][3][2] = {{{si0t, si0mt}, {si1t, si1mt}, {si2t, si2mt}},
                                        {{dsi0t, dsi0mt}, {dsi1t, dsi1mt}, {dsi2t, dsi2mt}},
                                        {{ddsi0t, ddsi0mt}, {ddsi1t, ddsi1mt}, {ddsi2t, ddsi2mt}}};
            const double dw[3][2] = {{si0d, si0md}, {si1d, si1md}, {si2d, si2md}};
            const double ddw[3][2] = {{dsi0d, dsi0md}, {dsi1d, dsi1md}, {dsi2d, dsi2md}};
            double g[3][3][2];   /* [temperature weight set][density order a][density node di] */
            for (int a = 0; a < 3; ++a)
                for (int di = 0; di < 2; ++di) {
                    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
                    for (int b = 0; b < 3; ++b)
                        for (int dj = 0; dj < 2; ++dj) {
                            double v = fi[4 * mslot[a][b] + di + 2 * dj];
                            s0 = fma(v, tw[0][b][dj], s0);
                            s1 = fma(v, tw[1][b][dj], s1);
                            s2 = fma(v, tw[2][b][dj], s2);
                        }
                    g[0][a][di] = s0; g[1][a][di] = s1; g[2][a][di] = s2;
                }
            free_e = df_d = df_t = df_tt = df_dt = 0.0;
            for (int a = 0; a < 3; ++a)
                for (int di = 0; di < 2; ++di) {
                    free_e = fma(g[0][a][di], dw[a][di], free_e);
                    df_d = fma(g[0][a][di], ddw[a][di], df_d);
                    df_t = fma(g[1][a][di], dw[a][di], df_t);
                    df_tt = fma(g[2][a][di], dw[a][di], df_tt);
                    df_dt = fma(g[1][a][di], ddw[a][di], df_dt);
                }
        }
#endif

        /* :362-385 */
        si0t = xpsi0(xt);
        si1t = xpsi1(xt) * tab_dt[jat];
        si0mt = xpsi0(mxt);
        si1mt = -xpsi1(mxt) * tab_dt[jat];
        si0d = xpsi0(xd);
        si1d = xpsi1(xd) * tab_dd[iat];
        si0md = xpsi0(mxd);
        si1md = -xpsi1(mxd) * tab_dd[iat];
        dsi0t = xdpsi0(xt) * tab_dti[jat];
        dsi1t = xdpsi1(xt);
        dsi0mt = -xdpsi0(mxt) * tab_dti[jat];
        dsi1mt = xdpsi1(mxt);
        dsi0d = xdpsi0(xd) * tab_ddi[iat];
        dsi1d = xdpsi1(xd);
        dsi0md = -xdpsi0(mxd) * tab_ddi[iat];
        dsi1md = xdpsi1(mxd);
        (void)dsi0t; (void)dsi1t; (void)dsi0mt; (void)dsi1mt;
        (void)dsi0d; (void)dsi1d; (void)dsi0md; (void)dsi1md;

        /* :388-409 */
        fill4(fi + 0, tdpdf, iat, jat);
        fill4(fi + 4, tdpdft, iat, jat);
        fill4(fi + 8, tdpdfd, iat, jat);
        fill4(fi + 12, tdpdfdt, iat, jat);
        dpepdd = h3(fi, si0t, si1t, si0mt, si1mt, si0d, si1d, si0md, si1md);
        dpepdd = fmx(ye * dpepdd, 0.0);

        /* :412-432 */
        fill4(fi + 0, tef, iat, jat);
        fill4(fi + 4, teft, iat, jat);
        fill4(fi + 8, tefd, iat, jat);
        fill4(fi + 12, tefdt, iat, jat);
        state->eta = h3(fi, si0t, si1t, si0mt, si1mt, si0d, si1d, si0md, si1md);

        /* :435-456 */
        fill4(fi + 0, txf, iat, jat);
        fill4(fi + 4, txft, iat, jat);
        fill4(fi + 8, txfd, iat, jat);
        fill4(fi + 12, txfdt, iat, jat);
        state->xne = h3(fi, si0t, si1t, si0mt, si1mt, si0d, si1d, si0md, si1md);
        state->xnp = 0.0;

        /* :464-475 */
        x = din * din;
        pele = x * df_d;
        dpepdt = x * df_dt;
        x = ye * ye;
        sele = -df_t * ye;
        dsepdt = -df_tt * ye;
        dsepdd = -df_dt * x;
        eele = ye * free_e + temp * sele;
        deepdt = temp * dsepdt;
        deepdd = x * df_d + temp * dsepdd;

        /* :478-489 */
        pres = prad + pion + pele;
        ener = erad + eion + eele;
        entr = srad + sion + sele;
        dpresdd = dpraddd + dpiondd + dpepdd;
        dpresdt = dpraddt + dpiondt + dpepdt;
        denerdd = deraddd + deiondd + deepdd;
        denerdt = deraddt + deiondt + deepdt;
        dentrdd = dsraddd + dsiondd + dsepdd;
        dentrdt = dsraddt + dsiondt + dsepdt;

        if (g_coulomb) {
            coulomb_t c;
            coulomb(den, temp, ytot1, state->zbar, pion, dpiondd, dpiondt, &c);
            /* kept only while the totals stay positive */
            if (pres + c.p > 0.0 && ener + c.e > 0.0) {
                pres = pres + c.p;
                ener = ener + c.e;
                entr = entr + c.s;
                dpresdd = dpresdd + c.dpdd;
                dpresdt = dpresdt + c.dpdt;
                denerdd = denerdd + c.dedd;
                denerdt = denerdt + c.dedt;
                dentrdd = dentrdd + c.dsdd;
                dentrdt = dentrdt + c.dsdt;
            }
        }

        /* :491-518 */
        zz = pres * deni;
        zzi = den / pres;
        chit = temp / pres * dpresdt;
        chid = dpresdd * zzi;
        state->cv = denerdt;
        state->gam1 = chit * zz * chit / (temp * state->cv) + chid;
        state->cp = state->cv * state->gam1 / chid;
        state->p = pres;
        state->dpdT = dpresdt;
        state->dpdr = dpresdd;
        state->dpde = dpresdt / denerdt;
        state->dpdr_e = dpresdd - dpresdt * denerdd / denerdt;
        state->e = ener;
        state->dedT = denerdt;
        state->dedr = denerdd;
        state->s = entr;
        state->dsdT = dentrdt;
        state->dsdr = dentrdd;
        state->h = ener + pres / den;
        state->dhdr = denerdd + dpresdd / den - pres / (den * den);
        state->dhdT = denerdt + dpresdt / den;
        state->pele = pele;
        state->ppos = 0.0;

        if (converged) break;                                          /* :520-522 */

        temp_old = temp;                                               /* :526-550 */
        if (input == ORACLE_EOS_INPUT_RE) { v = state->e; dvdx = state->dedT; }
        else { v = state->p; dvdx = state->dpdT; }
        temp = temp - (v - v_want) / dvdx;
        temp = fmx(0.5 * temp_old, fmn(temp, 2.0 * temp_old));
        temp = fmx(mintemp, temp);
        state->T = temp;
        error = fabs((temp - temp_old) / temp_old);
        if (error < ttol) converged = 1;
    }

    state->cs = sqrt(state->gam1 * state->p / state->rho);            /* :556 */
    state->dpdA = 0.0; state->dpdZ = 0.0; state->dedA = 0.0; state->dedZ = 0.0;
    if (input == ORACLE_EOS_INPUT_RE) state->e = v_want;               /* :566-574 */
    else if (input == ORACLE_EOS_INPUT_RP) state->p = v_want;
}

/* abar/zbar as the state-cleaning kernels form them from rho*X
 * (e.g. Source/Castro_nd.F90:285-286) */
static inline void abar_zbar_cons(const double* ux, double rhoInv, double* abar, double* zbar)
{
    double s1 = 0.0, s2 = 0.0;
    for (int n = 0; n < nspec; ++n) s1 = s1 + ux[n] * aion_inv[n];
    for (int n = 0; n < nspec; ++n) s2 = s2 + ux[n] * zion[n] * aion_inv[n];
    *abar = ONE / (s1 * rhoInv);
    *zbar = *abar * (s2 * rhoInv);
}

/* ------------------------------------------------------------------------ */
/* State-cleaning kernels, Source/Castro_nd.F90                              */
/* ------------------------------------------------------------------------ */

/* enforce_minimum_density, Source/Castro_nd.F90:69-125 */
void oracle_enforce_minimum_density(const int* lo, const int* hi, double* up, const int* u_lo, const int* u_hi)
{
    fab_t u = mkfab(up, u_lo, u_hi);
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                if (AT(u, i, j, k, URHO) < small_dens) {
                    for (int n = 0; n < nspec; ++n)
                        AT(u, i, j, k, UFS + n) = AT(u, i, j, k, UFS + n) * (small_dens / AT(u, i, j, k, URHO));
                    oracle_eos_t es;
                    memset(&es, 0, sizeof es);
                    es.rho = small_dens;
                    es.T = small_temp;
                    double s1 = 0.0, s2 = 0.0;
                    for (int n = 0; n < nspec; ++n) s1 = s1 + AT(u, i, j, k, UFS + n) * aion_inv[n];
                    for (int n = 0; n < nspec; ++n) s2 = s2 + AT(u, i, j, k, UFS + n) * zion[n] * aion_inv[n];
                    es.abar = ONE / (s1 / small_dens);
                    es.zbar = es.abar * (s2 / small_dens);
                    oracle_eos(ORACLE_EOS_INPUT_RT, &es);
                    AT(u, i, j, k, URHO) = es.rho;
                    AT(u, i, j, k, UTEMP) = es.T;
                    AT(u, i, j, k, UMX) = ZERO;
                    AT(u, i, j, k, UMY) = ZERO;
                    AT(u, i, j, k, UMZ) = ZERO;
                    AT(u, i, j, k, UEINT) = es.rho * es.e;
                    AT(u, i, j, k, UEDEN) = AT(u, i, j, k, UEINT);
                }
            }
}

/* normalize_species, Source/Castro_nd.F90:129-160 */
void oracle_normalize_species(const int* lo, const int* hi, double* up, const int* u_lo, const int* u_hi)
{
    fab_t u = mkfab(up, u_lo, u_hi);
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double rho = AT(u, i, j, k, URHO);
                double sum = 0.0;
                for (int n = 0; n < nspec; ++n) {
                    double x = fmx(1.0e-30 * rho, fmn(rho, AT(u, i, j, k, UFS + n)));
                    AT(u, i, j, k, UFS + n) = x;
                }
                for (int n = 0; n < nspec; ++n) sum = sum + AT(u, i, j, k, UFS + n);
                for (int n = 0; n < nspec; ++n) AT(u, i, j, k, UFS + n) = AT(u, i, j, k, UFS + n) / sum;
            }
}

/* reset_internal_e, Source/Castro_nd.F90:164-249 */
void oracle_reset_internal_e(const int* lo, const int* hi, double* up, const int* u_lo, const int* u_hi)
{
    const double dual_energy_eta2 = 1.e-4;
    fab_t u = mkfab(up, u_lo, u_hi);
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double rhoInv = ONE / AT(u, i, j, k, URHO);
                double Up = AT(u, i, j, k, UMX) * rhoInv;
                double Vp = AT(u, i, j, k, UMY) * rhoInv;
                double Wp = AT(u, i, j, k, UMZ) * rhoInv;
                double ke = HALF * (Up * Up + Vp * Vp + Wp * Wp);
                double ux[ORACLE_MAX_SPEC];
                for (int n = 0; n < nspec; ++n) ux[n] = AT(u, i, j, k, UFS + n);
                if (AT(u, i, j, k, UEDEN) < ZERO) {
                    if (AT(u, i, j, k, UEINT) < ZERO) {
                        oracle_eos_t es;
                        memset(&es, 0, sizeof es);
                        es.rho = AT(u, i, j, k, URHO);
                        es.T = small_temp;
                        abar_zbar_cons(ux, rhoInv, &es.abar, &es.zbar);
                        oracle_eos(ORACLE_EOS_INPUT_RT, &es);
                        AT(u, i, j, k, UEINT) = AT(u, i, j, k, URHO) * es.e;
                    }
                    AT(u, i, j, k, UEDEN) = AT(u, i, j, k, UEINT) + AT(u, i, j, k, URHO) * ke;
                } else {
                    double rho_eint = AT(u, i, j, k, UEDEN) - AT(u, i, j, k, URHO) * ke;
                    if (rho_eint > ZERO && rho_eint / AT(u, i, j, k, UEDEN) > dual_energy_eta2) {
                        AT(u, i, j, k, UEINT) = rho_eint;
                    } else if (AT(u, i, j, k, UEINT) <= ZERO) {
                        oracle_eos_t es;
                        memset(&es, 0, sizeof es);
                        es.rho = AT(u, i, j, k, URHO);
                        es.T = small_temp;
                        abar_zbar_cons(ux, rhoInv, &es.abar, &es.zbar);
                        oracle_eos(ORACLE_EOS_INPUT_RT, &es);
                        double eint_new = es.e;
                        AT(u, i, j, k, UEINT) = AT(u, i, j, k, URHO) * eint_new;
                    }
                }
            }
}

/* compute_temp, Source/Castro_nd.F90:253-297 */
void oracle_compute_temp(const int* lo, const int* hi, double* up, const int* u_lo, const int* u_hi)
{
    fab_t u = mkfab(up, u_lo, u_hi);
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double rhoInv = ONE / AT(u, i, j, k, URHO);
                oracle_eos_t es;
                memset(&es, 0, sizeof es);
                es.rho = AT(u, i, j, k, URHO);
                es.T = AT(u, i, j, k, UTEMP);
                es.e = AT(u, i, j, k, UEINT) * rhoInv;
                double ux[ORACLE_MAX_SPEC];
                for (int n = 0; n < nspec; ++n) ux[n] = AT(u, i, j, k, UFS + n);
                abar_zbar_cons(ux, rhoInv, &es.abar, &es.zbar);
                oracle_eos(ORACLE_EOS_INPUT_RE, &es);
                AT(u, i, j, k, UTEMP) = es.T;
                AT(u, i, j, k, UEINT) = AT(u, i, j, k, URHO) * es.e;
            }
}

/* estdt, Source/timestep.F90:12-72 (reduce_min, Source/reduction.F90:41-69) */
void oracle_estdt(const int* lo, const int* hi, const double* up, const int* u_lo, const int* u_hi,
                  const double* dx, double* dt)
{
    fab_t u = mkfab(up, u_lo, u_hi);
    double dtl = *dt;
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double rhoInv = ONE / AT(u, i, j, k, URHO);
                oracle_eos_t es;
                memset(&es, 0, sizeof es);
                es.rho = AT(u, i, j, k, URHO);
                es.T = AT(u, i, j, k, UTEMP);
                es.e = AT(u, i, j, k, UEINT) * rhoInv;
                double ux[ORACLE_MAX_SPEC];
                for (int n = 0; n < nspec; ++n) ux[n] = AT(u, i, j, k, UFS + n);
                abar_zbar_cons(ux, rhoInv, &es.abar, &es.zbar);
                oracle_eos(ORACLE_EOS_INPUT_RE, &es);
                double ux_ = AT(u, i, j, k, UMX) * rhoInv;
                double uy_ = AT(u, i, j, k, UMY) * rhoInv;
                double uz_ = AT(u, i, j, k, UMZ) * rhoInv;
                double c = es.cs;
                double dt1 = dx[0] / (c + fabs(ux_));
                double dt2 = dx[1] / (c + fabs(uy_));
                double dt3 = dx[2] / (c + fabs(uz_));
                double m = fmn(fmn(dt1, dt2), dt3);
                dtl = fmn(dtl, m);
            }
    *dt = dtl;
}

/* ------------------------------------------------------------------------ */
/* Hydro kernels, Source/Castro_hydro_nd.F90                                 */
/* ------------------------------------------------------------------------ */

/* divu, Source/Castro_hydro_nd.F90:11-69 */
void oracle_divu(const int* lo, const int* hi, const double* qp, const int* q_lo, const int* q_hi,
                 const double* dx, double* dp, const int* d_lo, const int* d_hi)
{
    fab_t q = mkfab(qp, q_lo, q_hi);
    fab_t div = mkfab(dp, d_lo, d_hi);
    double dxinv = ONE / dx[0], dyinv = ONE / dx[1], dzinv = ONE / dx[2];
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double ux = FOURTH * (
                      + AT(q, i, j, k, QU) - AT(q, i - 1, j, k, QU)
                      + AT(q, i, j, k - 1, QU) - AT(q, i - 1, j, k - 1, QU)
                      + AT(q, i, j - 1, k, QU) - AT(q, i - 1, j - 1, k, QU)
                      + AT(q, i, j - 1, k - 1, QU) - AT(q, i - 1, j - 1, k - 1, QU)) * dxinv;
                double vy = FOURTH * (
                      + AT(q, i, j, k, QV) - AT(q, i, j - 1, k, QV)
                      + AT(q, i, j, k - 1, QV) - AT(q, i, j - 1, k - 1, QV)
                      + AT(q, i - 1, j, k, QV) - AT(q, i - 1, j - 1, k, QV)
                      + AT(q, i - 1, j, k - 1, QV) - AT(q, i - 1, j - 1, k - 1, QV)) * dyinv;
                double wz = FOURTH * (
                      + AT(q, i, j, k, QW) - AT(q, i, j, k - 1, QW)
                      + AT(q, i, j - 1, k, QW) - AT(q, i, j - 1, k - 1, QW)
                      + AT(q, i - 1, j, k, QW) - AT(q, i - 1, j, k - 1, QW)
                      + AT(q, i - 1, j - 1, k, QW) - AT(q, i - 1, j - 1, k - 1, QW)) * dzinv;
                AT(div, i, j, k, 0) = ux + vy + wz;
            }
}

/* ctoprim, Source/Castro_hydro_nd.F90:73-170 */
void oracle_ctoprim(const int* lo, const int* hi,
                    const double* up, const int* u_lo, const int* u_hi,
                    double* qp, const int* q_lo, const int* q_hi,
                    double* qap, const int* qa_lo, const int* qa_hi)
{
    fab_t u = mkfab(up, u_lo, u_hi);
    fab_t q = mkfab(qp, q_lo, q_hi);
    fab_t qaux = mkfab(qap, qa_lo, qa_hi);
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                AT(q, i, j, k, QRHO) = AT(u, i, j, k, URHO);
                double rhoinv = ONE / AT(q, i, j, k, QRHO);
                double vel0 = AT(u, i, j, k, UMX) * rhoinv;
                double vel1 = AT(u, i, j, k, UMY) * rhoinv;
                double vel2 = AT(u, i, j, k, UMZ) * rhoinv;
                AT(q, i, j, k, QU) = vel0;
                AT(q, i, j, k, QV) = vel1;
                AT(q, i, j, k, QW) = vel2;
                double kineng = HALF * AT(q, i, j, k, QRHO) *
                    (AT(q, i, j, k, QU) * AT(q, i, j, k, QU) + AT(q, i, j, k, QV) * AT(q, i, j, k, QV)
                     + AT(q, i, j, k, QW) * AT(q, i, j, k, QW));
                if ((AT(u, i, j, k, UEDEN) - kineng) / AT(u, i, j, k, UEDEN) > dual_energy_eta1)
                    AT(q, i, j, k, QREINT) = (AT(u, i, j, k, UEDEN) - kineng) * rhoinv;
                else
                    AT(q, i, j, k, QREINT) = AT(u, i, j, k, UEINT) * rhoinv;
                AT(q, i, j, k, QTEMP) = AT(u, i, j, k, UTEMP);
                for (int n = 0; n < nspec; ++n)
                    AT(q, i, j, k, QFS + n) = AT(u, i, j, k, UFS + n) * rhoinv;

                oracle_eos_t es;
                memset(&es, 0, sizeof es);
                es.T = AT(q, i, j, k, QTEMP);
                es.rho = AT(q, i, j, k, QRHO);
                es.e = AT(q, i, j, k, QREINT);
                double s1 = 0.0, s2 = 0.0;
                for (int n = 0; n < nspec; ++n) s1 = s1 + AT(q, i, j, k, QFS + n) * aion_inv[n];
                for (int n = 0; n < nspec; ++n) s2 = s2 + AT(q, i, j, k, QFS + n) * zion[n] * aion_inv[n];
                es.abar = ONE / s1;
                es.zbar = es.abar * s2;
                oracle_eos(ORACLE_EOS_INPUT_RE, &es);

                AT(q, i, j, k, QTEMP) = es.T;
                AT(q, i, j, k, QREINT) = es.e * AT(q, i, j, k, QRHO);
                AT(q, i, j, k, QPRES) = es.p;
                AT(q, i, j, k, QGAME) = AT(q, i, j, k, QPRES) / AT(q, i, j, k, QREINT) + ONE;
                AT(qaux, i, j, k, QDPDR) = es.dpdr_e;
                AT(qaux, i, j, k, QDPDE) = es.dpde;
                AT(qaux, i, j, k, QGAMC) = es.gam1;
                AT(qaux, i, j, k, QC) = es.cs;
            }
}

/* apply_av, Source/Castro_hydro_nd.F90:174-245 (stencil reproduced as written) */
void oracle_apply_av(const int* lo, const int* hi, int idir, const double* dx,
                     const double* dvp, const int* d_lo, const int* d_hi,
                     const double* up, const int* u_lo, const int* u_hi,
                     double* fp, const int* f_lo, const int* f_hi)
{
    const double difmag = 0.1;
    fab_t div = mkfab(dvp, d_lo, d_hi);
    fab_t u = mkfab(up, u_lo, u_hi);
    fab_t flux = mkfab(fp, f_lo, f_hi);
    for (int n = 0; n < NVAR; ++n)
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    if (n == UTEMP) continue;
                    double div1;
                    if (idir == 1) {
                        div1 = FOURTH * (AT(div, i, j, k, 0) + AT(div, i, j + 1, k, 0) +
                                         AT(div, i, j, k + 1, 0) + AT(div, i, j + 1, k, 0));
                        div1 = difmag * fmn(ZERO, div1);
                        div1 = div1 * (AT(u, i, j, k, n) - AT(u, i - 1, j, k, n));
                    } else if (idir == 2) {
                        div1 = FOURTH * (AT(div, i, j, k, 0) + AT(div, i + 1, j, k, 0) +
                                         AT(div, i, j, k + 1, 0) + AT(div, i + 1, j, k, 0));
                        div1 = difmag * fmn(ZERO, div1);
                        div1 = div1 * (AT(u, i, j, k, n) - AT(u, i, j - 1, k, n));
                    } else {
                        div1 = FOURTH * (AT(div, i, j, k, 0) + AT(div, i + 1, j, k, 0) +
                                         AT(div, i, j + 1, k, 0) + AT(div, i + 1, j + 1, k, 0));
                        div1 = difmag * fmn(ZERO, div1);
                        div1 = div1 * (AT(u, i, j, k, n) - AT(u, i, j, k - 1, n));
                    }
                    AT(flux, i, j, k, n) = AT(flux, i, j, k, n) + dx[idir - 1] * div1;
                }
}

/* normalize_species_fluxes, Source/Castro_hydro_nd.F90:248-297 */
void oracle_normalize_species_fluxes(const int* lo, const int* hi, double* fp, const int* f_lo, const int* f_hi)
{
    fab_t flux = mkfab(fp, f_lo, f_hi);
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double sum = ZERO, fac;
                for (int n = UFS; n < UFS + nspec; ++n) sum = sum + AT(flux, i, j, k, n);
                if (sum != ZERO) fac = AT(flux, i, j, k, URHO) / sum;
                else fac = ONE;
                for (int n = UFS; n < UFS + nspec; ++n) AT(flux, i, j, k, n) = AT(flux, i, j, k, n) * fac;
            }
}

/* store_flux, Source/Castro_hydro_nd.F90:301-340 */
void oracle_store_flux(const int* lo, const int* hi,
                       double* fop, const int* fo_lo, const int* fo_hi,
                       const double* fip, const int* fi_lo, const int* fi_hi,
                       const double* ap, const int* a_lo, const int* a_hi, double dt)
{
    fab_t fo = mkfab(fop, fo_lo, fo_hi);
    fab_t fi = mkfab(fip, fi_lo, fi_hi);
    fab_t area = mkfab(ap, a_lo, a_hi);
    for (int n = 0; n < NVAR; ++n)
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i)
                    AT(fo, i, j, k, n) = dt * AT(fi, i, j, k, n) * AT(area, i, j, k, 0);
}

/* fill_hydro_source, Source/Castro_hydro_nd.F90:344-441 */
void oracle_fill_hydro_source(const int* lo, const int* hi,
                              const double* up, const int* u_lo, const int* u_hi,
                              const double* qp, const int* q_lo, const int* q_hi,
                              double* sp, const int* s_lo, const int* s_hi,
                              const double* f1p, const int* f1_lo, const int* f1_hi,
                              const double* f2p, const int* f2_lo, const int* f2_hi,
                              const double* f3p, const int* f3_lo, const int* f3_hi,
                              const double* qxp, const int* qx_lo, const int* qx_hi,
                              const double* qyp, const int* qy_lo, const int* qy_hi,
                              const double* qzp, const int* qz_lo, const int* qz_hi,
                              const double* a1p, const int* a1_lo, const int* a1_hi,
                              const double* a2p, const int* a2_lo, const int* a2_hi,
                              const double* a3p, const int* a3_lo, const int* a3_hi,
                              const double* vp, const int* v_lo, const int* v_hi,
                              const double* dx, double dt)
{
    (void)up; (void)u_lo; (void)u_hi; (void)qp; (void)q_lo; (void)q_hi; (void)dt;
    fab_t src = mkfab(sp, s_lo, s_hi);
    fab_t f1 = mkfab(f1p, f1_lo, f1_hi), f2 = mkfab(f2p, f2_lo, f2_hi), f3 = mkfab(f3p, f3_lo, f3_hi);
    fab_t qx = mkfab(qxp, qx_lo, qx_hi), qy = mkfab(qyp, qy_lo, qy_hi), qz = mkfab(qzp, qz_lo, qz_hi);
    fab_t a1 = mkfab(a1p, a1_lo, a1_hi), a2 = mkfab(a2p, a2_lo, a2_hi), a3 = mkfab(a3p, a3_lo, a3_hi);
    fab_t vol = mkfab(vp, v_lo, v_hi);
    for (int n = 0; n < NVAR; ++n)
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    double volinv = ONE / AT(vol, i, j, k, 0);
                    AT(src, i, j, k, n) = AT(src, i, j, k, n) +
                        (AT(f1, i, j, k, n) * AT(a1, i, j, k, 0) - AT(f1, i + 1, j, k, n) * AT(a1, i + 1, j, k, 0)
                       + AT(f2, i, j, k, n) * AT(a2, i, j, k, 0) - AT(f2, i, j + 1, k, n) * AT(a2, i, j + 1, k, 0)
                       + AT(f3, i, j, k, n) * AT(a3, i, j, k, 0) - AT(f3, i, j, k + 1, n) * AT(a3, i, j, k + 1, 0)
                        ) * volinv;
                    if (n == UEINT) {
                        double pdivu =
                            HALF * (AT(qx, i + 1, j, k, GDPRES) + AT(qx, i, j, k, GDPRES)) *
                                   (AT(qx, i + 1, j, k, GDU) - AT(qx, i, j, k, GDU)) / dx[0] +
                            HALF * (AT(qy, i, j + 1, k, GDPRES) + AT(qy, i, j, k, GDPRES)) *
                                   (AT(qy, i, j + 1, k, GDV) - AT(qy, i, j, k, GDV)) / dx[1] +
                            HALF * (AT(qz, i, j, k + 1, GDPRES) + AT(qz, i, j, k, GDPRES)) *
                                   (AT(qz, i, j, k + 1, GDW) - AT(qz, i, j, k, GDW)) / dx[2];
                        AT(src, i, j, k, n) = AT(src, i, j, k, n) - pdivu;
                    }
                }
}

/* ------------------------------------------------------------------------ */
/* PPM, Source/ppm.F90                                                        */
/* ------------------------------------------------------------------------ */

/* uflatten, Source/ppm.F90:11-128 */
static double uflatten(int i, int j, int k, fab_t q)
{
    const double shktst = 0.33, zcut1 = 0.75, zcut2 = 0.85;
    const double dzcut = ONE / (zcut2 - zcut1);
    double flatn = ONE;
    for (int idir = 1; idir <= 3; ++idir) {
        int ex = (idir == 1), ey = (idir == 2), ez = (idir == 3);
        int qun = (idir == 1) ? QU : (idir == 2) ? QV : QW;
        double pr = AT(q, i + ex, j + ey, k + ez, QPRES);
        double pl = AT(q, i - ex, j - ey, k - ez, QPRES);
        double dp2 = AT(q, i + 2 * ex, j + 2 * ey, k + 2 * ez, QPRES) - AT(q, i - 2 * ex, j - 2 * ey, k - 2 * ez, QPRES);
        double du = AT(q, i + ex, j + ey, k + ez, qun) - AT(q, i - ex, j - ey, k - ez, qun);
        double dp = pr - pl;
        int ishft = (dp > ZERO) ? 1 : -1;
        double denom = fmx(small_pres, fabs(dp2));
        double denominv = ONE / denom;
        double zeta = fabs(dp) * denominv;
        double z = fmn(ONE, fmx(ZERO, dzcut * (zeta - zcut1)));
        double tst = (du <= ZERO) ? ONE : ZERO;
        double tmp = fmn(pr, pl);
        double chi = (fabs(dp) > shktst * tmp) ? tst : ZERO;

        int s = -ishft;
        pr = AT(q, i + (1 + s) * ex, j + (1 + s) * ey, k + (1 + s) * ez, QPRES);
        pl = AT(q, i + (-1 + s) * ex, j + (-1 + s) * ey, k + (-1 + s) * ez, QPRES);
        dp2 = AT(q, i + (2 + s) * ex, j + (2 + s) * ey, k + (2 + s) * ez, QPRES)
            - AT(q, i + (-2 + s) * ex, j + (-2 + s) * ey, k + (-2 + s) * ez, QPRES);
        du = AT(q, i + (1 + s) * ex, j + (1 + s) * ey, k + (1 + s) * ez, qun)
           - AT(q, i + (-1 + s) * ex, j + (-1 + s) * ey, k + (-1 + s) * ez, qun);
        dp = pr - pl;
        denom = fmx(small_pres, fabs(dp2));
        denominv = ONE / denom;
        zeta = fabs(dp) * denominv;
        double z2 = fmn(ONE, fmx(ZERO, dzcut * (zeta - zcut1)));
        tst = (du <= ZERO) ? ONE : ZERO;
        tmp = fmn(pr, pl);
        double chi2 = (fabs(dp) > shktst * tmp) ? tst : ZERO;
        flatn = fmn(flatn, ONE - fmx(chi2 * z2, chi * z));
    }
    return flatn;
}

/* ppm_reconstruct, Source/ppm.F90:132-236; s[0..4] holds s(-2..2) */
static void ppm_reconstruct(const double* s, double flatn, double* smo, double* spo)
{
    double dsl, dsr, dsc, dsvl_l, dsvl_r, sm, sp;
    dsl = TWO * (s[1] - s[0]);
    dsr = TWO * (s[2] - s[1]);
    if (dsl * dsr > ZERO) {
        dsc = HALF * (s[2] - s[0]);
        dsvl_l = copysign(ONE, dsc) * fmn(fmn(fabs(dsc), fabs(dsl)), fabs(dsr));
    } else dsvl_l = ZERO;
    dsl = TWO * (s[2] - s[1]);
    dsr = TWO * (s[3] - s[2]);
    if (dsl * dsr > ZERO) {
        dsc = HALF * (s[3] - s[1]);
        dsvl_r = copysign(ONE, dsc) * fmn(fmn(fabs(dsc), fabs(dsl)), fabs(dsr));
    } else dsvl_r = ZERO;
    sm = HALF * (s[2] + s[1]) - SIXTH * (dsvl_r - dsvl_l);
    sm = fmx(sm, fmn(s[2], s[1]));
    sm = fmn(sm, fmx(s[2], s[1]));

    dsl = TWO * (s[2] - s[1]);
    dsr = TWO * (s[3] - s[2]);
    if (dsl * dsr > ZERO) {
        dsc = HALF * (s[3] - s[1]);
        dsvl_l = copysign(ONE, dsc) * fmn(fmn(fabs(dsc), fabs(dsl)), fabs(dsr));
    } else dsvl_l = ZERO;
    dsl = TWO * (s[3] - s[2]);
    dsr = TWO * (s[4] - s[3]);
    if (dsl * dsr > ZERO) {
        dsc = HALF * (s[4] - s[2]);
        dsvl_r = copysign(ONE, dsc) * fmn(fmn(fabs(dsc), fabs(dsl)), fabs(dsr));
    } else dsvl_r = ZERO;
    sp = HALF * (s[3] + s[2]) - SIXTH * (dsvl_r - dsvl_l);
    sp = fmx(sp, fmn(s[3], s[2]));
    sp = fmn(sp, fmx(s[3], s[2]));

    sm = flatn * sm + (ONE - flatn) * s[2];
    sp = flatn * sp + (ONE - flatn) * s[2];

    if ((sp - s[2]) * (s[2] - sm) <= ZERO) {
        sp = s[2];
        sm = s[2];
    } else if (fabs(sp - s[2]) >= TWO * fabs(sm - s[2])) {
        sp = THREE * s[2] - TWO * sm;
    } else if (fabs(sm - s[2]) >= TWO * fabs(sp - s[2])) {
        sm = THREE * s[2] - TWO * sp;
    }
    *smo = sm;
    *spo = sp;
}

/* ppm_int_profile, Source/ppm.F90:240-305 */
static void ppm_int_profile(double sm, double sp, double sc, double u, double c, double dtdx,
                            double* Ip, double* Im)
{
    double s6 = SIX * sc - THREE * (sm + sp);
    double speeds[3] = {u - c, u, u + c};
    for (int w = 0; w < 3; ++w) {
        double speed = speeds[w];
        double sigma = fabs(speed) * dtdx;
        if (speed <= ZERO) {
            Ip[w] = sp;
            Im[w] = sm + HALF * sigma * (sp - sm + (ONE - TWO3RD * sigma) * s6);
        } else {
            Ip[w] = sp - HALF * sigma * (sp - sm - (ONE - TWO3RD * sigma) * s6);
            Im[w] = sm;
        }
    }
}

/* trace_ppm, Source/ppm.F90:309-743 */
void oracle_trace_ppm(const int* lo, const int* hi, const int* vlo, const int* vhi, int idir,
                      const double* qdp, const int* q_lo, const int* q_hi,
                      const double* qap, const int* qa_lo, const int* qa_hi,
                      double* qmp, const int* qm_lo, const int* qm_hi,
                      double* qpp, const int* qp_lo, const int* qp_hi,
                      const int* domlo, const int* domhi, const double* dx, double dt)
{
    (void)domlo; (void)domhi;
    fab_t q = mkfab(qdp, q_lo, q_hi);
    fab_t qaux = mkfab(qap, qa_lo, qa_hi);
    fab_t qm = mkfab(qmp, qm_lo, qm_hi);
    fab_t qp = mkfab(qpp, qp_lo, qp_hi);
    double dtdx = dt / dx[idir - 1];
    int QUN, QUT, QUTT;
    if (idir == 1) { QUN = QU; QUT = QV; QUTT = QW; }
    else if (idir == 2) { QUN = QV; QUT = QW; QUTT = QU; }
    else { QUN = QW; QUT = QU; QUTT = QV; }
    int ex = (idir == 1), ey = (idir == 2), ez = (idir == 3);

    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double Ip[QTHERM][3], Im[QTHERM][3], Ip_gc[3], Im_gc[3], Ip_sp[3], Im_sp[3];
                double s[5], sm, sp;
                double cc = AT(qaux, i, j, k, QC);
                double un = AT(q, i, j, k, QUN);
                double flatn = uflatten(i, j, k, q);
                int idx = (idir == 1) ? i : (idir == 2) ? j : k;

                for (int n = 0; n < QTHERM; ++n) {
                    if (n == QGAME || n == QTEMP) continue;
                    for (int m = -2; m <= 2; ++m) s[m + 2] = AT(q, i + m * ex, j + m * ey, k + m * ez, n);
                    ppm_reconstruct(s, flatn, &sm, &sp);
                    ppm_int_profile(sm, sp, s[2], un, cc, dtdx, Ip[n], Im[n]);
                }
                for (int m = -2; m <= 2; ++m) s[m + 2] = AT(qaux, i + m * ex, j + m * ey, k + m * ez, QGAMC);
                ppm_reconstruct(s, flatn, &sm, &sp);
                ppm_int_profile(sm, sp, s[2], un, cc, dtdx, Ip_gc, Im_gc);

                for (int ispec = 0; ispec < nspec; ++ispec) {
                    int n = QFS + ispec;
                    for (int m = -2; m <= 2; ++m) s[m + 2] = AT(q, i + m * ex, j + m * ey, k + m * ez, n);
                    ppm_reconstruct(s, flatn, &sm, &sp);
                    ppm_int_profile(sm, sp, s[2], un, cc, dtdx, Ip_sp, Im_sp);
                    if (idx >= vlo[idir - 1]) AT(qp, i, j, k, n) = Im_sp[1];
                    if (idx <= vhi[idir - 1]) AT(qm, i + ex, j + ey, k + ez, n) = Ip_sp[1];
                }

                if (idx >= vlo[idir - 1]) {
                    double rho_ref = Im[QRHO][0];
                    double un_ref = Im[QUN][0];
                    double p_ref = Im[QPRES][0];
                    double rhoe_g_ref = Im[QREINT][0];
                    double gam_g_ref = Im_gc[0];
                    rho_ref = fmx(rho_ref, small_dens);
                    double rho_ref_inv = ONE / rho_ref;
                    p_ref = fmx(p_ref, small_pres);
                    double csq_ref = gam_g_ref * p_ref * rho_ref_inv;
                    double cc_ref = sqrt(csq_ref);
                    double cc_ref_inv = ONE / cc_ref;
                    double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv;
                    double dum = un_ref - Im[QUN][0];
                    double dptotm = p_ref - Im[QPRES][0];
                    double drho = rho_ref - Im[QRHO][1];
                    double dptot = p_ref - Im[QPRES][1];
                    double drhoe_g = rhoe_g_ref - Im[QREINT][1];
                    double dup = un_ref - Im[QUN][2];
                    double dptotp = p_ref - Im[QPRES][2];
                    double alpham = HALF * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
                    double alphap = HALF * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
                    double alpha0r = drho - dptot / csq_ref;
                    double alpha0e_g = drhoe_g - dptot * h_g_ref / csq_ref;
                    alpham = (un - cc > ZERO) ? ZERO : -alpham;
                    alphap = (un + cc > ZERO) ? ZERO : -alphap;
                    alpha0r = (un > ZERO) ? ZERO : -alpha0r;
                    alpha0e_g = (un > ZERO) ? ZERO : -alpha0e_g;
                    AT(qp, i, j, k, QRHO) = fmx(small_dens, rho_ref + alphap + alpham + alpha0r);
                    AT(qp, i, j, k, QUN) = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
                    AT(qp, i, j, k, QREINT) = rhoe_g_ref + (alphap + alpham) * h_g_ref + alpha0e_g;
                    AT(qp, i, j, k, QPRES) = fmx(small_pres, p_ref + (alphap + alpham) * csq_ref);
                    AT(qp, i, j, k, QUT) = Im[QUT][1];
                    AT(qp, i, j, k, QUTT) = Im[QUTT][1];
                }

                if (idx <= vhi[idir - 1]) {
                    double rho_ref = Ip[QRHO][2];
                    double un_ref = Ip[QUN][2];
                    double p_ref = Ip[QPRES][2];
                    double rhoe_g_ref = Ip[QREINT][2];
                    double gam_g_ref = Ip_gc[2];
                    rho_ref = fmx(rho_ref, small_dens);
                    double rho_ref_inv = ONE / rho_ref;
                    p_ref = fmx(p_ref, small_pres);
                    double csq_ref = gam_g_ref * p_ref * rho_ref_inv;
                    double cc_ref = sqrt(csq_ref);
                    double cc_ref_inv = ONE / cc_ref;
                    double h_g_ref = (p_ref + rhoe_g_ref) * rho_ref_inv;
                    double dum = un_ref - Ip[QUN][0];
                    double dptotm = p_ref - Ip[QPRES][0];
                    double drho = rho_ref - Ip[QRHO][1];
                    double dptot = p_ref - Ip[QPRES][1];
                    double drhoe_g = rhoe_g_ref - Ip[QREINT][1];
                    double dup = un_ref - Ip[QUN][2];
                    double dptotp = p_ref - Ip[QPRES][2];
                    double alpham = HALF * (dptotm * rho_ref_inv * cc_ref_inv - dum) * rho_ref * cc_ref_inv;
                    double alphap = HALF * (dptotp * rho_ref_inv * cc_ref_inv + dup) * rho_ref * cc_ref_inv;
                    double alpha0r = drho - dptot / csq_ref;
                    double alpha0e_g = drhoe_g - dptot * h_g_ref / csq_ref;
                    alpham = (un - cc > ZERO) ? -alpham : ZERO;
                    alphap = (un + cc > ZERO) ? -alphap : ZERO;
                    alpha0r = (un > ZERO) ? -alpha0r : ZERO;
                    alpha0e_g = (un > ZERO) ? -alpha0e_g : ZERO;
                    int ii = i + ex, jj = j + ey, kk = k + ez;
                    AT(qm, ii, jj, kk, QRHO) = fmx(small_dens, rho_ref + alphap + alpham + alpha0r);
                    AT(qm, ii, jj, kk, QUN) = un_ref + (alphap - alpham) * cc_ref * rho_ref_inv;
                    AT(qm, ii, jj, kk, QREINT) = rhoe_g_ref + (alphap + alpham) * h_g_ref + alpha0e_g;
                    AT(qm, ii, jj, kk, QPRES) = fmx(small_pres, p_ref + (alphap + alpham) * csq_ref);
                    AT(qm, ii, jj, kk, QUT) = Ip[QUT][1];
                    AT(qm, ii, jj, kk, QUTT) = Ip[QUTT][1];
                }
            }
}

/* ------------------------------------------------------------------------ */
/* CGF Riemann solver, Source/riemann.F90:10-331                             */
/* ------------------------------------------------------------------------ */
void oracle_compute_flux(const int* lo, const int* hi,
                         const double* qlp, const int* ql_lo, const int* ql_hi,
                         const double* qrp, const int* qr_lo, const int* qr_hi,
                         double* fxp, const int* fx_lo, const int* fx_hi,
                         double* qip, const int* qi_lo, const int* qi_hi,
                         double* qgp, const int* qg_lo, const int* qg_hi,
                         const double* qap, const int* qa_lo, const int* qa_hi,
                         int idir)
{
    fab_t ql = mkfab(qlp, ql_lo, ql_hi), qr = mkfab(qrp, qr_lo, qr_hi);
    fab_t flx = mkfab(fxp, fx_lo, fx_hi), qint = mkfab(qip, qi_lo, qi_hi);
    fab_t qgdnv = mkfab(qgp, qg_lo, qg_hi), qaux = mkfab(qap, qa_lo, qa_hi);
    int iu, iv1, iv2, im1, im2, im3;
    if (idir == 1) { iu = QU; iv1 = QV; iv2 = QW; im1 = UMX; im2 = UMY; im3 = UMZ; }
    else if (idir == 2) { iu = QV; iv1 = QU; iv2 = QW; im1 = UMY; im2 = UMX; im3 = UMZ; }
    else { iu = QW; iv1 = QU; iv2 = QV; im1 = UMZ; im2 = UMX; im3 = UMY; }
    int ex = (idir == 1), ey = (idir == 2), ez = (idir == 3);

    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double rl = fmx(AT(ql, i, j, k, QRHO), small_dens);
                double ul = AT(ql, i, j, k, iu);
                double v1l = AT(ql, i, j, k, iv1);
                double v2l = AT(ql, i, j, k, iv2);
                double pl = fmx(AT(ql, i, j, k, QPRES), small_pres);
                double rel = AT(ql, i, j, k, QREINT);
                double rr = fmx(AT(qr, i, j, k, QRHO), small_dens);
                double ur = AT(qr, i, j, k, iu);
                double v1r = AT(qr, i, j, k, iv1);
                double v2r = AT(qr, i, j, k, iv2);
                double pr = fmx(AT(qr, i, j, k, QPRES), small_pres);
                double rer = AT(qr, i, j, k, QREINT);

                double cR = AT(qaux, i, j, k, QC), cL = AT(qaux, i - ex, j - ey, k - ez, QC);
                double csmall = fmx(small, small * fmx(cR, cL));
                double cavg = HALF * (cR + cL);
                double gamcl = AT(qaux, i - ex, j - ey, k - ez, QGAMC);
                double gamcr = AT(qaux, i, j, k, QGAMC);

                double wsmall = small_dens * csmall;
                double wl = fmx(wsmall, sqrt(fabs(gamcl * pl * rl)));
                double wr = fmx(wsmall, sqrt(fabs(gamcr * pr * rr)));
                double wwinv = ONE / (wl + wr);
                double pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) * wwinv;
                double ustar = ((wl * ul + wr * ur) + (pl - pr)) * wwinv;
                pstar = fmx(pstar, small_pres);
                if (fabs(ustar) < smallu * HALF * (fabs(ul) + fabs(ur))) ustar = ZERO;

                double sgnm = copysign(ONE, ustar);
                if (ustar == ZERO) sgnm = ZERO;
                double fp = HALF * (ONE + sgnm);
                double fm = HALF * (ONE - sgnm);

                double ro = fp * rl + fm * rr;
                double uo = fp * ul + fm * ur;
                double po = fp * pl + fm * pr;
                double reo = fp * rel + fm * rer;
                double gamco = fp * gamcl + fm * gamcr;
                ro = fmx(small_dens, ro);
                double roinv = ONE / ro;
                double co = sqrt(fabs(gamco * po * roinv));
                co = fmx(csmall, co);
                double co2inv = ONE / (co * co);

                AT(qint, i, j, k, iv1) = fp * v1l + fm * v1r;
                AT(qint, i, j, k, iv2) = fp * v2l + fm * v2r;

                double drho = (pstar - po) * co2inv;
                double rstar = ro + drho;
                rstar = fmx(small_dens, rstar);
                double rstarinv = ONE / rstar;
                double entho = (reo + po) * roinv * co2inv;
                double estar = reo + (pstar - po) * entho;
                double cstar = sqrt(fabs(gamco * pstar * rstarinv));
                cstar = fmx(cstar, csmall);

                sgnm = copysign(ONE, ustar);
                double spout = co - sgnm * uo;
                double spin = cstar - sgnm * ustar;
                double ushock = HALF * (spin + spout);
                if (pstar - po > ZERO) { spin = ushock; spout = ushock; }
                double scr;
                if (spout - spin == ZERO) scr = small * cavg;
                else scr = spout - spin;
                double scrinv = ONE / scr;
                double frac = (ONE + (spout + spin) * scrinv) * HALF;
                frac = fmx(ZERO, fmn(ONE, frac));

                AT(qint, i, j, k, QRHO) = frac * rstar + (ONE - frac) * ro;
                AT(qint, i, j, k, iu) = frac * ustar + (ONE - frac) * uo;
                AT(qint, i, j, k, QPRES) = frac * pstar + (ONE - frac) * po;
                double regdnv = frac * estar + (ONE - frac) * reo;
                if (spout < ZERO) {
                    AT(qint, i, j, k, QRHO) = ro;
                    AT(qint, i, j, k, iu) = uo;
                    AT(qint, i, j, k, QPRES) = po;
                    regdnv = reo;
                }
                if (spin >= ZERO) {
                    AT(qint, i, j, k, QRHO) = rstar;
                    AT(qint, i, j, k, iu) = ustar;
                    AT(qint, i, j, k, QPRES) = pstar;
                    regdnv = estar;
                }
                double regdnvinv = ONE / regdnv;
                AT(qint, i, j, k, QGAME) = AT(qint, i, j, k, QPRES) * regdnvinv + ONE;
                AT(qint, i, j, k, QPRES) = fmx(AT(qint, i, j, k, QPRES), small_pres);
                AT(qint, i, j, k, QREINT) = regdnv;
                for (int ispec = 0; ispec < nspec; ++ispec) {
                    int nqp = QFS + ispec;
                    AT(qint, i, j, k, nqp) = fp * AT(ql, i, j, k, nqp) + fm * AT(qr, i, j, k, nqp);
                }

                AT(qgdnv, i, j, k, GDRHO) = AT(qint, i, j, k, QRHO);
                AT(qgdnv, i, j, k, GDU) = AT(qint, i, j, k, QU);
                AT(qgdnv, i, j, k, GDV) = AT(qint, i, j, k, QV);
                AT(qgdnv, i, j, k, GDW) = AT(qint, i, j, k, QW);
                AT(qgdnv, i, j, k, GDPRES) = AT(qint, i, j, k, QPRES);
                AT(qgdnv, i, j, k, GDGAME) = AT(qint, i, j, k, QGAME);

                double u_adv = AT(qint, i, j, k, iu);
                double rhoeint = AT(qint, i, j, k, QREINT);
                AT(flx, i, j, k, URHO) = AT(qint, i, j, k, QRHO) * u_adv;
                AT(flx, i, j, k, im1) = AT(flx, i, j, k, URHO) * AT(qint, i, j, k, iu);
                if (g_mom_flux_p) AT(flx, i, j, k, im1) = AT(flx, i, j, k, im1) + AT(qint, i, j, k, QPRES);
                AT(flx, i, j, k, im2) = AT(flx, i, j, k, URHO) * AT(qint, i, j, k, iv1);
                AT(flx, i, j, k, im3) = AT(flx, i, j, k, URHO) * AT(qint, i, j, k, iv2);
                double qu = AT(qint, i, j, k, iu), q1 = AT(qint, i, j, k, iv1), q2 = AT(qint, i, j, k, iv2);
                double rhoetot = rhoeint + HALF * AT(qint, i, j, k, QRHO) * (qu * qu + q1 * q1 + q2 * q2);
                AT(flx, i, j, k, UEDEN) = u_adv * (rhoetot + AT(qint, i, j, k, QPRES));
                AT(flx, i, j, k, UEINT) = u_adv * rhoeint;
                AT(flx, i, j, k, UTEMP) = ZERO;
                for (int ispec = 0; ispec < nspec; ++ispec)
                    AT(flx, i, j, k, UFS + ispec) = AT(flx, i, j, k, URHO) * AT(qint, i, j, k, QFS + ispec);
            }
}

/* ------------------------------------------------------------------------ */
/* Transverse corrections, Source/trans.F90                                  */
/* ------------------------------------------------------------------------ */

/* trans1, Source/trans.F90:14-243 */
void oracle_trans1(const int* lo, const int* hi, int idir1, int idir2,
                   const double* q2mp, const int* q2m_lo, const int* q2m_hi,
                   double* q2mop, const int* q2mo_lo, const int* q2mo_hi,
                   const double* q2pp, const int* q2p_lo, const int* q2p_hi,
                   double* q2pop, const int* q2po_lo, const int* q2po_hi,
                   const double* qap, const int* qa_lo, const int* qa_hi,
                   const double* f1p, const int* f1_lo, const int* f1_hi,
                   const double* q1p, const int* q1_lo, const int* q1_hi,
                   double cdtdx)
{
    fab_t q2m = mkfab(q2mp, q2m_lo, q2m_hi), q2mo = mkfab(q2mop, q2mo_lo, q2mo_hi);
    fab_t q2p = mkfab(q2pp, q2p_lo, q2p_hi), q2po = mkfab(q2pop, q2po_lo, q2po_hi);
    fab_t qaux = mkfab(qap, qa_lo, qa_hi), f1 = mkfab(f1p, f1_lo, f1_hi), q1 = mkfab(q1p, q1_lo, q1_hi);

    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                for (int d = -1; d <= 0; ++d) {
                    double lq2[8 + ORACLE_MAX_SPEC], lq2o[8 + ORACLE_MAX_SPEC];
                    for (int n = 0; n < QVAR; ++n) lq2o[n] = NAN;   /* never-written slots stay NaN */
                    int il = i, jl = j, kl = k, ir, jr, kr;
                    if (idir1 == 1) { ir = i + 1; jr = j; kr = k; }
                    else if (idir1 == 2) { ir = i; jr = j + 1; kr = k; }
                    else { ir = i; jr = j; kr = k + 1; }
                    if (idir2 == 1) { il += d; ir += d; }
                    else if (idir2 == 2) { jl += d; jr += d; }
                    else { kl += d; kr += d; }
                    if (d == -1) for (int n = 0; n < QVAR; ++n) lq2[n] = AT(q2m, i, j, k, n);
                    else for (int n = 0; n < QVAR; ++n) lq2[n] = AT(q2p, i, j, k, n);

                    for (int ispec = 0; ispec < nspec; ++ispec) {
                        int n = UFS + ispec, nqp = QFS + ispec;
                        double rrnew = lq2[QRHO] - cdtdx * (AT(f1, ir, jr, kr, URHO) - AT(f1, il, jl, kl, URHO));
                        double compu = lq2[QRHO] * lq2[nqp] - cdtdx * (AT(f1, ir, jr, kr, n) - AT(f1, il, jl, kl, n));
                        lq2o[nqp] = compu / rrnew;
                    }

                    double pgp = AT(q1, ir, jr, kr, GDPRES);
                    double pgm = AT(q1, il, jl, kl, GDPRES);
                    double ugp = AT(q1, ir, jr, kr, GDU + idir1 - 1);
                    double ugm = AT(q1, il, jl, kl, GDU + idir1 - 1);
                    double dup = pgp * ugp - pgm * ugm;
                    double du = ugp - ugm;
                    double pav = HALF * (pgp + pgm);
                    double gamc = AT(qaux, il, jl, kl, QGAMC);

                    double rrl2 = lq2[QRHO];
                    double rul2 = rrl2 * lq2[QU];
                    double rvl2 = rrl2 * lq2[QV];
                    double rwl2 = rrl2 * lq2[QW];
                    double ekenl2 = HALF * rrl2 * (lq2[QU] * lq2[QU] + lq2[QV] * lq2[QV] + lq2[QW] * lq2[QW]);
                    double rel2 = lq2[QREINT] + ekenl2;

                    double rrnewl2 = rrl2 - cdtdx * (AT(f1, ir, jr, kr, URHO) - AT(f1, il, jl, kl, URHO));
                    double runewl2 = rul2 - cdtdx * (AT(f1, ir, jr, kr, UMX) - AT(f1, il, jl, kl, UMX));
                    double rvnewl2 = rvl2 - cdtdx * (AT(f1, ir, jr, kr, UMY) - AT(f1, il, jl, kl, UMY));
                    double rwnewl2 = rwl2 - cdtdx * (AT(f1, ir, jr, kr, UMZ) - AT(f1, il, jl, kl, UMZ));
                    double renewl2 = rel2 - cdtdx * (AT(f1, ir, jr, kr, UEDEN) - AT(f1, il, jl, kl, UEDEN));

                    int reset_state = 0;
                    if (rrnewl2 < ZERO) {
                        rrnewl2 = rrl2; runewl2 = rul2; rvnewl2 = rvl2; rwnewl2 = rwl2; renewl2 = rel2;
                        reset_state = 1;
                    }
                    lq2o[QRHO] = rrnewl2;
                    double rhoinv = ONE / rrnewl2;
                    lq2o[QU] = runewl2 * rhoinv;
                    lq2o[QV] = rvnewl2 * rhoinv;
                    lq2o[QW] = rwnewl2 * rhoinv;
                    double rhoekenl2 = HALF * (runewl2 * runewl2 + rvnewl2 * rvnewl2 + rwnewl2 * rwnewl2) * rhoinv;
                    lq2o[QREINT] = renewl2 - rhoekenl2;
                    if (!reset_state) {
                        double pnewl2 = lq2[QPRES] - cdtdx * (dup + pav * du * (gamc - ONE));
                        lq2o[QPRES] = fmx(pnewl2, small_pres);
                    } else {
                        lq2o[QPRES] = lq2[QPRES];
                        lq2o[QGAME] = lq2[QGAME];
                    }
                    if (d == -1) for (int n = 0; n < QVAR; ++n) AT(q2mo, i, j, k, n) = lq2o[n];
                    else for (int n = 0; n < QVAR; ++n) AT(q2po, i, j, k, n) = lq2o[n];
                }
            }
}

/* trans2, Source/trans.F90:250-505 */
void oracle_trans2(const int* lo, const int* hi, int idir1, int idir2, int idir3,
                   const double* qm1p, const int* qm_lo, const int* qm_hi,
                   double* qm1op, const int* qmo_lo, const int* qmo_hi,
                   const double* qp1p, const int* qp_lo, const int* qp_hi,
                   double* qp1op, const int* qpo_lo, const int* qpo_hi,
                   const double* qap, const int* qa_lo, const int* qa_hi,
                   const double* f2p, const int* f2_lo, const int* f2_hi,
                   const double* f3p, const int* f3_lo, const int* f3_hi,
                   const double* q2p, const int* q2_lo, const int* q2_hi,
                   const double* q3p, const int* q3_lo, const int* q3_hi,
                   double cdtdx1, double cdtdx2, double cdtdx3)
{
    (void)cdtdx1;
    fab_t qm1 = mkfab(qm1p, qm_lo, qm_hi), qm1o = mkfab(qm1op, qmo_lo, qmo_hi);
    fab_t qp1 = mkfab(qp1p, qp_lo, qp_hi), qp1o = mkfab(qp1op, qpo_lo, qpo_hi);
    fab_t qaux = mkfab(qap, qa_lo, qa_hi);
    fab_t f2 = mkfab(f2p, f2_lo, f2_hi), f3 = mkfab(f3p, f3_lo, f3_hi);
    fab_t q2 = mkfab(q2p, q2_lo, q2_hi), q3 = mkfab(q3p, q3_lo, q3_hi);

    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                for (int d = -1; d <= 0; ++d) {
                    double lq[8 + ORACLE_MAX_SPEC], lqo[8 + ORACLE_MAX_SPEC];
                    for (int n = 0; n < QVAR; ++n) lqo[n] = NAN;
                    int il1 = i, jl1 = j, kl1 = k, il2 = i, jl2 = j, kl2 = k, il3 = i, jl3 = j, kl3 = k;
                    int ir2, jr2, kr2, ir3, jr3, kr3;
                    if (idir1 == 1) {
                        ir2 = i + d; jr2 = j + 1; kr2 = k;
                        ir3 = i + d; jr3 = j; kr3 = k + 1;
                        il1 = i + d; il2 = i + d; il3 = i + d;
                    } else if (idir1 == 2) {
                        ir2 = i + 1; jr2 = j + d; kr2 = k;
                        ir3 = i; jr3 = j + d; kr3 = k + 1;
                        jl1 = j + d; jl2 = j + d; jl3 = j + d;
                    } else {
                        ir2 = i + 1; jr2 = j; kr2 = k + d;
                        ir3 = i; jr3 = j + 1; kr3 = k + d;
                        kl1 = k + d; kl2 = k + d; kl3 = k + d;
                    }
                    if (d == -1) for (int n = 0; n < QVAR; ++n) lq[n] = AT(qm1, i, j, k, n);
                    else for (int n = 0; n < QVAR; ++n) lq[n] = AT(qp1, i, j, k, n);

                    for (int ispec = 0; ispec < nspec; ++ispec) {
                        int n = UFS + ispec, nqp = QFS + ispec;
                        double rrr = lq[QRHO];
                        double compr = rrr * lq[nqp];
                        double rrnewr = rrr - cdtdx2 * (AT(f2, ir2, jr2, kr2, URHO) - AT(f2, il2, jl2, kl2, URHO))
                                            - cdtdx3 * (AT(f3, ir3, jr3, kr3, URHO) - AT(f3, il3, jl3, kl3, URHO));
                        double compnr = compr - cdtdx2 * (AT(f2, ir2, jr2, kr2, n) - AT(f2, il2, jl2, kl2, n))
                                              - cdtdx3 * (AT(f3, ir3, jr3, kr3, n) - AT(f3, il3, jl3, kl3, n));
                        lqo[nqp] = compnr / rrnewr;
                    }

                    double gamc1 = AT(qaux, il1, jl1, kl1, QGAMC);
                    double pg2p = AT(q2, ir2, jr2, kr2, GDPRES);
                    double pg2m = AT(q2, il2, jl2, kl2, GDPRES);
                    double ug2p = AT(q2, ir2, jr2, kr2, GDU + idir2 - 1);
                    double ug2m = AT(q2, il2, jl2, kl2, GDU + idir2 - 1);
                    double du2p = pg2p * ug2p - pg2m * ug2m;
                    double p2av = HALF * (pg2p + pg2m);
                    double du2 = ug2p - ug2m;
                    double p2new = cdtdx2 * (du2p + p2av * du2 * (gamc1 - ONE));

                    double pg3p = AT(q3, ir3, jr3, kr3, GDPRES);
                    double pg3m = AT(q3, il3, jl3, kl3, GDPRES);
                    double ug3p = AT(q3, ir3, jr3, kr3, GDU + idir3 - 1);
                    double ug3m = AT(q3, il3, jl3, kl3, GDU + idir3 - 1);
                    double du3p = pg3p * ug3p - pg3m * ug3m;
                    double p3av = HALF * (pg3p + pg3m);
                    double du3 = ug3p - ug3m;
                    double p3new = cdtdx3 * (du3p + p3av * du3 * (gamc1 - ONE));

                    double rrr = lq[QRHO];
                    double rur = rrr * lq[QU];
                    double rvr = rrr * lq[QV];
                    double rwr = rrr * lq[QW];
                    double ekenr = HALF * rrr * (lq[QU] * lq[QU] + lq[QV] * lq[QV] + lq[QW] * lq[QW]);
                    double rer = lq[QREINT] + ekenr;

                    double rrnewr = rrr - cdtdx2 * (AT(f2, ir2, jr2, kr2, URHO) - AT(f2, il2, jl2, kl2, URHO))
                                        - cdtdx3 * (AT(f3, ir3, jr3, kr3, URHO) - AT(f3, il3, jl3, kl3, URHO));
                    double runewr = rur - cdtdx2 * (AT(f2, ir2, jr2, kr2, UMX) - AT(f2, il2, jl2, kl2, UMX))
                                        - cdtdx3 * (AT(f3, ir3, jr3, kr3, UMX) - AT(f3, il3, jl3, kl3, UMX));
                    double rvnewr = rvr - cdtdx2 * (AT(f2, ir2, jr2, kr2, UMY) - AT(f2, il2, jl2, kl2, UMY))
                                        - cdtdx3 * (AT(f3, ir3, jr3, kr3, UMY) - AT(f3, il3, jl3, kl3, UMY));
                    double rwnewr = rwr - cdtdx2 * (AT(f2, ir2, jr2, kr2, UMZ) - AT(f2, il2, jl2, kl2, UMZ))
                                        - cdtdx3 * (AT(f3, ir3, jr3, kr3, UMZ) - AT(f3, il3, jl3, kl3, UMZ));
                    double renewr = rer - cdtdx2 * (AT(f2, ir2, jr2, kr2, UEDEN) - AT(f2, il2, jl2, kl2, UEDEN))
                                        - cdtdx3 * (AT(f3, ir3, jr3, kr3, UEDEN) - AT(f3, il3, jl3, kl3, UEDEN));

                    int reset_state = 0;
                    if (rrnewr < ZERO) {
                        rrnewr = rrr; runewr = rur; rvnewr = rvr; rwnewr = rwr; renewr = rer;
                        reset_state = 1;
                    }
                    lqo[QRHO] = rrnewr;
                    lqo[QU] = runewr / rrnewr;
                    lqo[QV] = rvnewr / rrnewr;
                    lqo[QW] = rwnewr / rrnewr;
                    double rhoekenr = HALF * (runewr * runewr + rvnewr * rvnewr + rwnewr * rwnewr) / rrnewr;
                    lqo[QREINT] = renewr - rhoekenr;
                    if (!reset_state) {
                        double pnewr = lq[QPRES] - p2new - p3new;
                        lqo[QPRES] = pnewr;
                    } else {
                        lqo[QPRES] = lq[QPRES];
                        lqo[QGAME] = lq[QGAME];
                    }
                    lqo[QPRES] = fmx(lqo[QPRES], small_pres);
                    if (d == -1) for (int n = 0; n < QVAR; ++n) AT(qm1o, i, j, k, n) = lqo[n];
                    else for (int n = 0; n < QVAR; ++n) AT(qp1o, i, j, k, n) = lqo[n];
                }
            }
}

/* ------------------------------------------------------------------------ */
/* Problem setup, Source/Prob.F90:19-129                                     */
/* ------------------------------------------------------------------------ */
static oracle_prob_t prob = {
    0, 1.e4, 1.e21, 1.e6, 1.e52, 1.25e8, 10,
    {1.0}, 1.e9, NULL, {0, 0, 0}, {0, 0, 0}, 0.0
};

void oracle_set_problem(const oracle_prob_t* p) { prob = *p; }

/* Option (off by default, as in the reference): the interface pressure in the
 * normal momentum flux, as full Castro has it for Cartesian geometry.  The
 * reference's compute_flux omits it (Source/riemann.F90:306-308), and nothing
 * else adds a pressure gradient to the momentum (consup adds only p div u to
 * rho e, Source/Castro_hydro_nd.F90:425-434). */
void oracle_set_momentum_flux_pressure(int on) { g_mom_flux_p = on; }

/* Option (off by default, as in the reference): the EOS with the Coulomb
 * corrections above, as the reference's 2017 runs used them
 * (scaling/summitdev_20171020/1.out:14). */
void oracle_set_coulomb_corrections(int on) { g_coulomb = on; }

void oracle_initdata(const int* lo, const int* hi, double* up, const int* u_lo, const int* u_hi,
                     const double* dx, const double* problo, const double* probhi)
{
    fab_t u = mkfab(up, u_lo, u_hi);
    oracle_eos_t es;
    memset(&es, 0, sizeof es);
    double s1 = 0.0, s2 = 0.0;
    for (int n = 0; n < nspec; ++n) s1 = s1 + prob.X[n] * aion_inv[n];
    for (int n = 0; n < nspec; ++n) s2 = s2 + prob.X[n] * zion[n] * aion_inv[n];
    es.rho = prob.dens_ambient;
    if (prob.ambient_from_T) {
        es.T = prob.T_ambient;
        es.abar = ONE / s1;
        es.zbar = es.abar * s2;
        oracle_eos(ORACLE_EOS_INPUT_RT, &es);
    } else {                                   /* Prob.F90:51-57: species 1 only */
        es.p = prob.p_ambient;
        es.T = 1.e4;
        es.abar = aion[0];
        es.zbar = zion[0];
        oracle_eos(ORACLE_EOS_INPUT_RP, &es);
    }
    double e_ambient = es.e;
    double r_init = prob.r_init;
    double vctr = FOUR3RD * M_PI * (r_init * r_init * r_init);
    double e_exp = prob.exp_energy / vctr / prob.dens_ambient;
    double center[3];
    for (int d = 0; d < 3; ++d) center[d] = (problo[d] + probhi[d]) / 2.e0;
    int nsub = prob.nsub;
    fab_t pert;
    if (prob.pert) pert = mkfab(prob.pert, prob.pert_lo, prob.pert_hi);

    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double xmin = problo[0] + dx[0] * (double)i;
                double ymin = problo[1] + dx[1] * (double)j;
                double zmin = problo[2] + dx[2] * (double)k;
                int npert = 0, nambient = 0;
                for (int kk = 0; kk < nsub; ++kk) {
                    double zz = zmin + (dx[2] / (double)nsub) * (kk + 0.5e0);
                    for (int jj = 0; jj < nsub; ++jj) {
                        double yy = ymin + (dx[1] / (double)nsub) * (jj + 0.5e0);
                        for (int ii = 0; ii < nsub; ++ii) {
                            double xx = xmin + (dx[0] / (double)nsub) * (ii + 0.5e0);
                            double dist = (center[0] - xx) * (center[0] - xx) + (center[1] - yy) * (center[1] - yy)
                                        + (center[2] - zz) * (center[2] - zz);
                            if (dist <= r_init * r_init) npert = npert + 1;
                            else nambient = nambient + 1;
                        }
                    }
                }
                double eint = ((double)npert * e_exp + (double)nambient * e_ambient) / (double)(nsub * nsub * nsub);
                double rho = prob.dens_ambient;
                if (prob.pert) rho = prob.dens_ambient * (1.0 + prob.pert_amp * AT(pert, i, j, k, 0));
                AT(u, i, j, k, URHO) = rho;
                AT(u, i, j, k, UMX) = 0.e0;
                AT(u, i, j, k, UMY) = 0.e0;
                AT(u, i, j, k, UMZ) = 0.e0;
                AT(u, i, j, k, UTEMP) = prob.T_init;
                AT(u, i, j, k, UEDEN) = AT(u, i, j, k, URHO) * eint;
                AT(u, i, j, k, UEINT) = AT(u, i, j, k, URHO) * eint;
                for (int n = 0; n < nspec; ++n) AT(u, i, j, k, UFS + n) = prob.X[n] * AT(u, i, j, k, URHO);
            }
}

/* denerror, Source/Castro_nd.F90:301-345 */
void oracle_denerror(const int* lo, const int* hi, signed char* tag, const int* t_lo, const int* t_hi,
                     const double* dp, const int* d_lo, const int* d_hi, signed char tagval, signed char clearval)
{
    (void)clearval;
    const double dengrad_rel = 0.25;
    fab_t den = mkfab(dp, d_lo, d_hi);
    long tnx = t_hi[0] - t_lo[0] + 1, tny = t_hi[1] - t_lo[1] + 1;
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double ax = fabs(AT(den, i + 1, j, k, 0) - AT(den, i, j, k, 0));
                double ay = fabs(AT(den, i, j + 1, k, 0) - AT(den, i, j, k, 0));
                double az = fabs(AT(den, i, j, k + 1, 0) - AT(den, i, j, k, 0));
                ax = fmx(ax, fabs(AT(den, i, j, k, 0) - AT(den, i - 1, j, k, 0)));
                ay = fmx(ay, fabs(AT(den, i, j, k, 0) - AT(den, i, j - 1, k, 0)));
                az = fmx(az, fabs(AT(den, i, j, k, 0) - AT(den, i, j, k - 1, 0)));
                if (fmx(fmx(ax, ay), az) >= fabs(dengrad_rel * AT(den, i, j, k, 0)))
                    tag[(i - t_lo[0]) + tnx * ((j - t_lo[1]) + tny * (long)(k - t_lo[2]))] = tagval;
            }
}

/* calculate_blast_radius, Source/Castro_nd.F90:349-400 */
void oracle_calculate_blast_radius(const int* lo, const int* hi, const double* up, const int* u_lo, const int* u_hi,
                                   const double* dx, const double* problo, const double* probhi,
                                   double* blast_mass, double* blast_radius, double max_density)
{
    const double density_tolerance = 0.1;
    fab_t u = mkfab(up, u_lo, u_hi);
    double center[3];
    for (int d = 0; d < 3; ++d) center[d] = (probhi[d] - problo[d]) / TWO;
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                double x = problo[0] + (i + HALF) * dx[0] - center[0];
                double y = problo[1] + (j + HALF) * dx[1] - center[1];
                double z = problo[2] + (k + HALF) * dx[2] - center[2];
                if (fabs(AT(u, i, j, k, URHO) - max_density) / max_density <= density_tolerance) {
                    *blast_mass = *blast_mass + AT(u, i, j, k, URHO);
                    *blast_radius = *blast_radius + AT(u, i, j, k, URHO) * sqrt(x * x + y * y + z * z);
                }
            }
}

/* ------------------------------------------------------------------------ */
/* construct_hydro_source for one tile, Source/Castro_hydro.cpp:31-395       */
/* ------------------------------------------------------------------------ */
typedef struct { int lo[3], hi[3]; } box_t;

static box_t grow_box(box_t b, int gx, int gy, int gz)
{
    b.lo[0] -= gx; b.lo[1] -= gy; b.lo[2] -= gz;
    b.hi[0] += gx; b.hi[1] += gy; b.hi[2] += gz;
    return b;
}
static box_t surrounding_nodes(box_t b, int d) { b.hi[d] += 1; return b; }
static long box_npts(box_t b)
{
    return (long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
}
/* an uninitialised FArrayBox: NaN-filled so that any read of a value the
 * reference never writes shows up in the outputs */
static double* fab_alloc(box_t b, int ncomp)
{
    long n = box_npts(b) * ncomp;
    double* p = (double*)malloc(sizeof(double) * (size_t)n);
    for (long m = 0; m < n; ++m) p[m] = NAN;
    return p;
}

void oracle_construct_hydro_source_tile(const int* bx_lo, const int* bx_hi,
                                        const double* sb, const int* sb_lo, const int* sb_hi,
                                        double* src, const int* s_lo, const int* s_hi,
                                        const int* domlo, const int* domhi,
                                        const double* dx, double dt)
{
    box_t bx; memcpy(bx.lo, bx_lo, sizeof bx.lo); memcpy(bx.hi, bx_hi, sizeof bx.hi);
    box_t obx = grow_box(bx, 1, 1, 1);
    box_t qbx = grow_box(bx, 4, 4, 4);
    box_t ebx[3], gebx[3], tbx[3][3];

    double* q = fab_alloc(qbx, QVAR);
    double* qaux = fab_alloc(qbx, NQAUX);
    oracle_ctoprim(qbx.lo, qbx.hi, sb, sb_lo, sb_hi, q, qbx.lo, qbx.hi, qaux, qbx.lo, qbx.hi);

    double* flux[3]; double* qe[3];
    for (int d = 0; d < 3; ++d) {
        ebx[d] = surrounding_nodes(bx, d);
        gebx[d] = grow_box(ebx[d], 1, 1, 1);
        flux[d] = fab_alloc(gebx[d], NVAR);
        qe[d] = fab_alloc(gebx[d], NGDNV);
    }
    tbx[0][0] = grow_box(ebx[0], 0, 1, 1);
    tbx[0][1] = grow_box(ebx[0], 0, 0, 1);
    tbx[0][2] = grow_box(ebx[0], 0, 1, 0);
    tbx[1][0] = grow_box(ebx[1], 0, 0, 1);
    tbx[1][1] = grow_box(ebx[1], 1, 0, 1);
    tbx[1][2] = grow_box(ebx[1], 1, 0, 0);
    tbx[2][0] = grow_box(ebx[2], 0, 1, 0);
    tbx[2][1] = grow_box(ebx[2], 1, 0, 0);
    tbx[2][2] = grow_box(ebx[2], 1, 1, 0);

    double* qm[3][3]; double* qp[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            qm[a][b] = fab_alloc(tbx[a][b], QVAR);
            qp[a][b] = fab_alloc(tbx[a][b], QVAR);
        }

    double* div = fab_alloc(obx, 1);
    oracle_divu(obx.lo, obx.hi, q, qbx.lo, qbx.hi, dx, div, obx.lo, obx.hi);

    double* q_int = fab_alloc(obx, QVAR);
    double* ftmp1 = fab_alloc(obx, NVAR);
    double* ftmp2 = fab_alloc(obx, NVAR);
    double* qg1 = fab_alloc(obx, NGDNV);
    double* qg2 = fab_alloc(obx, NGDNV);
    double* ql = fab_alloc(obx, QVAR);
    double* qr = fab_alloc(obx, QVAR);

    double hdtdx[3], cdtdx[3];
    for (int d = 0; d < 3; ++d) { hdtdx[d] = 0.5 * dt / dx[d]; cdtdx[d] = dt / dx[d] / 3.0; }

    for (int d = 0; d < 3; ++d)
        oracle_trace_ppm(obx.lo, obx.hi, bx.lo, bx.hi, d + 1, q, qbx.lo, qbx.hi, qaux, qbx.lo, qbx.hi,
                         qm[d][d], tbx[d][d].lo, tbx[d][d].hi, qp[d][d], tbx[d][d].lo, tbx[d][d].hi,
                         domlo, domhi, dx, dt);

    for (int d = 0; d < 3; ++d) {
        int t1 = (d == 0) ? 1 : 0;
        int t2 = (d == 2) ? 1 : 2;
        box_t b = tbx[d][d];
        oracle_compute_flux(b.lo, b.hi, qm[d][d], b.lo, b.hi, qp[d][d], b.lo, b.hi,
                            ftmp1, obx.lo, obx.hi, q_int, obx.lo, obx.hi, qg1, obx.lo, obx.hi,
                            qaux, qbx.lo, qbx.hi, d + 1);
        box_t b1 = tbx[t1][d];
        oracle_trans1(b1.lo, b1.hi, d + 1, t1 + 1,
                      qm[t1][t1], tbx[t1][t1].lo, tbx[t1][t1].hi, qm[t1][d], b1.lo, b1.hi,
                      qp[t1][t1], tbx[t1][t1].lo, tbx[t1][t1].hi, qp[t1][d], b1.lo, b1.hi,
                      qaux, qbx.lo, qbx.hi, ftmp1, obx.lo, obx.hi, qg1, obx.lo, obx.hi, cdtdx[d]);
        box_t b2 = tbx[t2][d];
        oracle_trans1(b2.lo, b2.hi, d + 1, t2 + 1,
                      qm[t2][t2], tbx[t2][t2].lo, tbx[t2][t2].hi, qm[t2][d], b2.lo, b2.hi,
                      qp[t2][t2], tbx[t2][t2].lo, tbx[t2][t2].hi, qp[t2][d], b2.lo, b2.hi,
                      qaux, qbx.lo, qbx.hi, ftmp1, obx.lo, obx.hi, qg1, obx.lo, obx.hi, cdtdx[d]);
    }

    for (int d = 0; d < 3; ++d) {
        int t1 = (d == 0) ? 1 : 0;
        int t2 = (d == 2) ? 1 : 2;
        box_t b = tbx[t1][t2];
        oracle_compute_flux(b.lo, b.hi, qm[t1][t2], b.lo, b.hi, qp[t1][t2], b.lo, b.hi,
                            ftmp1, obx.lo, obx.hi, q_int, obx.lo, obx.hi, qg1, obx.lo, obx.hi,
                            qaux, qbx.lo, qbx.hi, t1 + 1);
        b = tbx[t2][t1];
        oracle_compute_flux(b.lo, b.hi, qm[t2][t1], b.lo, b.hi, qp[t2][t1], b.lo, b.hi,
                            ftmp2, obx.lo, obx.hi, q_int, obx.lo, obx.hi, qg2, obx.lo, obx.hi,
                            qaux, qbx.lo, qbx.hi, t2 + 1);
        b = ebx[d];
        oracle_trans2(b.lo, b.hi, d + 1, t1 + 1, t2 + 1,
                      qm[d][d], tbx[d][d].lo, tbx[d][d].hi, ql, obx.lo, obx.hi,
                      qp[d][d], tbx[d][d].lo, tbx[d][d].hi, qr, obx.lo, obx.hi,
                      qaux, qbx.lo, qbx.hi, ftmp1, obx.lo, obx.hi, ftmp2, obx.lo, obx.hi,
                      qg1, obx.lo, obx.hi, qg2, obx.lo, obx.hi, hdtdx[d], hdtdx[t1], hdtdx[t2]);
        oracle_compute_flux(b.lo, b.hi, ql, obx.lo, obx.hi, qr, obx.lo, obx.hi,
                            flux[d], gebx[d].lo, gebx[d].hi, q_int, obx.lo, obx.hi, qe[d], gebx[d].lo, gebx[d].hi,
                            qaux, qbx.lo, qbx.hi, d + 1);
    }

    for (int d = 0; d < 3; ++d) {
        oracle_apply_av(ebx[d].lo, ebx[d].hi, d + 1, dx, div, obx.lo, obx.hi, sb, sb_lo, sb_hi,
                        flux[d], gebx[d].lo, gebx[d].hi);
        oracle_normalize_species_fluxes(ebx[d].lo, ebx[d].hi, flux[d], gebx[d].lo, gebx[d].hi);
    }

    /* Cartesian geometry: face areas and cell volume (AMReX GetFaceArea/GetVolume) */
    double area[3] = {dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1]};
    double volume = dx[0] * dx[1] * dx[2];
    double* ar[3];
    for (int d = 0; d < 3; ++d) {
        long n = box_npts(gebx[d]);
        ar[d] = (double*)malloc(sizeof(double) * (size_t)n);
        for (long m = 0; m < n; ++m) ar[d][m] = area[d];
    }
    long nv = box_npts(bx);
    double* vol = (double*)malloc(sizeof(double) * (size_t)nv);
    for (long m = 0; m < nv; ++m) vol[m] = volume;

    oracle_fill_hydro_source(bx.lo, bx.hi, sb, sb_lo, sb_hi, q, qbx.lo, qbx.hi, src, s_lo, s_hi,
                             flux[0], gebx[0].lo, gebx[0].hi, flux[1], gebx[1].lo, gebx[1].hi,
                             flux[2], gebx[2].lo, gebx[2].hi,
                             qe[0], gebx[0].lo, gebx[0].hi, qe[1], gebx[1].lo, gebx[1].hi,
                             qe[2], gebx[2].lo, gebx[2].hi,
                             ar[0], gebx[0].lo, gebx[0].hi, ar[1], gebx[1].lo, gebx[1].hi,
                             ar[2], gebx[2].lo, gebx[2].hi, vol, bx.lo, bx.hi, dx, dt);

    free(vol);
    for (int d = 0; d < 3; ++d) { free(ar[d]); free(flux[d]); free(qe[d]); }
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) { free(qm[a][b]); free(qp[a][b]); }
    free(div); free(q_int); free(ftmp1); free(ftmp2); free(qg1); free(qg2); free(ql); free(qr);
    free(q); free(qaux);
}

/* ------------------------------------------------------------------------ */
/* Single-level driver: Castro::advance (Source/Castro_advance.cpp:12-100),   */
/* clean_state (Source/Castro.cpp:546-593), estTimeStep (:175-216),          */
/* computeInitialDt/computeNewDt (:218-341), post_timestep (:343-426).       */
/* ------------------------------------------------------------------------ */
struct oracle_level {
    int nbox;
    box_t* boxes;
    double** U;            /* valid FAB per box */
    box_t dom;
    double problo[3], probhi[3], dx[3];
    int bc;
    int nthreads;
    double time, dt;
    int steps;
};

oracle_level* oracle_level_create(int nbox, const int* box_lo, const int* box_hi,
                                  const int* dom_lo, const int* dom_hi,
                                  const double* problo, const double* probhi, int bc)
{
    oracle_level* L = (oracle_level*)calloc(1, sizeof(oracle_level));
    L->nbox = nbox;
    L->boxes = (box_t*)malloc(sizeof(box_t) * (size_t)nbox);
    L->U = (double**)malloc(sizeof(double*) * (size_t)nbox);
    for (int b = 0; b < nbox; ++b) {
        for (int d = 0; d < 3; ++d) { L->boxes[b].lo[d] = box_lo[3 * b + d]; L->boxes[b].hi[d] = box_hi[3 * b + d]; }
        L->U[b] = (double*)calloc((size_t)box_npts(L->boxes[b]) * NVAR, sizeof(double));
    }
    for (int d = 0; d < 3; ++d) {
        L->dom.lo[d] = dom_lo[d]; L->dom.hi[d] = dom_hi[d];
        L->problo[d] = problo[d]; L->probhi[d] = probhi[d];
        L->dx[d] = (probhi[d] - problo[d]) / (double)(dom_hi[d] - dom_lo[d] + 1);
    }
    L->bc = bc;
    L->nthreads = 0;
    L->time = 0.0; L->dt = 0.0; L->steps = 0;
    return L;
}

void oracle_level_destroy(oracle_level* L)
{
    if (!L) return;
    for (int b = 0; b < L->nbox; ++b) free(L->U[b]);
    free(L->U); free(L->boxes); free(L);
}

double* oracle_level_state(oracle_level* L, int ibox) { return L->U[ibox]; }
int oracle_level_nbox(const oracle_level* L) { return L->nbox; }
void oracle_level_set_threads(oracle_level* L, int n) { L->nthreads = n; }
double oracle_level_time(const oracle_level* L) { return L->time; }
double oracle_level_dt(const oracle_level* L) { return L->dt; }
int oracle_level_steps(const oracle_level* L) { return L->steps; }

/* MFIter tiling with tile size (1024,16,16) (Source/Castro.cpp:26) */
typedef struct { int box; box_t t; } tile_t;

static int make_tiles(const oracle_level* L, tile_t** out)
{
    const int ts[3] = {1024, 16, 16};
    int cap = 64, n = 0;
    tile_t* tl = (tile_t*)malloc(sizeof(tile_t) * (size_t)cap);
    for (int b = 0; b < L->nbox; ++b) {
        box_t bx = L->boxes[b];
        int nt[3], len[3];
        for (int d = 0; d < 3; ++d) {
            len[d] = bx.hi[d] - bx.lo[d] + 1;
            nt[d] = len[d] / ts[d];
            if (nt[d] < 1) nt[d] = 1;
        }
        for (int tk = 0; tk < nt[2]; ++tk)
            for (int tj = 0; tj < nt[1]; ++tj)
                for (int ti = 0; ti < nt[0]; ++ti) {
                    int tix[3] = {ti, tj, tk};
                    tile_t t; t.box = b;
                    for (int d = 0; d < 3; ++d) {
                        int base = len[d] / nt[d], rem = len[d] % nt[d];
                        int start = bx.lo[d] + tix[d] * base + (tix[d] < rem ? tix[d] : rem);
                        int size = base + (tix[d] < rem ? 1 : 0);
                        t.t.lo[d] = start; t.t.hi[d] = start + size - 1;
                    }
                    if (n == cap) { cap *= 2; tl = (tile_t*)realloc(tl, sizeof(tile_t) * (size_t)cap); }
                    tl[n++] = t;
                }
    }
    *out = tl;
    return n;
}

static void set_threads(const oracle_level* L)
{
#ifdef _OPENMP
    if (L->nthreads > 0) omp_set_num_threads(L->nthreads);
#else
    (void)L;
#endif
}

void oracle_level_init_data(oracle_level* L)
{
    set_threads(L);
    tile_t* tl; int nt = make_tiles(L, &tl);
    #pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < nt; ++m) {
        box_t b = L->boxes[tl[m].box];
        oracle_initdata(tl[m].t.lo, tl[m].t.hi, L->U[tl[m].box], b.lo, b.hi, L->dx, L->problo, L->probhi);
    }
    free(tl);
}

/* clean_state on FABs; 'grown' selects growntilebox(ng) for Sborder */
static void clean_fab(const int* lo, const int* hi, double* u, const int* u_lo, const int* u_hi)
{
    oracle_enforce_minimum_density(lo, hi, u, u_lo, u_hi);
    oracle_normalize_species(lo, hi, u, u_lo, u_hi);
    oracle_reset_internal_e(lo, hi, u, u_lo, u_hi);
    oracle_compute_temp(lo, hi, u, u_lo, u_hi);
}

void oracle_level_clean_state(oracle_level* L)
{
    set_threads(L);
    tile_t* tl; int nt = make_tiles(L, &tl);
    #pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < nt; ++m) {
        box_t b = L->boxes[tl[m].box];
        clean_fab(tl[m].t.lo, tl[m].t.hi, L->U[tl[m].box], b.lo, b.hi);
    }
    free(tl);
}

double oracle_level_est_time_step(oracle_level* L)
{
    set_threads(L);
    tile_t* tl; int nt = make_tiles(L, &tl);
    double dt = DBL_MAX;
    #pragma omp parallel for schedule(dynamic) reduction(min:dt)
    for (int m = 0; m < nt; ++m) {
        box_t b = L->boxes[tl[m].box];
        double dtl = DBL_MAX;
        oracle_estdt(tl[m].t.lo, tl[m].t.hi, L->U[tl[m].box], b.lo, b.hi, L->dx, &dtl);
        if (dtl < dt) dt = dtl;
    }
    free(tl);
    dt *= cfl;
    return dt;
}

/* domain-index -> valid index under the level's boundary condition */
static inline int map_index(int i, int lo, int hi, int bc)
{
    int n = hi - lo + 1;
    if (bc == 0) {
        int r = (i - lo) % n;
        if (r < 0) r += n;
        return lo + r;
    }
    return i < lo ? lo : (i > hi ? hi : i);
}

/* FillPatch of Sborder (4 ghosts) from the valid data of every box */
static void fill_patch(const oracle_level* L, double* const* sb, int ng, double* const* U)
{
    box_t dom = L->dom;
    long dnx = dom.hi[0] - dom.lo[0] + 1, dny = dom.hi[1] - dom.lo[1] + 1, dnz = dom.hi[2] - dom.lo[2] + 1;
    /* owner map: for each domain cell, (box, offset) */
    int* owner = (int*)malloc(sizeof(int) * (size_t)(dnx * dny * dnz));
    for (int b = 0; b < L->nbox; ++b) {
        box_t bx = L->boxes[b];
        for (int k = bx.lo[2]; k <= bx.hi[2]; ++k)
            for (int j = bx.lo[1]; j <= bx.hi[1]; ++j)
                for (int i = bx.lo[0]; i <= bx.hi[0]; ++i)
                    owner[(i - dom.lo[0]) + dnx * ((j - dom.lo[1]) + dny * (long)(k - dom.lo[2]))] = b;
    }
    #pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < L->nbox; ++b) {
        box_t bx = L->boxes[b];
        box_t g = grow_box(bx, ng, ng, ng);
        fab_t s = mkfab(sb[b], g.lo, g.hi);
        for (int n = 0; n < NVAR; ++n)
            for (int k = g.lo[2]; k <= g.hi[2]; ++k)
                for (int j = g.lo[1]; j <= g.hi[1]; ++j)
                    for (int i = g.lo[0]; i <= g.hi[0]; ++i) {
                        int ii = map_index(i, dom.lo[0], dom.hi[0], L->bc);
                        int jj = map_index(j, dom.lo[1], dom.hi[1], L->bc);
                        int kk = map_index(k, dom.lo[2], dom.hi[2], L->bc);
                        int ob = owner[(ii - dom.lo[0]) + dnx * ((jj - dom.lo[1]) + dny * (long)(kk - dom.lo[2]))];
                        fab_t u = mkfab(U[ob], L->boxes[ob].lo, L->boxes[ob].hi);
                        AT(s, i, j, k, n) = AT(u, ii, jj, kk, n);
                    }
    }
    free(owner);
}

void oracle_level_advance(oracle_level* L, double dt)
{
    set_threads(L);
    const int ng = 4;
    /* clean_state(S_old), Source/Castro_advance.cpp:51 */
    oracle_level_clean_state(L);
    /* S_new = S_old (:55) is implicit: L->U is updated in place at the end */
    double** sb = (double**)malloc(sizeof(double*) * (size_t)L->nbox);
    double** src = (double**)malloc(sizeof(double*) * (size_t)L->nbox);
    for (int b = 0; b < L->nbox; ++b) {
        box_t g = grow_box(L->boxes[b], ng, ng, ng);
        sb[b] = (double*)malloc(sizeof(double) * (size_t)(box_npts(g) * NVAR));
        src[b] = (double*)calloc((size_t)(box_npts(L->boxes[b]) * NVAR), sizeof(double));   /* setVal(0) */
    }
    /* FillPatch (:62) and clean_state(Sborder) over growntilebox(4) (:66) */
    fill_patch(L, sb, ng, L->U);
    tile_t* tl; int nt = make_tiles(L, &tl);
    #pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < nt; ++m) {
        box_t b = L->boxes[tl[m].box];
        box_t g = grow_box(b, ng, ng, ng);
        /* growntilebox: a tile grows into the ghost region only on the box faces it touches */
        box_t t = tl[m].t;
        for (int d = 0; d < 3; ++d) {
            if (t.lo[d] == b.lo[d]) t.lo[d] -= ng;
            if (t.hi[d] == b.hi[d]) t.hi[d] += ng;
        }
        clean_fab(t.lo, t.hi, sb[tl[m].box], g.lo, g.hi);
    }
    /* construct_hydro_source (:70) */
    #pragma omp parallel for schedule(dynamic)
    for (int m = 0; m < nt; ++m) {
        box_t b = L->boxes[tl[m].box];
        box_t g = grow_box(b, ng, ng, ng);
        oracle_construct_hydro_source_tile(tl[m].t.lo, tl[m].t.hi, sb[tl[m].box], g.lo, g.hi,
                                           src[tl[m].box], b.lo, b.hi, L->dom.lo, L->dom.hi, L->dx, dt);
    }
    free(tl);
    /* Saxpy(S_new, dt, hydro_source) (:74) */
    #pragma omp parallel for schedule(dynamic)
    for (int b = 0; b < L->nbox; ++b) {
        long n = box_npts(L->boxes[b]) * NVAR;
        double* u = L->U[b];
        const double* s = src[b];
        for (long m = 0; m < n; ++m) u[m] += dt * s[m];
    }
    for (int b = 0; b < L->nbox; ++b) { free(sb[b]); free(src[b]); }
    free(sb); free(src);
    /* clean_state(S_new) (:78) */
    oracle_level_clean_state(L);
}

double oracle_level_coarse_step(oracle_level* L, double stop_time)
{
    double dt_0;
    if (L->steps == 0) {
        /* computeInitialDt, Source/Castro.cpp:298-341; initialTimeStep :162-173 */
        dt_0 = 0.01 * oracle_level_est_time_step(L);
    } else {
        /* computeNewDt, Source/Castro.cpp:219-295 */
        double change_max = 1.1e0;
        double dt_min = oracle_level_est_time_step(L);
        dt_min = fmn(dt_min, change_max * L->dt);
        dt_0 = fmn(1.0e+100, dt_min);
    }
    double eps = 0.001 * dt_0;
    if (stop_time >= 0.0) {
        if ((L->time + dt_0) > (stop_time - eps)) dt_0 = stop_time - L->time;
    }
    L->dt = dt_0;
    oracle_level_advance(L, dt_0);
    /* post_timestep: clean_state(S_new), Source/Castro.cpp:369 */
    oracle_level_clean_state(L);
    L->time += dt_0;
    L->steps += 1;
    return dt_0;
}

double oracle_level_blast_radius(oracle_level* L, double* blast_mass_out)
{
    double max_density = -DBL_MAX;
    for (int b = 0; b < L->nbox; ++b) {
        long n = box_npts(L->boxes[b]);
        for (long m = 0; m < n; ++m) if (L->U[b][m] > max_density) max_density = L->U[b][m];
    }
    double bm = 0.0, br = 0.0;
    for (int b = 0; b < L->nbox; ++b)
        oracle_calculate_blast_radius(L->boxes[b].lo, L->boxes[b].hi, L->U[b], L->boxes[b].lo, L->boxes[b].hi,
                                      L->dx, L->problo, L->probhi, &bm, &br, max_density);
    if (blast_mass_out) *blast_mass_out = bm;
    return br / bm;
}
