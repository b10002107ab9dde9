// castro_table.h -- host-side reader of helm_table.dat (Source/eos.F90:580-734)
// into the per-node packed layout the EOS kernels read.  Header-only plain
// C++, shared by the library's eos_init and by host-side checks.
#pragma once

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include "castro_device.cuh"

namespace castro {

struct HostTable {
    std::vector<double> node, trow, drow;
    EosTableDev consts;   // scalars filled, pointers left for the caller
};

// one list-directed READ of n values (starts a new record, may span records)
inline bool table_read_record(FILE* fp, double* v, int n)
{
    char line[4096];
    int got = 0;
    while (got < n) {
        if (!fgets(line, sizeof line, fp)) return false;
        for (char* c = line; *c; ++c)
            if (*c == 'D' || *c == 'd') *c = 'E';
        char* s = line;
        while (got < n) {
            while (*s == ',' || *s == ' ' || *s == '\t') ++s;
            if (*s == '\n' || *s == '\r' || *s == 0) break;   // the record continues on the next line
            char* e;
            double x = strtod(s, &e);
            if (e == s) return false;                            // not a number: a malformed table
            v[got++] = x;
            s = e;
        }
    }
    return true;
}

// 0 on success, 1 when the file cannot be opened, 2 when it is truncated or malformed
inline int read_helm_table(const char* path, HostTable& T)
{
    const int IM = IMAX, JM = JMAX;
    // grid and deltas, Source/eos.F90:62-71,626-632,700-712
    const double tlo = 3.0, thi = 13.0, dlo = -12.0, dhi = 15.0;
    const double tstp = (thi - tlo) / (double)(float)(JM - 1);
    const double dstp = (dhi - dlo) / (double)(float)(IM - 1);
    std::vector<double> t(JM), d(IM);
    for (int j = 0; j < JM; ++j) t[j] = pow(10.0, tlo + j * tstp);
    for (int i = 0; i < IM; ++i) d[i] = pow(10.0, dlo + i * dstp);

    FILE* fp = fopen(path, "r");
    if (!fp) return 1;
    // the 13 tables the hydro path reads, packed per node
    T.node.assign((size_t)JM * IM * NODE_STRIDE, 0.0);
    double v[9];
    bool ok = true;
    for (int j = 0; j < JM && ok; ++j)
        for (int i = 0; i < IM && ok; ++i) {
            if (!table_read_record(fp, v, 9)) { ok = false; break; }
            double* r = &T.node[((size_t)j * IM + i) * NODE_STRIDE];
            // file order f, fd, ft, fdd, ftt, fdt, fddt, fdtt, fddtt (eos.F90:646-647)
            r[N_F] = v[0]; r[N_FD] = v[1]; r[N_FT] = v[2]; r[N_FDD] = v[3]; r[N_FTT] = v[4];
            r[N_FDT] = v[5]; r[N_FDDT] = v[6]; r[N_FDTT] = v[7]; r[N_FDDTT] = v[8];
        }
    for (int j = 0; j < JM && ok; ++j)
        for (int i = 0; i < IM && ok; ++i) {
            if (!table_read_record(fp, v, 4)) { ok = false; break; }
            double* r = &T.node[((size_t)j * IM + i) * NODE_STRIDE];
            // dpdf, dpdfd, dpdft, dpdfdt (eos.F90:654)
            r[N_DPDF] = v[0]; r[N_DPDFD] = v[1]; r[N_DPDFT] = v[2]; r[N_DPDFDT] = v[3];
        }
    // the chemical-potential and number-density blocks (eos.F90:659-670) are
    // read for format validation only; no hydro quantity depends on them
    for (int b = 0; b < 2 && ok; ++b)
        for (int j = 0; j < JM && ok; ++j)
            for (int i = 0; i < IM && ok; ++i)
                if (!table_read_record(fp, v, 4)) ok = false;
    fclose(fp);
    if (!ok) return 2;
    T.trow.assign((size_t)JM * ROW_STRIDE, 0.0);
    T.drow.assign((size_t)IM * ROW_STRIDE, 0.0);
    for (int j = 0; j < JM; ++j) {
        double dt = (j < JM - 1) ? t[j + 1] - t[j] : 0.0;
        double dt2 = dt * dt;
        T.trow[(size_t)j * ROW_STRIDE + 0] = t[j];
        T.trow[(size_t)j * ROW_STRIDE + 1] = dt;
        T.trow[(size_t)j * ROW_STRIDE + 2] = dt2;
        T.trow[(size_t)j * ROW_STRIDE + 3] = (j < JM - 1) ? 1.0 / dt : 0.0;
        T.trow[(size_t)j * ROW_STRIDE + 4] = (j < JM - 1) ? 1.0 / dt2 : 0.0;
        T.trow[(size_t)j * ROW_STRIDE + ROW_NEXT] = (j < JM - 1) ? t[j + 1] : HUGE_VAL;
    }
    for (int i = 0; i < IM; ++i) {
        double dd = (i < IM - 1) ? d[i + 1] - d[i] : 0.0;
        double dd2 = dd * dd;
        T.drow[(size_t)i * ROW_STRIDE + 0] = d[i];
        T.drow[(size_t)i * ROW_STRIDE + 1] = dd;
        T.drow[(size_t)i * ROW_STRIDE + 2] = dd2;
        T.drow[(size_t)i * ROW_STRIDE + 3] = (i < IM - 1) ? 1.0 / dd : 0.0;
        T.drow[(size_t)i * ROW_STRIDE + 4] = (i < IM - 1) ? 1.0 / dd2 : 0.0;
        T.drow[(size_t)i * ROW_STRIDE + ROW_NEXT] = (i < IM - 1) ? d[i + 1] : HUGE_VAL;
    }
    // physical constants, Source/eos.F90:129-137
    const double h = 6.6260689633e-27, avo_eos = 6.0221417930e23, clight = 2.99792458e10;
    const double kerg = 1.380650424e-16, amu = 1.66053878283e-24;
    const double asol = 4.0 * 5.67051e-5 / clight;
    EosTableDev& c = T.consts;
    c.node = c.trow = c.drow = nullptr;
    c.tlo = tlo;
    c.dlo = dlo;
    c.tstpi = 1.0 / tstp;
    c.dstpi = 1.0 / dstp;
    c.mintemp = pow(10.0, tlo);
    c.asoli3 = asol / 3.0;
    c.kergavo = kerg * avo_eos;
    c.avo_eos = avo_eos;
    c.kerg = kerg;
    c.sioncon = (2.0 * M_PI * amu * kerg) / (h * h);
    c.fail_count = nullptr;
    return 0;
}

}  // namespace castro
