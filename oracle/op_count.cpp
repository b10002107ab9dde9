/*
 * op_count.cpp -- the oracle with every floating-point operation counted.
 *
 * TEST INFRASTRUCTURE ONLY (a measurement of the reference algorithm's
 * arithmetic; nothing in the product links it).  castro_oracle.c is compiled
 * unchanged as C++ with `double` replaced by CountedDouble, a one-member
 * struct whose operators do the same IEEE double operation and bump a
 * per-thread counter by class: add (and subtract), mul, div, sqrt,
 * transcendental (log, log10, exp, pow, cbrt), compare (<, >, ==, ... and so every
 * max/min), and sign operations (fabs, copysign).  Built with
 * -ffp-contract=off like the parity build, so a*b+c stays a multiply and an
 * add and the results are bit for bit the parity build's (the operators only
 * wrap the plain operations).  Literal-only expressions are folded by the
 * compiler and, like the reference's constants, not counted.
 *
 * Exports, besides every oracle_* entry point of castro_oracle.h (same
 * signatures and memory layout: CountedDouble is a standard-layout double):
 *   oracle_op_counts(unsigned long long out[7])  sums over all threads so far
 *   oracle_op_counts_reset()
 */
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>
#include <omp.h>

namespace opcount {
enum { ADD, MUL, DIV, SQRT, TRANSC, CMP, SIGN, NCLASS };

struct Slot {
    unsigned long long n[NCLASS] = {};
};

std::mutex g_mu;
std::vector<Slot*> g_slots;

inline Slot& slot()
{
    thread_local Slot* s = nullptr;
    if (!s) {
        s = new Slot();
        std::lock_guard<std::mutex> lk(g_mu);
        g_slots.push_back(s);
    }
    return *s;
}
inline void bump(int c) { ++slot().n[c]; }
}  // namespace opcount

struct CountedDouble {
    double v;
    CountedDouble() = default;
    constexpr CountedDouble(double x) : v(x) {}
    explicit operator int() const { return (int)v; }
    explicit operator long() const { return (long)v; }
    explicit operator float() const { return (float)v; }
    explicit operator double() const { return v; }

    CountedDouble& operator+=(CountedDouble b) { opcount::bump(opcount::ADD); v = v + b.v; return *this; }
    CountedDouble& operator-=(CountedDouble b) { opcount::bump(opcount::ADD); v = v - b.v; return *this; }
    CountedDouble& operator*=(CountedDouble b) { opcount::bump(opcount::MUL); v = v * b.v; return *this; }
    CountedDouble& operator/=(CountedDouble b) { opcount::bump(opcount::DIV); v = v / b.v; return *this; }
    CountedDouble operator-() const { return CountedDouble(-v); }
    CountedDouble operator+() const { return *this; }
};
static_assert(sizeof(CountedDouble) == sizeof(double), "CountedDouble must lay out as a double");

using CD = CountedDouble;
inline CD operator+(CD a, CD b) { opcount::bump(opcount::ADD); return CD(a.v + b.v); }
inline CD operator-(CD a, CD b) { opcount::bump(opcount::ADD); return CD(a.v - b.v); }
inline CD operator*(CD a, CD b) { opcount::bump(opcount::MUL); return CD(a.v * b.v); }
inline CD operator/(CD a, CD b) { opcount::bump(opcount::DIV); return CD(a.v / b.v); }
inline CD operator+(double a, CD b) { return CD(a) + b; }
inline CD operator-(double a, CD b) { return CD(a) - b; }
inline CD operator*(double a, CD b) { return CD(a) * b; }
inline CD operator/(double a, CD b) { return CD(a) / b; }
inline CD operator+(CD a, double b) { return a + CD(b); }
inline CD operator-(CD a, double b) { return a - CD(b); }
inline CD operator*(CD a, double b) { return a * CD(b); }
inline CD operator/(CD a, double b) { return a / CD(b); }

#define OPC_CMP(op)                                                                          \
    inline bool operator op(CD a, CD b) { opcount::bump(opcount::CMP); return a.v op b.v; }    \
    inline bool operator op(double a, CD b) { opcount::bump(opcount::CMP); return a op b.v; }  \
    inline bool operator op(CD a, double b) { opcount::bump(opcount::CMP); return a.v op b; }
OPC_CMP(<)
OPC_CMP(>)
OPC_CMP(<=)
OPC_CMP(>=)
OPC_CMP(==)
OPC_CMP(!=)
#undef OPC_CMP

inline CD sqrt(CD x) { opcount::bump(opcount::SQRT); return CD(std::sqrt(x.v)); }
inline CD log(CD x) { opcount::bump(opcount::TRANSC); return CD(std::log(x.v)); }
inline CD log10(CD x) { opcount::bump(opcount::TRANSC); return CD(std::log10(x.v)); }
inline CD exp(CD x) { opcount::bump(opcount::TRANSC); return CD(std::exp(x.v)); }
inline CD pow(CD x, CD y) { opcount::bump(opcount::TRANSC); return CD(std::pow(x.v, y.v)); }
inline CD pow(double x, CD y) { return pow(CD(x), y); }
inline CD pow(CD x, double y) { return pow(x, CD(y)); }
inline CD cbrt(CD x) { opcount::bump(opcount::TRANSC); return CD(std::cbrt(x.v)); }
inline CD fabs(CD x) { opcount::bump(opcount::SIGN); return CD(std::fabs(x.v)); }
inline CD copysign(CD x, CD y) { opcount::bump(opcount::SIGN); return CD(std::copysign(x.v, y.v)); }
inline CD copysign(double x, CD y) { return copysign(CD(x), y); }

// the level's dt is an OpenMP min-reduction; its combiner is bookkeeping, not counted
#pragma omp declare reduction(min : CountedDouble : omp_out = (omp_in.v < omp_out.v ? omp_in : omp_out)) \
    initializer(omp_priv = CountedDouble(DBL_MAX))

#define double CountedDouble
#include "castro_oracle.c"
#undef double

extern "C" void oracle_op_counts(unsigned long long* out)
{
    std::lock_guard<std::mutex> lk(opcount::g_mu);
    for (int c = 0; c < opcount::NCLASS; ++c) out[c] = 0;
    for (opcount::Slot* s : opcount::g_slots)
        for (int c = 0; c < opcount::NCLASS; ++c) out[c] += s->n[c];
}

extern "C" void oracle_op_counts_reset(void)
{
    std::lock_guard<std::mutex> lk(opcount::g_mu);
    for (opcount::Slot* s : opcount::g_slots)
        for (int c = 0; c < opcount::NCLASS; ++c) s->n[c] = 0;
}
