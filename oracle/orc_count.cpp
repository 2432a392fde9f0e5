/*
 * orc_count.cpp -- operation counts of the CPU oracle.
 *
 * TEST AND MEASUREMENT INFRASTRUCTURE ONLY: never linked into the product
 * library.  It compiles mgcm_rt_oracle.c unchanged as C++ with `double`
 * replaced by a number type that carries one double and counts the
 * floating-point operations done on it, so the counts are those of the
 * reference's own operation order (the oracle restates it line by line):
 *
 *   add   + and - (binary, compound forms included)
 *   mul   *
 *   div   /
 *   sqrt, exp, log (LOG10 and natural log), pow, erf   one each; the
 *         deterministic routines of include/mgcm_rt_math.h are counted as
 *         one operation, not by their internal steps
 *   gather  k-table reads of OPTCV/OPTCI (8 per level, band and Gauss point)
 *
 * Negation, fabs, fmin/fmax, comparisons and integer work are not counted.
 * The arithmetic is the oracle's (IEEE double, no contraction), so this
 * build's results equal liboracle.so's bit for bit.  Counters are global:
 * run the batch on one thread (orc_run_batch(..., 1)) between
 * orc_count_reset() and orc_count_read().
 */
#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "../include/mgcm_rt_math.h"

namespace orc_count {
enum { ADD, MUL, DIV, SQRT, EXP, LOG, POW, ERF, GATHER, NKIND };
static unsigned long long n[NKIND];
}  // namespace orc_count

struct cnum {
    double v;
    cnum() = default;
    constexpr cnum(double x) : v(x) {}
    explicit constexpr operator float() const { return (float)v; }
    explicit constexpr operator int() const { return (int)v; }
    explicit constexpr operator long() const { return (long)v; }
    cnum &operator+=(cnum o) { ++orc_count::n[orc_count::ADD]; v += o.v; return *this; }
    cnum &operator-=(cnum o) { ++orc_count::n[orc_count::ADD]; v -= o.v; return *this; }
    cnum &operator*=(cnum o) { ++orc_count::n[orc_count::MUL]; v *= o.v; return *this; }
    cnum &operator/=(cnum o) { ++orc_count::n[orc_count::DIV]; v /= o.v; return *this; }
};
static_assert(sizeof(cnum) == sizeof(double), "cnum must have the layout of a double");

static inline cnum operator+(cnum a, cnum b) { ++orc_count::n[orc_count::ADD]; return cnum(a.v + b.v); }
static inline cnum operator-(cnum a, cnum b) { ++orc_count::n[orc_count::ADD]; return cnum(a.v - b.v); }
static inline cnum operator*(cnum a, cnum b) { ++orc_count::n[orc_count::MUL]; return cnum(a.v * b.v); }
static inline cnum operator/(cnum a, cnum b) { ++orc_count::n[orc_count::DIV]; return cnum(a.v / b.v); }
static inline cnum operator-(cnum a) { return cnum(-a.v); }
static inline cnum operator+(cnum a) { return a; }
static inline bool operator<(cnum a, cnum b) { return a.v < b.v; }
static inline bool operator>(cnum a, cnum b) { return a.v > b.v; }
static inline bool operator<=(cnum a, cnum b) { return a.v <= b.v; }
static inline bool operator>=(cnum a, cnum b) { return a.v >= b.v; }
static inline bool operator==(cnum a, cnum b) { return a.v == b.v; }
static inline bool operator!=(cnum a, cnum b) { return a.v != b.v; }

static inline cnum fabs(cnum a) { return cnum(::fabs(a.v)); }
static inline cnum fmin(cnum a, cnum b) { return cnum(::fmin(a.v, b.v)); }
static inline cnum fmax(cnum a, cnum b) { return cnum(::fmax(a.v, b.v)); }
static inline cnum sqrt(cnum a) { ++orc_count::n[orc_count::SQRT]; return cnum(::sqrt(a.v)); }
static inline cnum exp(cnum a) { ++orc_count::n[orc_count::EXP]; return cnum(::exp(a.v)); }
static inline cnum log(cnum a) { ++orc_count::n[orc_count::LOG]; return cnum(::log(a.v)); }
static inline cnum log10(cnum a) { ++orc_count::n[orc_count::LOG]; return cnum(::log10(a.v)); }
static inline cnum pow(cnum a, cnum b) { ++orc_count::n[orc_count::POW]; return cnum(::pow(a.v, b.v)); }
static inline cnum mgcm_rt_exp(cnum a) { ++orc_count::n[orc_count::EXP]; return cnum(mgcm_rt_exp(a.v)); }
static inline cnum mgcm_rt_log10(cnum a) { ++orc_count::n[orc_count::LOG]; return cnum(mgcm_rt_log10(a.v)); }
static inline cnum mgcm_rt_ln(cnum a) { ++orc_count::n[orc_count::LOG]; return cnum(mgcm_rt_ln(a.v)); }
static inline cnum mgcm_rt_pow(cnum a, cnum b) {
    ++orc_count::n[orc_count::POW];
    return cnum(mgcm_rt_pow(a.v, b.v));
}
static inline cnum mgcm_rt_erf(cnum a) { ++orc_count::n[orc_count::ERF]; return cnum(mgcm_rt_erf(a.v)); }

#define ORC_GATHERS(k) (orc_count::n[orc_count::GATHER] += (k))
#define double cnum
#include "mgcm_rt_oracle.c"
#undef double

extern "C" {
void orc_count_reset(void) { memset(orc_count::n, 0, sizeof orc_count::n); }
/* add, mul, div, sqrt, exp, log, pow, erf, gather */
void orc_count_read(unsigned long long *out) { memcpy(out, orc_count::n, sizeof orc_count::n); }
int orc_count_kinds(void) { return orc_count::NKIND; }
}
