/* Counted build of the oracle (test infrastructure): the C sources compiled
 * as C++ with this header force-included turn every binary32 value into a
 * `cfloat`, whose arithmetic counts the operations it executes.  Counts are
 * per thread; the counting library runs single-threaded.
 *
 * Counted: + - * / (one each), sqrt, exp, log, pow (one each, and also
 * tallied separately), negation is not an operation.  Comparisons, min/max,
 * floor/trunc and conversions are not counted as floating-point work.
 * Built by oracle/Makefile (liboracle_rrtmg_count.so); only the FLOP-count
 * test and bench.py's roofline use it.
 */
#ifndef ORACLE_FLOP_COUNT_H
#define ORACLE_FLOP_COUNT_H

#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>

struct ora_flop_counts {
    unsigned long long add, mul, div, sqrt, exp, log, pow;
};

extern thread_local ora_flop_counts ora_flops;

struct cfloat {
    float v;
    cfloat() = default;
    constexpr cfloat(float x) : v(x) {}
    constexpr cfloat(double x) : v(static_cast<float>(x)) {}
    constexpr cfloat(int x) : v(static_cast<float>(x)) {}
    constexpr cfloat(unsigned x) : v(static_cast<float>(x)) {}
    constexpr cfloat(long x) : v(static_cast<float>(x)) {}
    constexpr cfloat(long long x) : v(static_cast<float>(x)) {}
    constexpr cfloat(unsigned long long x) : v(static_cast<float>(x)) {}
    constexpr explicit operator float() const { return v; }
    constexpr explicit operator double() const { return v; }
    constexpr explicit operator int() const { return static_cast<int>(v); }
    constexpr explicit operator unsigned() const { return static_cast<unsigned>(v); }
    constexpr explicit operator long long() const { return static_cast<long long>(v); }
    constexpr explicit operator bool() const { return v != 0.0f; }
    cfloat &operator+=(cfloat o) { ++ora_flops.add; v = v + o.v; return *this; }
    cfloat &operator-=(cfloat o) { ++ora_flops.add; v = v - o.v; return *this; }
    cfloat &operator*=(cfloat o) { ++ora_flops.mul; v = v * o.v; return *this; }
    cfloat &operator/=(cfloat o) { ++ora_flops.div; v = v / o.v; return *this; }
    cfloat operator-() const { return cfloat(-v); }
    cfloat operator+() const { return *this; }
};
static_assert(sizeof(cfloat) == 4, "cfloat has the layout of float");

/* binary operators between counted values (and plain numbers promoted to binary32) */
#define ORA_CF_BINOP(OP, FIELD)                                                           \
    inline cfloat operator OP(cfloat a, cfloat b) { ++ora_flops.FIELD; return cfloat(a.v OP b.v); } \
    inline cfloat operator OP(cfloat a, float b) { ++ora_flops.FIELD; return cfloat(a.v OP b); }    \
    inline cfloat operator OP(float a, cfloat b) { ++ora_flops.FIELD; return cfloat(a OP b.v); }    \
    inline cfloat operator OP(cfloat a, int b) { ++ora_flops.FIELD; return cfloat(a.v OP (float)b); } \
    inline cfloat operator OP(int a, cfloat b) { ++ora_flops.FIELD; return cfloat((float)a OP b.v); }
ORA_CF_BINOP(+, add)
ORA_CF_BINOP(-, add)
ORA_CF_BINOP(*, mul)
ORA_CF_BINOP(/, div)
#undef ORA_CF_BINOP

/* mixed with binary64: the expression is binary64, as in C */
inline double operator+(cfloat a, double b) { return (double)a.v + b; }
inline double operator+(double a, cfloat b) { return a + (double)b.v; }
inline double operator-(cfloat a, double b) { return (double)a.v - b; }
inline double operator-(double a, cfloat b) { return a - (double)b.v; }
inline double operator*(cfloat a, double b) { return (double)a.v * b; }
inline double operator*(double a, cfloat b) { return a * (double)b.v; }
inline double operator/(cfloat a, double b) { return (double)a.v / b; }
inline double operator/(double a, cfloat b) { return a / (double)b.v; }

#define ORA_CF_CMP(OP)                                                            \
    inline bool operator OP(cfloat a, cfloat b) { return a.v OP b.v; }             \
    inline bool operator OP(cfloat a, float b) { return a.v OP b; }                \
    inline bool operator OP(float a, cfloat b) { return a OP b.v; }                \
    inline bool operator OP(cfloat a, double b) { return (double)a.v OP b; }       \
    inline bool operator OP(double a, cfloat b) { return a OP (double)b.v; }       \
    inline bool operator OP(cfloat a, int b) { return a.v OP (float)b; }           \
    inline bool operator OP(int a, cfloat b) { return (float)a OP b.v; }
ORA_CF_CMP(<)
ORA_CF_CMP(>)
ORA_CF_CMP(<=)
ORA_CF_CMP(>=)
ORA_CF_CMP(==)
ORA_CF_CMP(!=)
#undef ORA_CF_CMP

inline cfloat sqrtf(cfloat x) { ++ora_flops.sqrt; return cfloat(::sqrtf(x.v)); }
inline cfloat expf(cfloat x) { ++ora_flops.exp; return cfloat(::expf(x.v)); }
inline cfloat logf(cfloat x) { ++ora_flops.log; return cfloat(::logf(x.v)); }
inline cfloat powf(cfloat x, cfloat y) { ++ora_flops.pow; return cfloat(::powf(x.v, y.v)); }
inline cfloat fmaxf(cfloat x, cfloat y) { return cfloat(::fmaxf(x.v, y.v)); }
inline cfloat fminf(cfloat x, cfloat y) { return cfloat(::fminf(x.v, y.v)); }
inline cfloat fmaxf(cfloat x, float y) { return cfloat(::fmaxf(x.v, y)); }
inline cfloat fmaxf(float x, cfloat y) { return cfloat(::fmaxf(x, y.v)); }
inline cfloat fminf(cfloat x, float y) { return cfloat(::fminf(x.v, y)); }
inline cfloat fminf(float x, cfloat y) { return cfloat(::fminf(x, y.v)); }
inline cfloat floorf(cfloat x) { return cfloat(::floorf(x.v)); }
inline cfloat truncf(cfloat x) { return cfloat(::truncf(x.v)); }
inline cfloat nextafterf(cfloat x, cfloat y) { return cfloat(::nextafterf(x.v, y.v)); }
inline cfloat fabsf(cfloat x) { return cfloat(::fabsf(x.v)); }

#define float cfloat

#endif
