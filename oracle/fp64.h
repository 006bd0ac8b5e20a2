/* Binary64 build of the oracle (test infrastructure): the C sources compiled
 * as C++ with this header force-included turn every binary32 value into a
 * `dfloat`, which holds a binary64 value and does every operation in
 * binary64.  It is the "FP64 run of the reference path" that the GPU's
 * binary32 and FP64 modes are measured against:
 *
 *   - every arithmetic operation, glibc exp/log/pow/sqrt call and comparison
 *     of the restatement runs in binary64 (exp, log, pow, sqrt of binary64);
 *   - the tables are the same binary32 data, widened exactly at load time;
 *   - literal constants written as binary32 literals keep their binary32
 *     values (the reference's constants are binary32 too: JAX rounds a Python
 *     scalar to the array's float32 type), below 6e-8 relative from the
 *     decimal values;
 *   - the McICA random stream and its cloud decisions stay binary32
 *     (ora_binary32), so both runs sample the same subcolumns;
 *   - inputs and outputs are binary64 arrays (exact copies of the binary32
 *     inputs; outputs not rounded).
 *
 * Built by oracle/Makefile (liboracle_rrtmg_f64.so); only the FP64 error
 * tests and oracle/fp64_errors.py use it.
 */
#ifndef ORACLE_FP64_H
#define ORACLE_FP64_H

#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>

typedef float ora_binary32;
#define ORA_BINARY32_DEFINED 1
#define ORA_WIDE_TABLES 1

struct dfloat {
    double v;
    dfloat() = default;
    constexpr dfloat(double x) : v(x) {}
    constexpr dfloat(float x) : v(x) {}
    constexpr dfloat(int x) : v(x) {}
    constexpr dfloat(unsigned x) : v(x) {}
    constexpr dfloat(long x) : v(static_cast<double>(x)) {}
    constexpr dfloat(unsigned long x) : v(static_cast<double>(x)) {}
    constexpr dfloat(long long x) : v(static_cast<double>(x)) {}
    constexpr dfloat(unsigned long long x) : v(static_cast<double>(x)) {}
    constexpr explicit operator float() const { return static_cast<float>(v); }
    constexpr explicit operator double() const { return v; }
    constexpr explicit operator int() const { return static_cast<int>(v); }
    constexpr explicit operator unsigned() const { return static_cast<unsigned>(v); }
    constexpr explicit operator long long() const { return static_cast<long long>(v); }
    constexpr explicit operator unsigned char() const { return static_cast<unsigned char>(v); }
    constexpr explicit operator bool() const { return v != 0.0; }
    dfloat &operator+=(dfloat o) { v = v + o.v; return *this; }
    dfloat &operator-=(dfloat o) { v = v - o.v; return *this; }
    dfloat &operator*=(dfloat o) { v = v * o.v; return *this; }
    dfloat &operator/=(dfloat o) { v = v / o.v; return *this; }
    constexpr dfloat operator-() const { return dfloat(-v); }
    constexpr dfloat operator+() const { return *this; }
};
static_assert(sizeof(dfloat) == 8, "dfloat has the layout of double");

/* arithmetic and comparisons; plain numbers convert to dfloat implicitly */
inline dfloat operator+(dfloat a, dfloat b) { return dfloat(a.v + b.v); }
inline dfloat operator-(dfloat a, dfloat b) { return dfloat(a.v - b.v); }
inline dfloat operator*(dfloat a, dfloat b) { return dfloat(a.v * b.v); }
inline dfloat operator/(dfloat a, dfloat b) { return dfloat(a.v / b.v); }
inline bool operator<(dfloat a, dfloat b) { return a.v < b.v; }
inline bool operator>(dfloat a, dfloat b) { return a.v > b.v; }
inline bool operator<=(dfloat a, dfloat b) { return a.v <= b.v; }
inline bool operator>=(dfloat a, dfloat b) { return a.v >= b.v; }
inline bool operator==(dfloat a, dfloat b) { return a.v == b.v; }
inline bool operator!=(dfloat a, dfloat b) { return a.v != b.v; }

inline dfloat sqrtf(dfloat x) { return dfloat(::sqrt(x.v)); }
inline dfloat expf(dfloat x) { return dfloat(::exp(x.v)); }
inline dfloat logf(dfloat x) { return dfloat(::log(x.v)); }
inline dfloat powf(dfloat x, dfloat y) { return dfloat(::pow(x.v, y.v)); }
inline dfloat fmaxf(dfloat x, dfloat y) { return dfloat(::fmax(x.v, y.v)); }
inline dfloat fminf(dfloat x, dfloat y) { return dfloat(::fmin(x.v, y.v)); }
inline dfloat floorf(dfloat x) { return dfloat(::floor(x.v)); }
inline dfloat truncf(dfloat x) { return dfloat(::trunc(x.v)); }
inline dfloat fabsf(dfloat x) { return dfloat(::fabs(x.v)); }
inline dfloat nextafterf(dfloat x, dfloat y) { return dfloat(::nextafter(x.v, y.v)); }

#define float dfloat

#endif
