/*
 * Operation-counting build of the oracle restatement (TEST/BENCH
 * INFRASTRUCTURE ONLY: it instruments the checker to count the arithmetic of
 * one cell-update; nothing here is shipped).
 *
 * oracle/src/cb_oracle.c is compiled as C++ with this header forced in front
 * and `double` defined as `cdbl`, a standard-layout wrapper of one double
 * (same size and alignment), so the counting library keeps the restatement's
 * C-ABI and array layout.  Every floating-point operation on a cdbl bumps a
 * counter of its kind; the arithmetic itself is unchanged IEEE double.
 */
#pragma once
#undef double
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

extern "C" {
/* counters: add/sub, mul, div, sqrt, pow and other transcendentals, compare, fabs/min/max */
enum { CNT_ADD = 0, CNT_MUL, CNT_DIV, CNT_SQRT, CNT_POW, CNT_CMP, CNT_ABS, CNT_N };
extern long long cbo_cnt[CNT_N];
void cbo_count_reset(void);
void cbo_count_read(long long *out);
}

struct cdbl {
  double v;
  cdbl() = default;
  constexpr cdbl(double x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  explicit operator long long() const { return (long long)v; }
  explicit operator unsigned char() const { return (unsigned char)v; }
  cdbl operator-() const { return cdbl(-v); }
  cdbl operator+() const { return *this; }
  cdbl &operator+=(cdbl o) { cbo_cnt[CNT_ADD]++; v += o.v; return *this; }
  cdbl &operator-=(cdbl o) { cbo_cnt[CNT_ADD]++; v -= o.v; return *this; }
  cdbl &operator*=(cdbl o) { cbo_cnt[CNT_MUL]++; v *= o.v; return *this; }
  cdbl &operator/=(cdbl o) { cbo_cnt[CNT_DIV]++; v /= o.v; return *this; }
};
static_assert(sizeof(cdbl) == sizeof(double) && alignof(cdbl) == alignof(double), "layout of the counted double");

inline cdbl operator+(cdbl a, cdbl b) { cbo_cnt[CNT_ADD]++; return cdbl(a.v + b.v); }
inline cdbl operator-(cdbl a, cdbl b) { cbo_cnt[CNT_ADD]++; return cdbl(a.v - b.v); }
inline cdbl operator*(cdbl a, cdbl b) { cbo_cnt[CNT_MUL]++; return cdbl(a.v * b.v); }
inline cdbl operator/(cdbl a, cdbl b) { cbo_cnt[CNT_DIV]++; return cdbl(a.v / b.v); }
inline bool operator<(cdbl a, cdbl b) { cbo_cnt[CNT_CMP]++; return a.v < b.v; }
inline bool operator>(cdbl a, cdbl b) { cbo_cnt[CNT_CMP]++; return a.v > b.v; }
inline bool operator<=(cdbl a, cdbl b) { cbo_cnt[CNT_CMP]++; return a.v <= b.v; }
inline bool operator>=(cdbl a, cdbl b) { cbo_cnt[CNT_CMP]++; return a.v >= b.v; }
inline bool operator==(cdbl a, cdbl b) { cbo_cnt[CNT_CMP]++; return a.v == b.v; }
inline bool operator!=(cdbl a, cdbl b) { cbo_cnt[CNT_CMP]++; return a.v != b.v; }
/* int operands (loop-index arithmetic mixed with doubles) */
#define CBO_INT_OPS(T)                                                   \
  inline cdbl operator+(cdbl a, T b) { return a + cdbl((double)b); }    \
  inline cdbl operator+(T a, cdbl b) { return cdbl((double)a) + b; }    \
  inline cdbl operator-(cdbl a, T b) { return a - cdbl((double)b); }    \
  inline cdbl operator-(T a, cdbl b) { return cdbl((double)a) - b; }    \
  inline cdbl operator*(cdbl a, T b) { return a * cdbl((double)b); }    \
  inline cdbl operator*(T a, cdbl b) { return cdbl((double)a) * b; }    \
  inline cdbl operator/(cdbl a, T b) { return a / cdbl((double)b); }    \
  inline cdbl operator/(T a, cdbl b) { return cdbl((double)a) / b; }    \
  inline bool operator<(cdbl a, T b) { return a < cdbl((double)b); }    \
  inline bool operator>(cdbl a, T b) { return a > cdbl((double)b); }    \
  inline bool operator<=(cdbl a, T b) { return a <= cdbl((double)b); }  \
  inline bool operator>=(cdbl a, T b) { return a >= cdbl((double)b); }  \
  inline bool operator==(cdbl a, T b) { return a == cdbl((double)b); }  \
  inline bool operator!=(cdbl a, T b) { return a != cdbl((double)b); }  \
  inline bool operator<(T a, cdbl b) { return cdbl((double)a) < b; }    \
  inline bool operator>(T a, cdbl b) { return cdbl((double)a) > b; }
CBO_INT_OPS(double)
CBO_INT_OPS(int)
CBO_INT_OPS(long)
CBO_INT_OPS(long long)
#undef CBO_INT_OPS

inline cdbl sqrt(cdbl a) { cbo_cnt[CNT_SQRT]++; return cdbl(std::sqrt(a.v)); }
inline cdbl fabs(cdbl a) { cbo_cnt[CNT_ABS]++; return cdbl(std::fabs(a.v)); }
inline cdbl pow(cdbl a, cdbl b) { cbo_cnt[CNT_POW]++; return cdbl(std::pow(a.v, b.v)); }
inline cdbl pow(cdbl a, double b) { return pow(a, cdbl(b)); }
inline cdbl pow(double a, cdbl b) { return pow(cdbl(a), b); }
inline cdbl tanh(cdbl a) { cbo_cnt[CNT_POW]++; return cdbl(std::tanh(a.v)); }
inline cdbl exp(cdbl a) { cbo_cnt[CNT_POW]++; return cdbl(std::exp(a.v)); }
inline cdbl sin(cdbl a) { cbo_cnt[CNT_POW]++; return cdbl(std::sin(a.v)); }
inline cdbl cos(cdbl a) { cbo_cnt[CNT_POW]++; return cdbl(std::cos(a.v)); }
inline cdbl log(cdbl a) { cbo_cnt[CNT_POW]++; return cdbl(std::log(a.v)); }
inline cdbl fmin(cdbl a, cdbl b) { cbo_cnt[CNT_ABS]++; return cdbl(std::fmin(a.v, b.v)); }
inline cdbl fmax(cdbl a, cdbl b) { cbo_cnt[CNT_ABS]++; return cdbl(std::fmax(a.v, b.v)); }
inline bool isfinite(cdbl a) { return std::isfinite(a.v); }
inline bool isnan(cdbl a) { return std::isnan(a.v); }
using std::sqrt;
using std::fabs;
using std::pow;
using std::tanh;
using std::sin;
using std::cos;
using std::exp;

#define double cdbl
