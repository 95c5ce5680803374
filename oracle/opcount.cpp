// opcount.cpp -- operation-counting build of the CPU restatement
// (oracle/mam4_oracle.c), for the algorithmic flop count of the step.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY (oracle/libmam4oracle_count.so,
// driven by oracle/count_flops.py). The restatement is compiled as C++ with
// its `real` type replaced by CountReal, a double that tallies every
// arithmetic operation it takes part in: + - * / count one each (the
// restatement has no fused multiply-add: it is compiled without
// contraction), each libm call (exp, log, pow, sqrt, cbrt, erfc, log10,
// hypot, atan2, sin, cos) counts as one "special"; fabs, fmax, fmin and
// round are tallied apart as min/max and comparisons as compares, neither
// counted as flops. The values computed are those of the plain build, so
// the counted path (branches, SOA sub-step counts) is the oracle's own.
// Single-threaded: the tally is one global.
#include <float.h>
#include <math.h>
#include <stddef.h>
#include <string.h>

struct OpTally {
  unsigned long long add, mul, div, special, minmax, cmp;
};
static OpTally g_tally;

struct CountReal {
  double v;
  CountReal() = default;
  constexpr CountReal(double x) : v(x) {}
  explicit operator double() const { return v; }
  explicit operator int() const { return (int)v; }
  explicit operator unsigned() const { return (unsigned)v; }
  explicit operator long long() const { return (long long)v; }
  CountReal operator-() const { return CountReal(-v); }
  CountReal operator+() const { return *this; }
  friend CountReal operator+(CountReal a, CountReal b) { ++g_tally.add; return CountReal(a.v + b.v); }
  friend CountReal operator-(CountReal a, CountReal b) { ++g_tally.add; return CountReal(a.v - b.v); }
  friend CountReal operator*(CountReal a, CountReal b) { ++g_tally.mul; return CountReal(a.v * b.v); }
  friend CountReal operator/(CountReal a, CountReal b) { ++g_tally.div; return CountReal(a.v / b.v); }
  CountReal &operator+=(CountReal b) { ++g_tally.add; v += b.v; return *this; }
  CountReal &operator-=(CountReal b) { ++g_tally.add; v -= b.v; return *this; }
  CountReal &operator*=(CountReal b) { ++g_tally.mul; v *= b.v; return *this; }
  CountReal &operator/=(CountReal b) { ++g_tally.div; v /= b.v; return *this; }
  friend bool operator<(CountReal a, CountReal b) { ++g_tally.cmp; return a.v < b.v; }
  friend bool operator>(CountReal a, CountReal b) { ++g_tally.cmp; return a.v > b.v; }
  friend bool operator<=(CountReal a, CountReal b) { ++g_tally.cmp; return a.v <= b.v; }
  friend bool operator>=(CountReal a, CountReal b) { ++g_tally.cmp; return a.v >= b.v; }
  friend bool operator==(CountReal a, CountReal b) { ++g_tally.cmp; return a.v == b.v; }
  friend bool operator!=(CountReal a, CountReal b) { ++g_tally.cmp; return a.v != b.v; }
};

#define COUNT_SPECIAL1(f)                \
  static inline CountReal f(CountReal a) { \
    ++g_tally.special;                   \
    return CountReal(::f(a.v));          \
  }
COUNT_SPECIAL1(exp)
COUNT_SPECIAL1(log)
COUNT_SPECIAL1(sqrt)
COUNT_SPECIAL1(cbrt)
COUNT_SPECIAL1(erfc)
COUNT_SPECIAL1(log10)
COUNT_SPECIAL1(sin)
COUNT_SPECIAL1(cos)
#undef COUNT_SPECIAL1
static inline CountReal pow(CountReal a, CountReal b) { ++g_tally.special; return CountReal(::pow(a.v, b.v)); }
static inline CountReal atan2(CountReal a, CountReal b) { ++g_tally.special; return CountReal(::atan2(a.v, b.v)); }
static inline CountReal hypot(CountReal a, CountReal b) { ++g_tally.special; return CountReal(::hypot(a.v, b.v)); }
static inline CountReal round(CountReal a) { ++g_tally.minmax; return CountReal(::round(a.v)); }
static inline CountReal fabs(CountReal a) { ++g_tally.minmax; return CountReal(::fabs(a.v)); }
static inline CountReal fmax(CountReal a, CountReal b) { ++g_tally.minmax; return CountReal(::fmax(a.v, b.v)); }
static inline CountReal fmin(CountReal a, CountReal b) { ++g_tally.minmax; return CountReal(::fmin(a.v, b.v)); }
static inline bool isnan(CountReal a) { return a.v != a.v; }

#define ORACLE_REAL CountReal
#include "mam4_oracle.c"

// tally since the last call: add, mul, div, special, minmax, cmp; resets it
extern "C" void mam4cnt_tally(unsigned long long *t) {
  t[0] = g_tally.add;
  t[1] = g_tally.mul;
  t[2] = g_tally.div;
  t[3] = g_tally.special;
  t[4] = g_tally.minmax;
  t[5] = g_tally.cmp;
  memset(&g_tally, 0, sizeof(g_tally));
}
