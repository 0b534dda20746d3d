// Test infrastructure only: double-double arithmetic (a value is hi + lo
// with |lo| <= ulp(hi)/2, about 32 significant digits) for the double-double
// build of the T-matrix oracle's solve (tmatrix_oracle.cpp, -DTMO_DD).  It
// measures whether double-double suffices where the reference solves in
// REAL*16 and FP64 does not.
//
// The error-free transformations are the published ones (Knuth's two-sum,
// the FMA two-product; Dekker / Bailey double-double); the elementary
// functions are plain series with argument reduction, accurate to about
// 1e-30 relative on the arguments the solve uses (|x| < 1e3).
#pragma once
#include <cmath>

namespace ddm {

struct dd {
  double hi = 0.0, lo = 0.0;
  dd() = default;
  dd(double h) : hi(h), lo(0.0) {}
  dd(int v) : hi((double)v), lo(0.0) {}
  dd(double h, double l) : hi(h), lo(l) {}
  explicit operator double() const { return hi + lo; }
  explicit operator int() const { return (int)(hi + lo); }
};

static inline dd two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  return dd(s, (a - (s - bb)) + (b - bb));
}
static inline dd quick_two_sum(double a, double b) {
  const double s = a + b;
  return dd(s, b - (s - a));
}
static inline dd two_prod(double a, double b) {
  const double p = a * b;
  return dd(p, std::fma(a, b, -p));
}
static inline dd operator+(dd a, dd b) {
  dd s = two_sum(a.hi, b.hi), t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
static inline dd operator-(dd a) { return dd(-a.hi, -a.lo); }
static inline dd operator-(dd a, dd b) { return a + (-b); }
static inline dd operator*(dd a, dd b) {
  dd p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}
static inline dd operator/(dd a, dd b) {
  // long division: q1 + q2 + q3 with a remainder update each step
  const double q1 = a.hi / b.hi;
  dd r = a - b * dd(q1);
  const double q2 = r.hi / b.hi;
  r = r - b * dd(q2);
  const double q3 = r.hi / b.hi;
  dd q = quick_two_sum(q1, q2);
  return q + dd(q3);
}
static inline dd& operator+=(dd& a, dd b) { return a = a + b; }
static inline dd& operator-=(dd& a, dd b) { return a = a - b; }
static inline dd& operator*=(dd& a, dd b) { return a = a * b; }
static inline bool operator<(dd a, dd b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
static inline bool operator>(dd a, dd b) { return b < a; }
static inline bool operator<=(dd a, dd b) { return !(b < a); }
static inline bool operator>=(dd a, dd b) { return !(a < b); }
static inline bool operator==(dd a, dd b) { return a.hi == b.hi && a.lo == b.lo; }
static inline bool operator!=(dd a, dd b) { return !(a == b); }

static inline dd dd_abs(dd a) { return a.hi < 0.0 ? -a : a; }
static inline dd dd_sqrt(dd a) {
  if (a.hi <= 0.0) return dd(0.0);
  const double x = 1.0 / std::sqrt(a.hi);
  const double ax = a.hi * x;
  // one Newton step in double-double from the double estimate (Karp's trick)
  const dd d = a - two_prod(ax, ax);
  return two_sum(ax, d.hi * (x * 0.5));
}

// pi and ln 2 to double-double precision
static const dd DD_PI(3.141592653589793116e+00, 1.224646799147353207e-16);
static const dd DD_LN2(6.931471805599452862e-01, 2.319046813846299558e-17);

// exp by reduction x = k ln2 + r, |r| <= ln2/2, then r/2^10 and squaring back
static inline dd dd_exp(dd x) {
  const double k = std::floor(x.hi / DD_LN2.hi + 0.5);
  dd r = x - DD_LN2 * dd(k);
  r = r * dd(1.0 / 1024.0);
  dd term = r, sum = dd(1.0) + r;
  for (int i = 2; i < 30; i++) {
    term = term * r / dd((double)i);
    sum = sum + term;
    if (std::fabs(term.hi) < 1e-34 * std::fabs(sum.hi)) break;
  }
  for (int i = 0; i < 10; i++) sum = sum * sum;
  return dd(std::ldexp(sum.hi, (int)k), std::ldexp(sum.lo, (int)k));
}
// log by Newton on exp from the double estimate
static inline dd dd_log(dd a) {
  dd y = dd(std::log(a.hi));
  for (int i = 0; i < 2; i++) y = y + a * dd_exp(-y) - dd(1.0);
  return y;
}
static inline dd dd_pow(dd x, dd y) { return dd_exp(y * dd_log(x)); }
static inline dd dd_cosh(dd x) {
  const dd e = dd_exp(x);
  return (e + dd(1.0) / e) * dd(0.5);
}
static inline dd dd_sinh(dd x) {
  if (std::fabs(x.hi) < 0.1) {  // series, no cancellation
    dd x2 = x * x, term = x, sum = x;
    for (int i = 1; i < 20; i++) {
      term = term * x2 / dd((double)((2 * i) * (2 * i + 1)));
      sum = sum + term;
    }
    return sum;
  }
  const dd e = dd_exp(x);
  return (e - dd(1.0) / e) * dd(0.5);
}
// sin and cos of the reduced argument |r| <= pi/4 by their series
static inline void dd_sincos_red(dd r, dd& s, dd& c) {
  const dd r2 = r * r;
  dd term = r, ss = r;
  for (int i = 1; i < 25; i++) {
    term = -(term * r2) / dd((double)((2 * i) * (2 * i + 1)));
    ss = ss + term;
    if (std::fabs(term.hi) < 1e-34) break;
  }
  term = dd(1.0);
  dd cc = dd(1.0);
  for (int i = 1; i < 25; i++) {
    term = -(term * r2) / dd((double)((2 * i - 1) * (2 * i)));
    cc = cc + term;
    if (std::fabs(term.hi) < 1e-34) break;
  }
  s = ss;
  c = cc;
}
static inline void dd_sincos(dd x, dd& s, dd& c) {
  // x = j (pi/2) + r
  const dd half_pi = DD_PI * dd(0.5);
  const double j = std::floor(x.hi / half_pi.hi + 0.5);
  const dd r = x - half_pi * dd(j);
  dd sr, cr;
  dd_sincos_red(r, sr, cr);
  const int q = ((int)std::fmod(j, 4.0) + 4) % 4;
  switch (q) {
    case 0: s = sr; c = cr; break;
    case 1: s = cr; c = -sr; break;
    case 2: s = -sr; c = -cr; break;
    default: s = -cr; c = sr; break;
  }
}
static inline dd dd_cos(dd x) {
  dd s, c;
  dd_sincos(x, s, c);
  return c;
}
static inline dd dd_sin(dd x) {
  dd s, c;
  dd_sincos(x, s, c);
  return s;
}

}  // namespace ddm
