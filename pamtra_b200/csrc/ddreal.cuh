// Double-double real arithmetic (value = hi + lo, |lo| <= ulp(hi) / 2, about
// 32 significant digits) for the extended-precision T-matrix solve: the
// reference solves the EBCM system in REAL*16 (src/tmatrix_amplq.lp.f), and
// FP64 loses digits for large aspherical liquid drops while double-double
// reproduces the REAL*16 single-precision T-matrix (measured on the CPU).
//
// Host and device: every operation is IEEE double arithmetic plus fma, so the
// host build (tested against 50-digit arithmetic) and the device build give
// the same bits.  Published building blocks: Knuth's two-sum, the fma
// two-product, Dekker/Bailey double-double addition, multiplication and long
// division, Karp's square root; the elementary functions reduce the argument
// and sum their Taylor series in double-double (relative error about 1e-30
// for |x| < 1e3).
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define DDR_FN __host__ __device__ __forceinline__
#else
#define DDR_FN inline
#endif

namespace pb {

struct ddr {
  double hi, lo;
};

DDR_FN ddr ddr_of(double h) { return ddr{h, 0.0}; }
DDR_FN double ddr_to_double(ddr a) { return a.hi + a.lo; }

DDR_FN ddr ddr_two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  return ddr{s, (a - (s - bb)) + (b - bb)};
}
DDR_FN ddr ddr_quick_two_sum(double a, double b) {
  const double s = a + b;
  return ddr{s, b - (s - a)};
}
DDR_FN ddr ddr_two_prod(double a, double b) {
  const double p = a * b;
  return ddr{p, fma(a, b, -p)};
}
DDR_FN ddr operator+(ddr a, ddr b) {
  ddr s = ddr_two_sum(a.hi, b.hi);
  const ddr t = ddr_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = ddr_quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return ddr_quick_two_sum(s.hi, s.lo);
}
DDR_FN ddr operator-(ddr a) { return ddr{-a.hi, -a.lo}; }
DDR_FN ddr operator-(ddr a, ddr b) { return a + (-b); }
DDR_FN ddr operator*(ddr a, ddr b) {
  ddr p = ddr_two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return ddr_quick_two_sum(p.hi, p.lo);
}
DDR_FN ddr operator*(ddr a, double b) {
  ddr p = ddr_two_prod(a.hi, b);
  p.lo += a.lo * b;
  return ddr_quick_two_sum(p.hi, p.lo);
}
DDR_FN ddr operator/(ddr a, ddr b) {
  const double q1 = a.hi / b.hi;
  ddr r = a - b * q1;
  const double q2 = r.hi / b.hi;
  r = r - b * q2;
  const double q3 = r.hi / b.hi;
  return ddr_quick_two_sum(q1, q2) + ddr_of(q3);
}
DDR_FN bool operator<(ddr a, ddr b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }
DDR_FN bool operator>(ddr a, ddr b) { return b < a; }

DDR_FN ddr ddr_abs(ddr a) { return a.hi < 0.0 ? -a : a; }
DDR_FN ddr ddr_sqrt(ddr a) {
  if (a.hi <= 0.0) return ddr_of(0.0);
  const double x = 1.0 / sqrt(a.hi);
  const double ax = a.hi * x;
  const ddr d = a - ddr_two_prod(ax, ax);
  return ddr_two_sum(ax, d.hi * (x * 0.5));
}

// pi / 2 and ln 2 to double-double precision
DDR_FN ddr ddr_half_pi() { return ddr{1.5707963267948965580e+00, 6.1232339957367660359e-17}; }
DDR_FN ddr ddr_ln2() { return ddr{6.9314718055994528623e-01, 2.3190468138462995584e-17}; }

// exp: x = k ln 2 + r, r / 2^4 summed, squared back four times (each
// squaring doubles the relative error of the sum)
DDR_FN ddr ddr_exp(ddr x) {
  const ddr ln2 = ddr_ln2();
  const double k = floor(x.hi / ln2.hi + 0.5);
  ddr r = (x - ln2 * k) * (1.0 / 16.0);
  ddr term = r, sum = ddr_of(1.0) + r;
  for (int i = 2; i < 40; i++) {
    term = term * r / ddr_of((double)i);
    sum = sum + term;
    if (fabs(term.hi) < 1e-35 * fabs(sum.hi)) break;
  }
  for (int i = 0; i < 4; i++) sum = sum * sum;
  return ddr{ldexp(sum.hi, (int)k), ldexp(sum.lo, (int)k)};
}
// log: Newton on exp from the double estimate, y += a exp(-y) - 1
DDR_FN ddr ddr_log(ddr a) {
  ddr y = ddr_of(log(a.hi));
  for (int i = 0; i < 2; i++) y = y + a * ddr_exp(-y) - ddr_of(1.0);
  return y;
}
DDR_FN ddr ddr_pow(ddr x, ddr y) { return ddr_exp(y * ddr_log(x)); }
DDR_FN ddr ddr_sinh(ddr x) {
  if (fabs(x.hi) < 0.1) {
    const ddr x2 = x * x;
    ddr term = x, sum = x;
    for (int i = 1; i < 20; i++) {
      term = term * x2 / ddr_of((double)((2 * i) * (2 * i + 1)));
      sum = sum + term;
    }
    return sum;
  }
  const ddr e = ddr_exp(x);
  return (e - ddr_of(1.0) / e) * 0.5;
}
DDR_FN ddr ddr_cosh(ddr x) {
  const ddr e = ddr_exp(x);
  return (e + ddr_of(1.0) / e) * 0.5;
}
// sin and cos: x = j pi/2 + r, |r| <= pi/4, Taylor series of r
DDR_FN void ddr_sincos(ddr x, ddr& s, ddr& c) {
  const ddr hp = ddr_half_pi();
  const double j = floor(x.hi / hp.hi + 0.5);
  const ddr r = x - hp * j;
  const ddr r2 = r * r;
  ddr term = r, ss = r;
  for (int i = 1; i < 25; i++) {
    term = -(term * r2) / ddr_of((double)((2 * i) * (2 * i + 1)));
    ss = ss + term;
    if (fabs(term.hi) < 1e-34) break;
  }
  term = ddr_of(1.0);
  ddr cc = ddr_of(1.0);
  for (int i = 1; i < 25; i++) {
    term = -(term * r2) / ddr_of((double)((2 * i - 1) * (2 * i)));
    cc = cc + term;
    if (fabs(term.hi) < 1e-34) break;
  }
  const int q = ((int)fmod(j, 4.0) + 4) % 4;
  if (q == 0) { s = ss; c = cc; }
  else if (q == 1) { s = cc; c = -ss; }
  else if (q == 2) { s = -ss; c = -cc; }
  else { s = -cc; c = ss; }
}

}  // namespace pb
