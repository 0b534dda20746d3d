// Test infrastructure only: CPU restatement ("oracle") of the reference's
// T-matrix scattering branch for spheroids (scat_name 'tmatrix').  Linked by
// nothing in the product; only tests/ and bench.py's CPU-baseline leg load it
// (through oracle.py).
//
// Reference: src/tmatrix.f90:14-444 (calc_tmatrix, calc_single_tmatrix) and
// the vendored extended-precision EBCM code src/tmatrix_amplq.lp.f
// (Mishchenko's T-matrix method for axially symmetric particles: tmatrix_amplq
// :276-600, AMPL :602-888, VIGAMPL :890-970, CONST :972-1023, QGAUSS
// :1025-1112, VARY :1114-1192, RSP1 :1194-1225, BESS/RJB/RYB/CJB :1342-1524,
// TMATR0 :1526-1763, TMATR :1765-2047, VIG :2049-2105, TT :2107-2153).
//
// Precision model, kept from the reference: the T-matrix is computed in
// quadruple precision (REAL*16, here __float128), the final T = -RgQ Q^-1
// product is accumulated in double, the T-matrix is stored in single
// precision (REAL*4 common /TMAT/) and the amplitude matrix is evaluated in
// double from those single-precision elements.  The normalisation factors
// that the reference forms with single-precision float() arithmetic (CONST's
// sqrt(float(2n+1)/float(n(n+1))), VIG's sqrt(float(2i-1)/float(2i))) are
// reproduced with sqrtf on floats.
//
// Parity status: no golden vectors for this branch exist in the reference's
// test-suite; the oracle is pinned by the sphere limit (aspect ratio 1
// reproduces the Mie restatement's extinction and backscatter, which is pinned
// to the reference's golden fixture).
#if defined(TMO_DD)
#include "dd.h"
#elif !defined(TMO_DOUBLE)
#include <quadmath.h>
#endif

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle_common.h"

// Built twice: as the oracle (REAL*16 like the reference) and, with
// -DTMO_DOUBLE, as a double-precision twin of the same steps whose entry
// points carry the prefix orc64_.  The twin measures how far an FP64 solve
// (the precision of the CUDA path) departs from the REAL*16 one.
#if defined(TMO_DD)
#define TMO_NAME(x) orcdd_##x
#elif defined(TMO_DOUBLE)
#define TMO_NAME(x) orc64_##x
#else
#define TMO_NAME(x) orc_##x
#endif

namespace tmo {

#if defined(TMO_DD)
typedef ddm::dd Q;
static inline Q qsqrt(Q x) { return ddm::dd_sqrt(x); }
static inline Q qcos(Q x) { return ddm::dd_cos(x); }
static inline Q qsin(Q x) { return ddm::dd_sin(x); }
static inline Q qcosh(Q x) { return ddm::dd_cosh(x); }
static inline Q qsinh(Q x) { return ddm::dd_sinh(x); }
static inline Q qpow(Q x, Q y) { return ddm::dd_pow(x, y); }
static inline Q qacos(Q x) { return (double)x == -1.0 ? ddm::DD_PI : Q(std::acos((double)x)); }
static inline Q qfabs(Q x) { return ddm::dd_abs(x); }
static const Q Q_NEWTON_TOL = Q(1e-31), Q_TINY = Q(1e-300);
#elif defined(TMO_DOUBLE)
typedef double Q;
static inline Q qsqrt(Q x) { return std::sqrt(x); }
static inline Q qcos(Q x) { return std::cos(x); }
static inline Q qsin(Q x) { return std::sin(x); }
static inline Q qcosh(Q x) { return std::cosh(x); }
static inline Q qsinh(Q x) { return std::sinh(x); }
static inline Q qpow(Q x, Q y) { return std::pow(x, y); }
static inline Q qacos(Q x) { return std::acos(x); }
static inline Q qfabs(Q x) { return std::fabs(x); }
static const Q Q_NEWTON_TOL = (Q)1e-16, Q_TINY = (Q)1e-300;
#else
typedef __float128 Q;
static inline Q qsqrt(Q x) { return sqrtq(x); }
static inline Q qcos(Q x) { return cosq(x); }
static inline Q qsin(Q x) { return sinq(x); }
static inline Q qcosh(Q x) { return coshq(x); }
static inline Q qsinh(Q x) { return sinhq(x); }
static inline Q qpow(Q x, Q y) { return powq(x, y); }
static inline Q qacos(Q x) { return acosq(x); }
static inline Q qfabs(Q x) { return fabsq(x); }
static const Q Q_NEWTON_TOL = (Q)1e-33, Q_TINY = (Q)1e-40;
#endif

struct CQ {
  Q r, i;
};
static inline CQ cq(Q r, Q i) { return CQ{r, i}; }
static inline CQ operator+(CQ a, CQ b) { return {a.r + b.r, a.i + b.i}; }
static inline CQ operator-(CQ a, CQ b) { return {a.r - b.r, a.i - b.i}; }
static inline CQ operator*(CQ a, CQ b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
static inline CQ cdivq(CQ a, CQ b) {
  const Q d = b.r * b.r + b.i * b.i;
  return {(a.r * b.r + a.i * b.i) / d, (a.i * b.r - a.r * b.i) / d};
}
static inline Q cabsq2(CQ a) { return a.r * a.r + a.i * a.i; }

// Limits of the reference build (src/tmatrix_amplq.par.f): NPN1 = 100 orders,
// NPNG1 = 500 Gauss points per half.
constexpr int NPN1 = 100;
constexpr int NPNG1 = 500;

// Gauss-Legendre nodes (ascending on [-1, 1]) and weights (summing to 2) by
// Newton iteration on the Legendre recurrence in quadruple precision
// (QGAUSS, tmatrix_amplq.lp.f:1025-1112, with IND1 = 0).
static void gauss_legendre(int n, std::vector<Q>& z, std::vector<Q>& w) {
  z.assign(n, 0);
  w.assign(n, 0);
  const Q pi = qacos((Q)-1);
  for (int k = 0; k < (n + 1) / 2; k++) {
    Q x = qcos(pi * ((Q)k + (Q)0.75) / ((Q)n + (Q)0.5));
    Q dp = 1;
    for (int it = 0; it < 200; it++) {
      Q p0 = 1, p1 = x;
      for (int j = 2; j <= n; j++) {
        const Q p2 = (((Q)(2 * j - 1)) * x * p1 - ((Q)(j - 1)) * p0) / (Q)j;
        p0 = p1;
        p1 = p2;
      }
      // p1 = P_n(x), p0 = P_{n-1}(x)
      dp = ((Q)n) * (x * p1 - p0) / (x * x - 1);
      const Q dx = p1 / dp;
      x -= dx;
      if (qfabs(dx) <= Q_NEWTON_TOL * qfabs(x) || qfabs(dx) < Q_TINY) break;
    }
    Q p0 = 1, p1 = x;
    for (int j = 2; j <= n; j++) {
      const Q p2 = (((Q)(2 * j - 1)) * x * p1 - ((Q)(j - 1)) * p0) / (Q)j;
      p0 = p1;
      p1 = p2;
    }
    dp = ((Q)n) * (x * p1 - p0) / (x * x - 1);
    if ((n & 1) && k == (n - 1) / 2) x = 0;
    const Q wk = (Q)2 / ((1 - x * x) * dp * dp);
    z[n - 1 - k] = x;
    w[n - 1 - k] = wk;
    z[k] = -x;
    w[k] = wk;
  }
}

// Shared state of one solve (the reference's common blocks /CBESS/, /CT/).
struct Solve {
  int nmax = 0, ngauss = 0;
  std::vector<Q> x, w, s, ss, an, dd;   // CONST
  std::vector<Q> r, dr, ddr, drr, dri;  // VARY / RSP1
  Q ppi = 0, pir = 0, pii = 0;
  // Bessel tables [point][n], n = 1..nmax stored at n - 1
  std::vector<Q> J, Y, JR, JI, DJ, DY, DJR, DJI;
  // T of the last TMATR0 / TMATR call (double, column-major 2*nm square)
  std::vector<double> tr, ti;
  int tn = 0;
};

// CONST (tmatrix_amplq.lp.f:972-1023) for NP = -1: the order factors and the
// 2*ngauss-point quadrature with 1/sin and 1/sin^2 at each node.
static void cons(Solve& S) {
  const int nmax = S.nmax, ng = 2 * S.ngauss;
  S.an.assign(nmax + 1, 0);
  S.dd.assign(nmax + 1, 0);
  for (int n = 1; n <= nmax; n++) {
    S.an[n] = (Q)(n * (n + 1));
    // single-precision float() arithmetic of the reference
    S.dd[n] = (Q)sqrtf((float)(2 * n + 1) / (float)(n * (n + 1)));
  }
  gauss_legendre(ng, S.x, S.w);
  S.s.assign(ng, 0);
  S.ss.assign(ng, 0);
  for (int i = 0; i < S.ngauss; i++) {
    Q y = S.x[i];
    y = (Q)1 / ((Q)1 - y * y);
    S.ss[i] = y;
    S.ss[ng - 1 - i] = y;
    y = qsqrt(y);
    S.s[i] = y;
    S.s[ng - 1 - i] = y;
  }
}
static inline Q ann(const Solve& S, int n1, int n2) { return S.dd[n1] * S.dd[n2] * (Q)0.5; }

// RSP1 (tmatrix_amplq.lp.f:1194-1225): r^2(theta) and (dr/dtheta)/r of a
// spheroid with axis ratio eps and equal-volume radius rev.
static void rsp1(Solve& S, Q rev, Q eps) {
  const int ng = 2 * S.ngauss;
  S.r.assign(ng, 0);
  S.dr.assign(ng, 0);
  const Q a = rev * qpow(eps, (Q)1 / (Q)3);
  const Q aa = a * a, ee = eps * eps, ee1 = ee - 1;
  for (int i = 0; i < S.ngauss; i++) {
    const Q c = S.x[i], cc = c * c, ssv = 1 - cc, s = qsqrt(ssv);
    const Q rr = 1 / (ssv + ee * cc);
    S.r[i] = aa * rr;
    S.r[ng - 1 - i] = S.r[i];
    S.dr[i] = rr * c * s * ee1;
    S.dr[ng - 1 - i] = -S.dr[i];
  }
}

// RJB (tmatrix_amplq.lp.f:1383-1413): spherical Bessel j_n(x) by downward
// ratio recurrence from order nmax + nnmax, and u_n = j_{n-1} - n j_n / x.
static void rjb(Q x, Q* y, Q* u, int nmax, int nnmax) {
  const int L = nmax + nnmax;
  std::vector<Q> z(L + 1);
  const Q xx = 1 / x;
  z[L] = 1 / ((Q)(2 * L + 1) * xx);
  for (int i1 = L - 1; i1 >= 1; i1--) z[i1] = 1 / ((Q)(2 * i1 + 1) * xx - z[i1 + 1]);
  const Q z0 = 1 / (xx - z[1]);
  const Q y0 = z0 * qcos(x) * xx;
  const Q y1 = y0 * z[1];
  u[0] = y0 - y1 * xx;
  y[0] = y1;
  for (int i = 2; i <= nmax; i++) {
    const Q yi1 = y[i - 2], yi = yi1 * z[i];
    u[i - 1] = yi1 - (Q)i * yi * xx;
    y[i - 1] = yi;
  }
}

// RYB (tmatrix_amplq.lp.f:1416-1442): spherical Neumann y_n(x) by upward
// recurrence and v_n = y_{n-1} - n y_n / x.
static void ryb(Q x, Q* y, Q* v, int nmax) {
  const Q c = qcos(x), s = qsin(x), x1 = 1 / x, x2 = x1 * x1, x3 = x2 * x1;
  std::vector<Q> t(nmax + 2);
  t[1] = -c * x2 - s * x1;
  t[2] = (-3 * x3 + x1) * c - 3 * x2 * s;
  for (int i = 2; i <= nmax - 1; i++) t[i + 1] = (Q)(2 * i + 1) * x1 * t[i] - t[i - 1];
  for (int i = 1; i <= nmax; i++) y[i - 1] = t[i];
  v[0] = -x1 * (c + t[1]);
  for (int i = 2; i <= nmax; i++) v[i - 1] = t[i - 1] - (Q)i * x1 * t[i];
}

// CJB (tmatrix_amplq.lp.f:1445-1524): RJB for a complex argument m k r.
static void cjb(Q xr, Q xi, Q* yr, Q* yi, Q* ur, Q* ui, int nmax, int nnmax) {
  const int L = nmax + nnmax;
  std::vector<CQ> z(L + 1);
  const CQ x = cq(xr, xi);
  const CQ cx = cdivq(cq(1, 0), x);
  z[L] = cq(xr / (Q)(2 * L + 1), xi / (Q)(2 * L + 1));
  for (int i1 = L - 1; i1 >= 1; i1--) {
    const CQ a = cq((Q)(2 * i1 + 1) * cx.r - z[i1 + 1].r, (Q)(2 * i1 + 1) * cx.i - z[i1 + 1].i);
    z[i1] = cdivq(cq(1, 0), a);
  }
  const CQ z0 = cdivq(cq(1, 0), cx - z[1]);
  const CQ cosx = cq(qcos(xr) * qcosh(xi), -qsin(xr) * qsinh(xi));
  const CQ y0 = (z0 * cosx) * cx;
  CQ yprev = y0 * z[1];
  const CQ u1 = y0 - yprev * cx;
  yr[0] = yprev.r;
  yi[0] = yprev.i;
  ur[0] = u1.r;
  ui[0] = u1.i;
  for (int i = 2; i <= nmax; i++) {
    const CQ yv = yprev * z[i];
    const CQ a = yv * cx;
    const CQ uv = cq(yprev.r - (Q)i * a.r, yprev.i - (Q)i * a.i);
    yr[i - 1] = yv.r;
    yi[i - 1] = yv.i;
    ur[i - 1] = uv.r;
    ui[i - 1] = uv.i;
    yprev = yv;
  }
}

// VARY (tmatrix_amplq.lp.f:1114-1192) for NP = -1: the surface, the size
// parameters at each node and the Bessel tables (BESS :1342-1380).
// Returns nonzero when the reference reports NMAX + NNMAX2 >= 1200.
static int vary(Solve& S, Q lam, Q mrr, Q mri, Q a, Q eps) {
  const int ng = 2 * S.ngauss, nmax = S.nmax;
  rsp1(S, a, eps);
  const Q pi = qacos((Q)-1) * (Q)2 / lam;
  S.ppi = pi * pi;
  S.pir = S.ppi * mrr;
  S.pii = S.ppi * mri;
  Q v = (Q)1 / (mrr * mrr + mri * mri);
  const Q prr = mrr * v, pri = -mri * v;
  Q ta = 0;
  std::vector<Q> z(ng), zr(ng), zi(ng);
  S.ddr.assign(ng, 0);
  S.drr.assign(ng, 0);
  S.dri.assign(ng, 0);
  for (int i = 0; i < ng; i++) {
    const Q vv = qsqrt(S.r[i]);
    v = vv * pi;
    if (v > ta) ta = v;
    const Q iv = 1 / v;
    S.ddr[i] = iv;
    S.drr[i] = prr * iv;
    S.dri[i] = pri * iv;
    z[i] = v;
    zr[i] = v * mrr;
    zi[i] = v * mri;
  }
  Q tb = ta * qsqrt(mrr * mrr + mri * mri);
  if (tb < (Q)nmax) tb = (Q)nmax;
  const int nnmax1 = (int)((Q)8 * qsqrt(ta > (Q)nmax ? ta : (Q)nmax) + (Q)3);
  int nnmax2 = (int)(tb + (Q)4 * qpow(tb, (Q)33333 / (Q)100000) + (Q)8 * qsqrt(tb));
  nnmax2 = nnmax2 - nmax + 5;
  if (nmax + nnmax2 >= 1200) return 1;
  const size_t T = (size_t)ng * nmax;
  for (auto* p : {&S.J, &S.Y, &S.JR, &S.JI, &S.DJ, &S.DY, &S.DJR, &S.DJI}) p->assign(T, 0);
  for (int i = 0; i < ng; i++) {
    const size_t o = (size_t)i * nmax;
    rjb(z[i], &S.J[o], &S.DJ[o], nmax, nnmax1);
    ryb(z[i], &S.Y[o], &S.DY[o], nmax);
    cjb(zr[i], zi[i], &S.JR[o], &S.JI[o], &S.DJR[o], &S.DJI[o], nmax, nnmax2);
  }
  return 0;
}

// VIG (tmatrix_amplq.lp.f:2049-2105): Wigner d^n_{0m}(x) (dv1) and its
// theta-derivative (dv2) for n = 1..nmax (index n - 1), zero below n = m.
static void vig(Q x, int nmax, int m, Q* dv1, Q* dv2) {
  for (int n = 0; n < nmax; n++) dv1[n] = dv2[n] = 0;
  const Q qs = qsqrt(1 - x * x), qs1 = 1 / qs;
  if (m == 0) {
    Q d1 = 1, d2 = x;
    for (int n = 1; n <= nmax; n++) {
      const Q qn = n, qn1 = n + 1, qn2 = 2 * n + 1;
      const Q d3 = (qn2 * x * d2 - qn * d1) / qn1;
      const Q der = qs1 * (qn1 * qn / qn2) * (-d1 + d3);
      dv1[n - 1] = d2;
      dv2[n - 1] = der;
      d1 = d2;
      d2 = d3;
    }
    return;
  }
  const Q qmm = (Q)(m * m);
  Q a = 1;
  for (int i = 1; i <= m; i++) {
    const int i2 = 2 * i;
    // single-precision float() arithmetic of the reference
    a = a * (Q)sqrtf((float)(i2 - 1) / (float)i2) * qs;
  }
  Q d1 = 0, d2 = a;
  for (int n = m; n <= nmax; n++) {
    const Q qn = n, qn2 = 2 * n + 1, qn1 = n + 1;
    const Q qnm = qsqrt(qn * qn - qmm), qnm1 = qsqrt(qn1 * qn1 - qmm);
    const Q d3 = (qn2 * x * d2 - qnm * d1) / qnm1;
    const Q der = qs1 * (-qn1 * qnm * d1 + qn * qnm1 * d3) / qn2;
    dv1[n - 1] = d2;
    dv2[n - 1] = der;
    d1 = d2;
    d2 = d3;
  }
}

// TT (tmatrix_amplq.lp.f:2107-2153): T = -RgQ Q^-1.  Q is inverted in
// quadruple precision (Gauss-Jordan with partial pivoting; the reference uses
// LU + inversion in COMPLEX*32), the product is accumulated in double over
// k = 1..n as the reference does.
static int tt(Solve& S, int nm, const std::vector<CQ>& q, const std::vector<CQ>& rgq) {
  const int n = 2 * nm;
  std::vector<CQ> a(q), inv((size_t)n * n, cq(0, 0));
  for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = cq(1, 0);
  // row-major a[i*n + j] = Q(i, j)
  for (int c = 0; c < n; c++) {
    int p = c;
    Q best = cabsq2(a[(size_t)c * n + c]);
    for (int r2 = c + 1; r2 < n; r2++) {
      const Q v = cabsq2(a[(size_t)r2 * n + c]);
      if (v > best) { best = v; p = r2; }
    }
    if (best == 0) return 1;
    if (p != c)
      for (int j = 0; j < n; j++) {
        std::swap(a[(size_t)p * n + j], a[(size_t)c * n + j]);
        std::swap(inv[(size_t)p * n + j], inv[(size_t)c * n + j]);
      }
    const CQ piv = cdivq(cq(1, 0), a[(size_t)c * n + c]);
    for (int j = 0; j < n; j++) {
      a[(size_t)c * n + j] = a[(size_t)c * n + j] * piv;
      inv[(size_t)c * n + j] = inv[(size_t)c * n + j] * piv;
    }
    for (int r2 = 0; r2 < n; r2++) {
      if (r2 == c) continue;
      const CQ f = a[(size_t)r2 * n + c];
      if (f.r == 0 && f.i == 0) continue;
      for (int j = 0; j < n; j++) {
        a[(size_t)r2 * n + j] = a[(size_t)r2 * n + j] - f * a[(size_t)c * n + j];
        inv[(size_t)r2 * n + j] = inv[(size_t)r2 * n + j] - f * inv[(size_t)c * n + j];
      }
    }
  }
  S.tn = n;
  S.tr.assign((size_t)n * n, 0.0);
  S.ti.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double tr = 0.0, ti = 0.0;
      for (int k = 0; k < n; k++) {
        const double arr = (double)rgq[(size_t)i * n + k].r, ari = (double)rgq[(size_t)i * n + k].i;
        const double ar = (double)inv[(size_t)k * n + j].r, ai = (double)inv[(size_t)k * n + j].i;
        tr = tr - arr * ar + ari * ai;
        ti = ti - arr * ai - ari * ar;
      }
      S.tr[(size_t)j * n + i] = tr;  // column-major like TR1(I, J)
      S.ti[(size_t)j * n + i] = ti;
    }
  return 0;
}

// TMATR0 (m = 0, tmatrix_amplq.lp.f:1526-1763) and TMATR (m >= 1, :1765-2047)
// with NCHECK = 1 (mirror-symmetric spheroids: half the nodes, factor 2, and
// only the (n1 + n2)-parity blocks that do not vanish).  Builds Q and RgQ of
// order 2 (nmax - m' + 1), m' = max(m, 1), and leaves T in S.tr / S.ti.
static int tmatr(Solve& S, int m) {
  const int nmax = S.nmax, ngs = S.ngauss;
  const int mm1 = (m == 0) ? 1 : m;
  const Q qm = m, qmm = (Q)(m * m);
  std::vector<Q> d1((size_t)2 * ngs * nmax), d2((size_t)2 * ngs * nmax), dv1(nmax), dv2(nmax);
  auto sig = [](int n) { return (n & 1) ? (Q)-1 : (Q)1; };
  for (int i = 1; i <= ngs; i++) {
    const int i1 = ngs + i - 1, i2 = ngs - i;  // 0-based upper / mirrored node
    vig(S.x[i1], nmax, m, dv1.data(), dv2.data());
    for (int n = 1; n <= nmax; n++) {
      const Q si = sig(n + m);
      d1[(size_t)i1 * nmax + n - 1] = dv1[n - 1];
      d2[(size_t)i1 * nmax + n - 1] = dv2[n - 1];
      d1[(size_t)i2 * nmax + n - 1] = dv1[n - 1] * si;
      d2[(size_t)i2 * nmax + n - 1] = -dv2[n - 1] * si;
    }
  }
  const int nm = nmax - mm1 + 1, n2m = 2 * nm;
  // block integrals [11, 12, 21, 22] x (Q, RgQ) of each (n1, n2), complex
  std::vector<CQ> A[4], G[4];
  for (int k = 0; k < 4; k++) {
    A[k].assign((size_t)nm * nm, cq(0, 0));
    G[k].assign((size_t)nm * nm, cq(0, 0));
  }
  for (int n1 = mm1; n1 <= nmax; n1++) {
    const Q an1 = S.an[n1];
    for (int n2 = mm1; n2 <= nmax; n2++) {
      const Q an2 = S.an[n2];
      const bool even = sig(n1 + n2) > 0;  // NCHECK: 12/21 blocks only, else 11/22
      CQ a11 = cq(0, 0), a12 = a11, a21 = a11, a22 = a11, g11 = a11, g12 = a11, g21 = a11, g22 = a11;
      if (!(m == 0 && !even)) {
        for (int i = 0; i < ngs; i++) {
          const Q d1n1 = d1[(size_t)i * nmax + n1 - 1], d2n1 = d2[(size_t)i * nmax + n1 - 1];
          const Q d1n2 = d1[(size_t)i * nmax + n2 - 1], d2n2 = d2[(size_t)i * nmax + n2 - 1];
          const Q e11 = d1n1 * d1n2, e12 = d1n1 * d2n2, e21 = d2n1 * d1n2, e22 = d2n1 * d2n2;
          const size_t o1 = (size_t)i * nmax + n1 - 1, o2 = (size_t)i * nmax + n2 - 1;
          const Q qj1 = S.J[o1], qy1 = S.Y[o1], qdj1 = S.DJ[o1], qdy1 = S.DY[o1];
          const CQ jr2 = cq(S.JR[o2], S.JI[o2]), djr2 = cq(S.DJR[o2], S.DJI[o2]);
          const CQ h1 = cq(qj1, qy1), dh1 = cq(qdj1, qdy1);
          // c: regular (j_n(kr) j_n(mkr)); b: outgoing (h_n(kr) j_n(mkr))
          const CQ c1 = cq(jr2.r * qj1, jr2.i * qj1), b1 = cq(c1.r - jr2.i * qy1, c1.i + jr2.r * qy1);
          const CQ c2 = cq(jr2.r * qdj1, jr2.i * qdj1), b2 = cq(c2.r - jr2.i * qdy1, c2.i + jr2.r * qdy1);
          const Q ddri = S.ddr[i];
          const CQ c3 = cq(ddri * c1.r, ddri * c1.i), b3 = cq(ddri * b1.r, ddri * b1.i);
          const CQ c4 = cq(djr2.r * qj1, djr2.i * qj1), b4 = cq(c4.r - djr2.i * qy1, c4.i + djr2.r * qy1);
          const CQ dm = cq(S.drr[i], S.dri[i]);
          const CQ c5 = c1 * dm, b5 = b1 * dm;
          (void)h1;
          (void)dh1;
          const Q uri = S.dr[i], wr = S.w[i] * S.r[i];
          if (m == 0) {
            const Q f1 = wr * e22;
            Q f2 = wr * uri * an1 * e12;
            a12 = cq(a12.r + f1 * b2.r + f2 * b3.r, a12.i + f1 * b2.i + f2 * b3.i);
            g12 = cq(g12.r + f1 * c2.r + f2 * c3.r, g12.i + f1 * c2.i + f2 * c3.i);
            f2 = wr * uri * an2 * e21;
            a21 = cq(a21.r + f1 * b4.r + f2 * b5.r, a21.i + f1 * b4.i + f2 * b5.i);
            g21 = cq(g21.r + f1 * c4.r + f2 * c5.r, g21.i + f1 * c4.i + f2 * c5.i);
            continue;
          }
          const Q dsi = S.s[i] * qm * wr, dssi = S.ss[i] * qmm;
          const Q aa1 = e12 + e21, aa2 = e11 * dssi + e22;
          if (even) {
            const Q f1 = wr * aa2;
            Q f2 = wr * uri * an1 * e12;
            a12 = cq(a12.r + f1 * b2.r + f2 * b3.r, a12.i + f1 * b2.i + f2 * b3.i);
            g12 = cq(g12.r + f1 * c2.r + f2 * c3.r, g12.i + f1 * c2.i + f2 * c3.i);
            f2 = wr * uri * an2 * e21;
            a21 = cq(a21.r + f1 * b4.r + f2 * b5.r, a21.i + f1 * b4.i + f2 * b5.i);
            g21 = cq(g21.r + f1 * c4.r + f2 * c5.r, g21.i + f1 * c4.i + f2 * c5.i);
          } else {
            const CQ c6 = cq(djr2.r * qdj1, djr2.i * qdj1), b6 = cq(c6.r - djr2.i * qdy1, c6.i + djr2.r * qdy1);
            const CQ c7 = cq(c4.r * ddri, c4.i * ddri), b7 = cq(b4.r * ddri, b4.i * ddri);
            const CQ c8 = c2 * dm, b8 = b2 * dm;
            const Q e1 = dsi * aa1;
            a11 = cq(a11.r + e1 * b1.r, a11.i + e1 * b1.i);
            g11 = cq(g11.r + e1 * c1.r, g11.i + e1 * c1.i);
            Q e2 = dsi * uri * e11;
            const Q e3 = e2 * an2;
            e2 = e2 * an1;
            a22 = cq(a22.r + e1 * b6.r + e2 * b7.r + e3 * b8.r, a22.i + e1 * b6.i + e2 * b7.i + e3 * b8.i);
            g22 = cq(g22.r + e1 * c6.r + e2 * c7.r + e3 * c8.r, g22.i + e1 * c6.i + e2 * c7.i + e3 * c8.i);
          }
        }
      }
      const Q an12 = ann(S, n1, n2) * (Q)2;
      const size_t o = (size_t)(n1 - mm1) * nm + (n2 - mm1);
      A[0][o] = cq(a11.r * an12, a11.i * an12);
      A[1][o] = cq(a12.r * an12, a12.i * an12);
      A[2][o] = cq(a21.r * an12, a21.i * an12);
      A[3][o] = cq(a22.r * an12, a22.i * an12);
      G[0][o] = cq(g11.r * an12, g11.i * an12);
      G[1][o] = cq(g12.r * an12, g12.i * an12);
      G[2][o] = cq(g21.r * an12, g21.i * an12);
      G[3][o] = cq(g22.r * an12, g22.i * an12);
    }
  }
  // Q = k^2 m' X + k^2 X' with the block phases of the reference:
  // T11 = -(R11 + i I11), T12 = -i (R12 + i I12), T21 = i (R21 + i I21),
  // T22 = -(R22 + i I22); Q(1,1) = km^2 T21 + k^2 T12, Q(1,2) = km^2 T11 +
  // k^2 T22, Q(2,1) = km^2 T22 + k^2 T11, Q(2,2) = km^2 T12 + k^2 T21.
  const CQ km = cq(S.pir, S.pii);
  const Q kk = S.ppi;
  std::vector<CQ> q((size_t)n2m * n2m), rg((size_t)n2m * n2m);
  auto ph = [](int blk, CQ v) -> CQ {
    switch (blk) {
      case 0: return cq(-v.r, -v.i);
      case 1: return cq(v.i, -v.r);
      case 2: return cq(-v.i, v.r);
      default: return cq(-v.r, -v.i);
    }
  };
  for (int k1 = 0; k1 < nm; k1++)
    for (int k2 = 0; k2 < nm; k2++) {
      const size_t o = (size_t)k1 * nm + k2;
      CQ t[4], g[4];
      for (int b = 0; b < 4; b++) {
        t[b] = ph(b, A[b][o]);
        g[b] = ph(b, G[b][o]);
      }
      auto comb = [&](CQ x, CQ y) { return cq(km.r * x.r - km.i * x.i + kk * y.r, km.r * x.i + km.i * x.r + kk * y.i); };
      const int K1 = k1 + nm, K2 = k2 + nm;
      if (m == 0) {
        q[(size_t)k1 * n2m + k2] = comb(t[2], t[1]);
        rg[(size_t)k1 * n2m + k2] = comb(g[2], g[1]);
        q[(size_t)k1 * n2m + K2] = rg[(size_t)k1 * n2m + K2] = cq(0, 0);
        q[(size_t)K1 * n2m + k2] = rg[(size_t)K1 * n2m + k2] = cq(0, 0);
        q[(size_t)K1 * n2m + K2] = comb(t[1], t[2]);
        rg[(size_t)K1 * n2m + K2] = comb(g[1], g[2]);
      } else {
        q[(size_t)k1 * n2m + k2] = comb(t[2], t[1]);
        rg[(size_t)k1 * n2m + k2] = comb(g[2], g[1]);
        q[(size_t)k1 * n2m + K2] = comb(t[0], t[3]);
        rg[(size_t)k1 * n2m + K2] = comb(g[0], g[3]);
        q[(size_t)K1 * n2m + k2] = comb(t[3], t[0]);
        rg[(size_t)K1 * n2m + k2] = comb(g[3], g[0]);
        q[(size_t)K1 * n2m + K2] = comb(t[1], t[2]);
        rg[(size_t)K1 * n2m + K2] = comb(g[1], g[2]);
      }
    }
  return tt(S, nm, q, rg);
}

// Single-precision T-matrix of one particle (common /TMAT/ of the
// reference): element (m, block, n1, n2) with block 0..3 = 11, 12, 21, 22,
// m = 0..nmax, n1, n2 = 1..nmax.
struct TMat {
  int nmax = 0;
  std::vector<float> re, im;
  size_t at(int m, int blk, int n1, int n2) const {
    return (((size_t)m * 4 + blk) * nmax + (n1 - 1)) * nmax + (n2 - 1);
  }
};

// tmatrix_amplq (tmatrix_amplq.lp.f:276-600) for NP = -1, RAT = 1: the
// convergence in NMAX (from x + 4.05 x^(1/3)) and then in NGAUSS on the m = 0
// extinction and scattering sums (DDELT = 1e-3, NDGS = 2), then the m >= 1
// blocks, stored in single precision.  lam, mrr, mri, axi, as_ratio are the
// reference's double inputs.  Returns 0, or 1 when a limit of the reference
// build is reached (its fatal error paths).
static int amplq(double lam_d, double mrr_d, double mri_d, double axi, double as_ratio, TMat& out) {
  const Q eps = (Q)(1.0 / as_ratio);
  const double ddelt = 0.001;
  const int ndgs = 2;
  const Q lam = lam_d, mrr = mrr_d, mri = mri_d;
  const Q a = (Q)(1.0 * axi);
  const double pin = (double)qacos((Q)-1);
  const double dlam = lam_d;
  const double xev = (double)((Q)(2.0 * pin) * a / (Q)dlam);
  const int ixxx = (int)(xev + 4.05 * std::pow(xev, 0.333333));
  const int inm1 = std::max(4, ixxx);
  if (inm1 >= NPN1) return 1;
  Solve S;
  double qext1 = 0.0, qsca1 = 0.0;
  bool conv = false;
  auto sums = [&](double& qext, double& qsca) {
    qext = 0.0;
    qsca = 0.0;
    const int nmax = S.nmax, n = S.tn;
    for (int k = 1; k <= nmax; k++) {
      const int k1 = k + nmax;
      const double tr = S.tr[(size_t)(k - 1) * n + k - 1], ti = S.ti[(size_t)(k - 1) * n + k - 1];
      const double tr1 = S.tr[(size_t)(k1 - 1) * n + k1 - 1], ti1 = S.ti[(size_t)(k1 - 1) * n + k1 - 1];
      const double dn1 = (double)(2 * k + 1);
      qsca = qsca + dn1 * (tr * tr + ti * ti + tr1 * tr1 + ti1 * ti1);
      qext = qext + (tr + tr1) * dn1;
    }
  };
  for (int nma = inm1; nma <= NPN1; nma++) {
    S.nmax = nma;
    S.ngauss = nma * ndgs;
    if (S.ngauss > NPNG1) return 1;
    cons(S);
    if (vary(S, lam, mrr, mri, a, eps)) return 1;
    if (tmatr(S, 0)) return 1;
    double qext, qsca;
    sums(qext, qsca);
    const double dsca = std::fabs((qsca1 - qsca) / qsca), dext = std::fabs((qext1 - qext) / qext);
    qext1 = qext;
    qsca1 = qsca;
    if (dsca <= ddelt && dext <= ddelt) { conv = true; break; }
    if (nma == NPN1) return 1;
  }
  if (!conv) return 1;
  if (S.ngauss != NPNG1) {
    for (int ngaus = S.ngauss + 1; ngaus <= NPNG1; ngaus++) {
      S.ngauss = ngaus;
      cons(S);
      if (vary(S, lam, mrr, mri, a, eps)) return 1;
      if (tmatr(S, 0)) return 1;
      double qext, qsca;
      sums(qext, qsca);
      const double dsca = std::fabs((qsca1 - qsca) / qsca), dext = std::fabs((qext1 - qext) / qext);
      qext1 = qext;
      qsca1 = qsca;
      if (dsca <= ddelt && dext <= ddelt) break;
    }
  }
  const int nmax = S.nmax;
  out.nmax = nmax;
  out.re.assign((size_t)(nmax + 1) * 4 * nmax * nmax, 0.f);
  out.im.assign(out.re.size(), 0.f);
  auto put = [&](int m, int nm, int off) {
    const int n = S.tn;
    for (int n2 = 1; n2 <= nm; n2++)
      for (int n1 = 1; n1 <= nm; n1++) {
        const int r[4] = {n1, n1, n1 + nm, n1 + nm}, c[4] = {n2, n2 + nm, n2, n2 + nm};
        for (int b = 0; b < 4; b++) {
          const size_t src = (size_t)(c[b] - 1) * n + (r[b] - 1);
          const size_t dst = out.at(m, b, n1 + off, n2 + off);
          out.re[dst] = (float)S.tr[src];
          out.im[dst] = (float)S.ti[src];
        }
      }
  };
  put(0, nmax, 0);
  for (int m = 1; m <= nmax; m++) {
    if (tmatr(S, m)) return 1;
    put(m, nmax - m + 1, m - 1);
  }
  return 0;
}

// VIGAMPL (tmatrix_amplq.lp.f:890-970): d^n_{0m}(x) / sin(theta) (dv1) and
// the theta-derivative (dv2) in double, with the limit values at the poles.
static void vigampl(double x, int nmax, int m, double* dv1, double* dv2) {
  for (int n = 0; n < nmax; n++) dv1[n] = dv2[n] = 0.0;
  const double dx = std::fabs(x);
  if (std::fabs(1.0 - dx) <= 1e-10) {
    if (m != 1) return;
    for (int n = 1; n <= nmax; n++) {
      double dn = (double)(n * (n + 1));
      dn = 0.5 * std::sqrt(dn);
      if (x < 0.0) dn = dn * (((n + 1) & 1) ? -1.0 : 1.0);
      dv1[n - 1] = dn;
      if (x < 0.0) dn = -dn;
      dv2[n - 1] = dn;
    }
    return;
  }
  const double qs = std::sqrt(1.0 - x * x), qs1 = 1.0 / qs, dsi = qs1;
  if (m == 0) {
    double d1 = 1.0, d2 = x;
    for (int n = 1; n <= nmax; n++) {
      const double qn = n, qn1 = n + 1, qn2 = 2 * n + 1;
      const double d3 = (qn2 * x * d2 - qn * d1) / qn1;
      const double der = qs1 * (qn1 * qn / qn2) * (-d1 + d3);
      dv1[n - 1] = d2 * dsi;
      dv2[n - 1] = der;
      d1 = d2;
      d2 = d3;
    }
    return;
  }
  const double qmm = (double)(m * m);
  double a = 1.0;
  for (int i = 1; i <= m; i++) {
    const int i2 = 2 * i;
    a = a * std::sqrt((double)(i2 - 1) / (double)i2) * qs;
  }
  double d1 = 0.0, d2 = a;
  for (int n = m; n <= nmax; n++) {
    const double qn = n, qn2 = 2 * n + 1, qn1 = n + 1;
    const double qnm = std::sqrt(qn * qn - qmm), qnm1 = std::sqrt(qn1 * qn1 - qmm);
    const double d3 = (qn2 * x * d2 - qnm * d1) / qnm1;
    const double der = qs1 * (-qn1 * qnm * d1 + qn * qnm1 * d3) / qn2;
    dv1[n - 1] = d2 * dsi;
    dv2[n - 1] = der;
    d1 = d2;
    d2 = d3;
  }
}

struct C2 {
  double r, i;
};
static inline C2 c2(double r, double i) { return {r, i}; }
static inline C2 operator+(C2 a, C2 b) { return {a.r + b.r, a.i + b.i}; }
static inline C2 operator-(C2 a, C2 b) { return {a.r - b.r, a.i - b.i}; }
static inline C2 operator*(C2 a, C2 b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
static inline C2 operator*(C2 a, double s) { return {a.r * s, a.i * s}; }

// AMPL (tmatrix_amplq.lp.f:602-888): amplitude matrix (VV, VH, HV, HH) for
// incidence (tl, pl) and scattering (tl1, pl1) in degrees of a particle with
// orientation (alpha, beta), from the single-precision T-matrix.
static void ampl(const TMat& T, double dlam, double tl, double tl1, double pl, double pl1, double alpha,
                 double beta, C2& vv, C2& vh, C2& hv, C2& hh) {
  const int nmax = T.nmax;
  const double pin = std::acos(-1.0), pin2 = pin * 0.5, pi = pin / 180.0;
  const double alph = alpha * pi;
  double bet = beta * pi, thetl = tl * pi, phil = pl * pi, thetl1 = tl1 * pi, phil1 = pl1 * pi;
  const double eps = 1e-8;
  if (thetl < pin2) thetl = thetl + eps;
  if (thetl > pin2) thetl = thetl - eps;
  if (thetl1 < pin2) thetl1 = thetl1 + eps;
  if (thetl1 > pin2) thetl1 = thetl1 - eps;
  if (phil < pin) phil = phil + eps;
  if (phil > pin) phil = phil - eps;
  if (phil1 < pin) phil1 = phil1 + eps;
  if (phil1 > pin) phil1 = phil1 - eps;
  if (bet <= pin2 && pin2 - bet <= eps) bet = bet - eps;
  if (bet > pin2 && bet - pin2 <= eps) bet = bet + eps;
  // particle-frame angles of the incident and scattered directions
  const double cb = std::cos(bet), sb = std::sin(bet);
  double ct = std::cos(thetl), st = std::sin(thetl), cp = std::cos(phil - alph), sp = std::sin(phil - alph);
  const double ctp = ct * cb + st * sb * cp, thetp = std::acos(ctp);
  const double cpp = cb * st * cp - sb * ct, spp = st * sp;
  double phip = std::atan(spp / cpp);
  if (phip > 0.0 && sp < 0.0) phip = phip + pin;
  if (phip < 0.0 && sp > 0.0) phip = phip + pin;
  if (phip < 0.0) phip = phip + 2.0 * pin;
  double ct1 = std::cos(thetl1), st1 = std::sin(thetl1), cp1 = std::cos(phil1 - alph), sp1 = std::sin(phil1 - alph);
  const double ctp1 = ct1 * cb + st1 * sb * cp1, thetp1 = std::acos(ctp1);
  const double cpp1 = cb * st1 * cp1 - sb * ct1, spp1 = st1 * sp1;
  double phip1 = std::atan(spp1 / cpp1);
  if (phip1 > 0.0 && sp1 < 0.0) phip1 = phip1 + pin;
  if (phip1 < 0.0 && sp1 > 0.0) phip1 = phip1 + pin;
  if (phip1 < 0.0) phip1 = phip1 + 2.0 * pin;
  // polarisation-basis rotations lab -> particle frame
  const double ca = std::cos(alph), sa = std::sin(alph);
  const double B[3][3] = {{ca * cb, sa * cb, -sb}, {-sa, ca, 0.0}, {ca * sb, sa * sb, cb}};
  cp = std::cos(phil);
  sp = std::sin(phil);
  cp1 = std::cos(phil1);
  sp1 = std::sin(phil1);
  const double AL[3][2] = {{ct * cp, -sp}, {ct * sp, cp}, {-st, 0.0}};
  const double AL1[3][2] = {{ct1 * cp1, -sp1}, {ct1 * sp1, cp1}, {-st1, 0.0}};
  ct = ctp;
  st = std::sin(thetp);
  cp = std::cos(phip);
  sp = std::sin(phip);
  ct1 = ctp1;
  st1 = std::sin(thetp1);
  cp1 = std::cos(phip1);
  sp1 = std::sin(phip1);
  const double AP[2][3] = {{ct * cp, ct * sp, -st}, {-sp, cp, 0.0}};
  const double AP1[2][3] = {{ct1 * cp1, ct1 * sp1, -st1}, {-sp1, cp1, 0.0}};
  double C[3][2], R[2][2], R1[2][2];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 2; j++) {
      double x = 0.0;
      for (int k = 0; k < 3; k++) x = x + B[i][k] * AL[k][j];
      C[i][j] = x;
    }
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) {
      double x = 0.0;
      for (int k = 0; k < 3; k++) x = x + AP[i][k] * C[k][j];
      R[i][j] = x;
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 2; j++) {
      double x = 0.0;
      for (int k = 0; k < 3; k++) x = x + B[i][k] * AL1[k][j];
      C[i][j] = x;
    }
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++) {
      double x = 0.0;
      for (int k = 0; k < 3; k++) x = x + AP1[i][k] * C[k][j];
      R1[i][j] = x;
    }
  {
    const double d = 1.0 / (R1[0][0] * R1[1][1] - R1[0][1] * R1[1][0]);
    const double x = R1[0][0];
    R1[0][0] = R1[1][1] * d;
    R1[0][1] = -R1[0][1] * d;
    R1[1][0] = -R1[1][0] * d;
    R1[1][1] = x * d;
  }
  // CAL(n, nn) = i^(nn - n - 1) sqrt((2n+1)(2nn+1) / (n nn (n+1)(nn+1)))
  std::vector<C2> cal((size_t)nmax * nmax);
  for (int nn = 1; nn <= nmax; nn++)
    for (int n = 1; n <= nmax; n++) {
      const int e = ((nn - n - 1) % 4 + 4) % 4;
      const C2 cn = (e == 0) ? c2(1, 0) : (e == 1) ? c2(0, 1) : (e == 2) ? c2(-1, 0) : c2(0, -1);
      double dnn = (double)((2 * n + 1) * (2 * nn + 1));
      dnn = dnn / (double)(n * nn * (n + 1) * (nn + 1));
      cal[(size_t)(n - 1) * nmax + nn - 1] = cn * std::sqrt(dnn);
    }
  const double dcth0 = ctp, dcth = ctp1, ph = phip1 - phip;
  vv = vh = hv = hh = c2(0, 0);
  std::vector<double> dv1(nmax), dv2(nmax), dv01(nmax), dv02(nmax);
  for (int m = 0; m <= nmax; m++) {
    const int nmin = std::max(m, 1);
    vigampl(dcth, nmax, m, dv1.data(), dv2.data());
    vigampl(dcth0, nmax, m, dv01.data(), dv02.data());
    const double fc = 2.0 * std::cos(m * ph), fs = 2.0 * std::sin(m * ph);
    for (int nn = nmin; nn <= nmax; nn++) {
      const double dv1nn = m * dv01[nn - 1], dv2nn = dv02[nn - 1];
      for (int n = nmin; n <= nmax; n++) {
        const double dv1n = m * dv1[n - 1], dv2n = dv2[n - 1];
        const C2 ct11 = c2(T.re[T.at(m, 0, n, nn)], T.im[T.at(m, 0, n, nn)]);
        const C2 ct22 = c2(T.re[T.at(m, 3, n, nn)], T.im[T.at(m, 3, n, nn)]);
        const C2 cl = cal[(size_t)(n - 1) * nmax + nn - 1];
        if (m == 0) {
          const C2 cn = cl * dv2n * dv2nn;
          vv = vv + cn * ct22;
          hh = hh + cn * ct11;
        } else {
          const C2 ct12 = c2(T.re[T.at(m, 1, n, nn)], T.im[T.at(m, 1, n, nn)]);
          const C2 ct21 = c2(T.re[T.at(m, 2, n, nn)], T.im[T.at(m, 2, n, nn)]);
          const C2 cn1 = cl * fc, cn2 = cl * fs;
          const double d11 = dv1n * dv1nn, d12 = dv1n * dv2nn, d21 = dv2n * dv1nn, d22 = dv2n * dv2nn;
          vv = vv + (ct11 * d11 + ct21 * d21 + ct12 * d12 + ct22 * d22) * cn1;
          vh = vh + (ct11 * d12 + ct21 * d22 + ct12 * d11 + ct22 * d21) * cn2;
          hv = hv - (ct11 * d21 + ct21 * d11 + ct12 * d22 + ct22 * d12) * cn2;
          hh = hh + (ct11 * d22 + ct21 * d12 + ct12 * d21 + ct22 * d11) * cn1;
        }
      }
    }
  }
  const double dk = 2.0 * pin / dlam;
  vv = c2(vv.r / dk, vv.i / dk);
  vh = c2(vh.r / dk, vh.i / dk);
  hv = c2(hv.r / dk, hv.i / dk);
  hh = c2(hh.r / dk, hh.i / dk);
  const C2 cvv = vv * R[0][0] + vh * R[1][0], cvh = vv * R[0][1] + vh * R[1][1];
  const C2 chv = hv * R[0][0] + hh * R[1][0], chh = hv * R[0][1] + hh * R[1][1];
  vv = cvv * R1[0][0] + chv * R1[0][1];
  vh = cvh * R1[0][0] + chh * R1[0][1];
  hv = cvv * R1[1][0] + chv * R1[1][1];
  hh = cvh * R1[1][0] + chh * R1[1][1];
}

}  // namespace tmo

extern "C" void orc_lobatto(int num, double* mu, double* w);
extern "C" void orc_eps_mix_m(double re, double im, double dens, double* ore, double* oim);

namespace tmo {

// calc_single_tmatrix (src/tmatrix.f90:436-684): one particle at one
// frequency, fixed orientation (alpha = 0, beta = canting), 30 scattering
// azimuths and one incident azimuth, Lobatto quadrature of nummu angles.
// Outputs in the reference's Fortran (column-major) order:
// scat[2][nummu][2][nummu][2] as scatter_matrix(i2, ll, i1, jj, kk),
// ext[2][2][nummu], emis[2][nummu], sback[2][2].
static int single(int nummu, double frequency, double mrr, double mri_abs, double axi, double as_ratio,
                  double alpha, double beta, double* scat, double* ext, double* emis, double* sback) {
  const int azimuth_num = 30, azimuth0_num = 1;
  const double lam = orc::C_LIGHT / frequency;
  const double wave_num = 2.0 * orc::PI / lam;
  TMat T;
  if (amplq(lam, mrr, mri_abs, axi, as_ratio, T)) return 2;
  const int NS = 2 * nummu * 2 * nummu;
  for (int e = 0; e < 2 * NS; e++) scat[e] = 0.0;
  for (int e = 0; e < 4 * nummu; e++) ext[e] = 0.0;
  for (int e = 0; e < 2 * nummu; e++) emis[e] = 0.0;
  const double fact_sca = 0.5 / (wave_num * wave_num);
  // fact_ext = 2 pi i / k^2 (k**2.e0 as a real power)
  const double fext_i = 2.0 * orc::PI / std::pow(wave_num, 2.0);
  std::vector<double> mu(nummu), wq(nummu);
  orc_lobatto(nummu, mu.data(), wq.data());
  auto S_ = [&](int i2, int ll, int i1, int jj, int kk) -> double& {
    return scat[i2 + 2 * (ll + nummu * (i1 + 2 * (jj + nummu * kk)))];
  };
  auto E_ = [&](int i1, int i2, int jj) -> double& { return ext[i1 + 2 * (i2 + 2 * jj)]; };
  for (int jj = 0; jj < nummu; jj++) {
    double thet0 = std::acos(mu[jj] * 1.0) * 180.0 / orc::PI;
    if (thet0 > 179.9999) thet0 = 180.0;
    std::vector<double> e11(2 * nummu, 0.0), e12(2 * nummu, 0.0);
    for (int kk = 0; kk < 2; kk++) {
      for (int ll = 0; ll < nummu; ll++) {
        double thet = std::acos(mu[ll] * (kk == 0 ? 1.0 : -1.0)) * 180.0 / orc::PI;
        const double thet_weights = wq[ll];
        if (thet > 179.9999) thet = 180.0;
        for (int m = 1; m <= azimuth0_num; m++) {
          const double phi0 = 360.0 / (double)azimuth0_num * ((double)m - 1.0);
          const double phi0_weights = 1.0 / 360.0 * (360.0 / azimuth0_num);
          double z11 = 0.0, z12 = 0.0, z21 = 0.0, z22 = 0.0;
          for (int n = 1; n <= azimuth_num; n++) {
            const double phi = 360.0 / (double)azimuth_num * ((double)n - 1.0);
            const double phi_weights = 1.0 / 360.0 * (360.0 / azimuth_num);
            C2 s11, s12, s21, s22;
            ampl(T, lam, thet0, thet, phi0, phi, alpha, beta, s11, s12, s21, s22);
            s11 = s11 * wave_num;
            s12 = s12 * wave_num;
            s21 = s21 * wave_num;
            s22 = s22 * wave_num;
            const double a11 = s11.r * s11.r + s11.i * s11.i, a12 = s12.r * s12.r + s12.i * s12.i;
            const double a21 = s21.r * s21.r + s21.i * s21.i, a22 = s22.r * s22.r + s22.i * s22.i;
            if (thet == 180.0 && phi == phi0) {
              sback[0] = fact_sca * (a11 + a12 + a21 + a22);
              sback[2] = fact_sca * (a11 - a12 + a21 - a22);  // Sback(1,2)
              sback[1] = fact_sca * (a11 + a12 - a21 - a22);  // Sback(2,1)
              sback[3] = fact_sca * (a11 - a12 - a21 + a22);
            }
            z11 = z11 + (fact_sca * (a11 + a12 + a21 + a22)) * phi_weights;
            z12 = z12 + (fact_sca * (a11 - a12 + a21 - a22)) * phi_weights;
            z21 = z21 + (fact_sca * (a11 + a12 - a21 - a22)) * phi_weights;
            z22 = z22 + (fact_sca * (a11 - a12 - a21 + a22)) * phi_weights;
            if (phi0 == phi && thet0 == thet) {
              // -Re((s11 +- s22) * i fext) = Im(s11 +- s22) * fext
              const double sp = s11.i + s22.i, sm = s11.i - s22.i;
              E_(0, 0, jj) = E_(0, 0, jj) + phi0_weights * (fext_i * sp);
              E_(0, 1, jj) = E_(0, 1, jj) + phi0_weights * (fext_i * sm);
              E_(1, 0, jj) = E_(1, 0, jj) + phi0_weights * (fext_i * sm);
              E_(1, 1, jj) = E_(1, 1, jj) + phi0_weights * (fext_i * sp);
            }
          }
          S_(0, ll, 0, jj, kk) += z11 * phi0_weights;
          S_(0, ll, 1, jj, kk) += z12 * phi0_weights;
          S_(1, ll, 0, jj, kk) += z21 * phi0_weights;
          S_(1, ll, 1, jj, kk) += z22 * phi0_weights;
        }
        e11[ll + kk * nummu] = S_(0, ll, 0, jj, kk) * thet_weights * 2.0 * orc::PI;
        e12[ll + kk * nummu] = S_(0, ll, 1, jj, kk) * thet_weights * 2.0 * orc::PI;
      }
    }
    double s11 = 0.0, s12 = 0.0;
    for (int k = 0; k < 2 * nummu; k++) { s11 += e11[k]; s12 += e12[k]; }
    emis[0 + 2 * jj] = E_(0, 0, jj) - s11;
    emis[1 + 2 * jj] = E_(0, 1, jj) - s12;
  }
  return 0;
}

}  // namespace tmo

extern "C" {

// calc_single_tmatrix for one particle (alpha = 0).  mri is the magnitude of
// the imaginary part; returns 0 or 2 (the reference's fatal error).
int TMO_NAME(tmatrix_single)(int nummu, double frequency, double mrr, double mri, double axi, double as_ratio,
                       double beta, double* scat, double* ext, double* emis, double* sback) {
  return tmo::single(nummu, frequency, mrr, std::fabs(mri), axi, as_ratio, 0.0, beta, scat, ext, emis, sback);
}

// The single-precision T-matrix of one particle: returns nmax (0 on error)
// and fills re/im [(nmax+1)][4][nmax][nmax] when cap allows.
int TMO_NAME(tmatrix_tmat)(double lam, double mrr, double mri, double axi, double as_ratio, int cap, float* re,
                     float* im) {
  tmo::TMat T;
  if (tmo::amplq(lam, mrr, std::fabs(mri), axi, as_ratio, T)) return 0;
  const size_t n = T.re.size();
  if ((size_t)cap >= n)
    for (size_t i = 0; i < n; i++) { re[i] = T.re[i]; im[i] = T.im[i]; }
  return T.nmax;
}

// calc_tmatrix (src/tmatrix.f90:14-433) for one species at one frequency:
// bins with ndens = 0 are skipped; ice (phase -1) of density != 917 is mixed
// with air (eps_mix); the equal-volume radius follows the aspect ratio.
// back_spec is the "NN" backscattering per bin, 4 pi ndens Sback(1,1).
int TMO_NAME(tmatrix_species)(int nummu, double frequency, double ref_re, double ref_im, int phase, int nbins,
                        const double* dmax, const double* del_d, const double* ndens, const double* density,
                        const double* as_ratio, const double* canting, double* scat, double* ext, double* emis,
                        double* back_spec, double* sback) {
  const int NS = 2 * (2 * nummu) * (2 * nummu);
  for (int e = 0; e < NS; e++) scat[e] = 0.0;
  for (int e = 0; e < 4 * nummu; e++) ext[e] = 0.0;
  for (int e = 0; e < 2 * nummu; e++) emis[e] = 0.0;
  for (int e = 0; e < 4; e++) sback[e] = 0.0;
  std::vector<double> sp(NS), ep(4 * nummu), mp(2 * nummu);
  for (int ir = 0; ir < nbins; ir++) {
    back_spec[ir] = 0.0;
    const double nd = ndens[ir], dd = del_d[ir];
    if (nd == 0.0) continue;
    if (!(nd > 0.0) || !(dd > 0.0) || !(density[ir] > 0.0)) return 2;
    double mr = ref_re, mi = ref_im;
    if (phase == -1 && density[ir] != 917.0) orc_eps_mix_m(ref_re, ref_im, density[ir], &mr, &mi);
    // mindex = conjg(mMix): the solve takes |Im|
    double axi;
    if (as_ratio[ir] <= 1.0)
      axi = 0.5 * dmax[ir] * std::pow(as_ratio[ir], 1.0 / 3.0);
    else
      axi = 0.5 * dmax[ir] / std::pow(as_ratio[ir], 2.0 / 3.0);
    double sb[4] = {0, 0, 0, 0};
    if (tmo::single(nummu, frequency, mr, std::fabs(-mi), axi, as_ratio[ir], 0.0, canting[ir], sp.data(), ep.data(),
                    mp.data(), sb))
      return 2;
    back_spec[ir] = 4.0 * orc::PI * nd * sb[0];
    for (int e = 0; e < NS; e++) scat[e] = scat[e] + sp[e] * nd * dd;
    for (int e = 0; e < 4 * nummu; e++) ext[e] = ext[e] + ep[e] * nd * dd;
    for (int e = 0; e < 2 * nummu; e++) emis[e] = emis[e] + mp[e] * nd * dd;
    for (int e = 0; e < 4; e++) sback[e] = sback[e] + sb[e] * nd * dd;
  }
  return 0;
}

}  // extern "C"
