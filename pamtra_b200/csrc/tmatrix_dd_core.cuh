// Steps of the double-double T-matrix solve (see tmatrix_dd.cuh), written
// per node, per (n1, n2) pair and per matrix element so that the CTA
// drivers on the device and a serial driver on the host (the CPU test of
// this solve against the REAL*16 oracle) run the same code.  Reference:
// src/tmatrix_amplq.lp.f (CONST :972, QGAUSS :1025, VARY :1114, RSP1 :1194,
// BESS/RJB/RYB/CJB :1342-1524, TMATR0/TMATR :1526-2047, VIG :2049,
// TT :2107).
#pragma once
#include <cmath>

#include "ddreal.cuh"
#include "tmatrix_limits.cuh"

namespace pb {

struct ddc {
  ddr re, im;
};
DDR_FN ddc ddc_of(ddr r, ddr i) { return ddc{r, i}; }
DDR_FN ddc operator+(ddc a, ddc b) { return ddc{a.re + b.re, a.im + b.im}; }
DDR_FN ddc operator-(ddc a, ddc b) { return ddc{a.re - b.re, a.im - b.im}; }
DDR_FN ddc operator*(ddc a, ddc b) { return ddc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
DDR_FN ddc ddc_inv(ddc b) {
  const ddr d = b.re * b.re + b.im * b.im;
  return ddc{b.re / d, (-b.im) / d};
}
DDR_FN ddr ddr_i(int v) { return ddr_of((double)v); }

// Scratch of the solve, in doubles (a ddr is two, a ddc four): node arrays
// x w s ss r dr ddr drr dri v [TM_NG], Bessel tables J Y JR JI DJ DY DJR DJI
// [TM_NG][TM_NMAX], Wigner d1 d2 [TM_NG][TM_NMAX], [Q | I] [TM_N2][2 TM_N2]
// and RgQ [TM_N2][TM_N2] as ddc.
constexpr int TDN_X = 0, TDN_W = 1, TDN_S = 2, TDN_SS = 3, TDN_R = 4, TDN_DR = 5, TDN_DDR = 6, TDN_DRR = 7,
              TDN_DRI = 8, TDN_V = 9;
constexpr size_t TDO_NODE = 0;
constexpr size_t TDO_BES = TDO_NODE + 2 * 10 * (size_t)TM_NG;
constexpr size_t TDO_D = TDO_BES + 2 * 8 * (size_t)TM_NG * TM_NMAX;
constexpr size_t TDO_AUG = TDO_D + 2 * 2 * (size_t)TM_NG * TM_NMAX;
constexpr size_t TDO_RG = TDO_AUG + 4 * (size_t)TM_N2 * 2 * TM_N2;
constexpr size_t TDO_END = TDO_RG + 4 * (size_t)TM_N2 * TM_N2;

DDR_FN ddr* tdd_node(double* sd, int k) { return reinterpret_cast<ddr*>(sd + TDO_NODE) + (size_t)k * TM_NG; }
DDR_FN ddr* tdd_bes(double* sd, int k) {
  return reinterpret_cast<ddr*>(sd + TDO_BES) + (size_t)k * TM_NG * TM_NMAX;
}
DDR_FN ddr* tdd_d(double* sd, int k) { return reinterpret_cast<ddr*>(sd + TDO_D) + (size_t)k * TM_NG * TM_NMAX; }
DDR_FN ddc* tdd_aug(double* sd) { return reinterpret_cast<ddc*>(sd + TDO_AUG); }
DDR_FN ddc* tdd_rg(double* sd) { return reinterpret_cast<ddc*>(sd + TDO_RG); }
DDR_FN ddr tdd_k(double lam) { return ddr_half_pi() * 4.0 / ddr_of(lam); }  // P * 2 / LAM

// QGAUSS: root pair k of the n-point Gauss-Legendre rule, Newton in
// double-double from the double estimate; nodes ascending, weights sum to 2.
DDR_FN void tdd_gauss_pair(double* sd, int n, int k) {
  ddr* xo = tdd_node(sd, TDN_X);
  ddr* wo = tdd_node(sd, TDN_W);
  ddr x = ddr_of(cos(3.141592653589793 * ((double)k + 0.75) / ((double)n + 0.5)));
  ddr dp = ddr_of(1.0);
  for (int it = 0; it < 60; it++) {
    ddr p0 = ddr_of(1.0), p1 = x;
    for (int j = 2; j <= n; j++) {
      const ddr p2 = (ddr_i(2 * j - 1) * x * p1 - ddr_i(j - 1) * p0) / ddr_i(j);
      p0 = p1;
      p1 = p2;
    }
    dp = ddr_i(n) * (x * p1 - p0) / (x * x - ddr_of(1.0));
    const ddr dx = p1 / dp;
    x = x - dx;
    if (fabs(dx.hi) <= 1e-31 * fabs(x.hi) || fabs(dx.hi) < 1e-300) break;
  }
  ddr p0 = ddr_of(1.0), p1 = x;
  for (int j = 2; j <= n; j++) {
    const ddr p2 = (ddr_i(2 * j - 1) * x * p1 - ddr_i(j - 1) * p0) / ddr_i(j);
    p0 = p1;
    p1 = p2;
  }
  dp = ddr_i(n) * (x * p1 - p0) / (x * x - ddr_of(1.0));
  if ((n & 1) && k == (n - 1) / 2) x = ddr_of(0.0);
  const ddr wk = ddr_of(2.0) / ((ddr_of(1.0) - x * x) * dp * dp);
  xo[n - 1 - k] = x;
  wo[n - 1 - k] = wk;
  xo[k] = -x;
  wo[k] = wk;
}

// CONST (1/sin, 1/sin^2) and RSP1 (spheroid r^2, dr/r) at node t < ngauss and its mirror.
DDR_FN void tdd_surface_node(double* sd, int t, int ngauss, double rev_d, double eps_d) {
  const int ng = 2 * ngauss;
  ddr *X = tdd_node(sd, TDN_X), *S = tdd_node(sd, TDN_S), *SS = tdd_node(sd, TDN_SS), *R = tdd_node(sd, TDN_R),
      *DR = tdd_node(sd, TDN_DR);
  const ddr one = ddr_of(1.0), eps = ddr_of(eps_d);
  const ddr c = X[t], cc = c * c, ssv = one - cc, sv = ddr_sqrt(ssv);
  ddr y = one / (one - c * c);
  SS[t] = y;
  SS[ng - 1 - t] = y;
  y = ddr_sqrt(y);
  S[t] = y;
  S[ng - 1 - t] = y;
  const ddr a = ddr_of(rev_d) * ddr_pow(eps, one / ddr_of(3.0));
  const ddr aa = a * a, ee = eps * eps, ee1 = ee - one;
  const ddr rr = one / (ssv + ee * cc);
  R[t] = aa * rr;
  R[ng - 1 - t] = aa * rr;
  DR[t] = rr * c * sv * ee1;
  DR[ng - 1 - t] = -(rr * c * sv * ee1);
}

// VARY at node t < 2 ngauss: size parameter k r and the reciprocals; returns k r in double.
DDR_FN double tdd_size_node(double* sd, int t, double lam, double mrr_d, double mri_d) {
  const ddr one = ddr_of(1.0), mrr = ddr_of(mrr_d), mri = ddr_of(mri_d);
  const ddr v0 = one / (mrr * mrr + mri * mri);
  const ddr prr = mrr * v0, pri = -(mri * v0);
  const ddr vt = ddr_sqrt(tdd_node(sd, TDN_R)[t]) * tdd_k(lam);
  const ddr iv = one / vt;
  tdd_node(sd, TDN_V)[t] = vt;
  tdd_node(sd, TDN_DDR)[t] = iv;
  tdd_node(sd, TDN_DRR)[t] = prr * iv;
  tdd_node(sd, TDN_DRI)[t] = pri * iv;
  return ddr_to_double(vt);
}

// VARY: the downward-recurrence lengths from the largest size parameter ta;
// false where the reference stops (NMAX + NNMAX2 >= 1200).
DDR_FN bool tdd_lengths(double ta, int nmax, double mrr, double mri, int* nnmax1, int* nnmax2) {
  double tb = ta * sqrt(mrr * mrr + mri * mri);
  tb = fmax(tb, (double)nmax);
  if (!(ta > 0.0) || !(tb < (double)TM_LBES)) return false;
  *nnmax1 = (int)(8.0 * sqrt(fmax(ta, (double)nmax)) + 3.0);
  *nnmax2 = (int)(tb + 4.0 * pow(tb, 0.33333) + 8.0 * sqrt(tb)) - nmax + 5;
  return nmax + *nnmax2 < TM_LBES;
}

// BESS at node t: j_n, y_n of k r and j_n of m k r with their u_n (RJB, RYB, CJB).
DDR_FN void tdd_bessel_node(double* sd, int t, int nmax, int nnmax1, int nnmax2, double mrr, double mri) {
  ddr *J = tdd_bes(sd, 0) + (size_t)t * TM_NMAX, *Y = tdd_bes(sd, 1) + (size_t)t * TM_NMAX;
  ddr *JR = tdd_bes(sd, 2) + (size_t)t * TM_NMAX, *JI = tdd_bes(sd, 3) + (size_t)t * TM_NMAX;
  ddr *DJ = tdd_bes(sd, 4) + (size_t)t * TM_NMAX, *DY = tdd_bes(sd, 5) + (size_t)t * TM_NMAX;
  ddr *DJR = tdd_bes(sd, 6) + (size_t)t * TM_NMAX, *DJI = tdd_bes(sd, 7) + (size_t)t * TM_NMAX;
  const ddr one = ddr_of(1.0);
  const ddr x = tdd_node(sd, TDN_V)[t], xr = x * ddr_of(mrr), xi = x * ddr_of(mri);
  ddr sx, cx;
  ddr_sincos(x, sx, cx);
  {  // RJB: ratios j_n / j_{n-1} downward; those of orders <= nmax wait in J
    const int L = nmax + nnmax1;
    const ddr xx = one / x;
    ddr z = one / (ddr_i(2 * L + 1) * xx);
    if (L <= nmax) J[L - 1] = z;
    for (int i1 = L - 1; i1 >= 1; i1--) {
      z = one / (ddr_i(2 * i1 + 1) * xx - z);
      if (i1 <= nmax) J[i1 - 1] = z;
    }
    const ddr z0 = one / (xx - J[0]);
    const ddr y0 = z0 * cx * xx;
    ddr yp = y0 * J[0];
    DJ[0] = y0 - yp * xx;
    J[0] = yp;
    for (int i = 2; i <= nmax; i++) {
      const ddr yi = yp * J[i - 1];
      DJ[i - 1] = yp - ddr_i(i) * yi * xx;
      J[i - 1] = yi;
      yp = yi;
    }
  }
  {  // RYB: y_n upward
    const ddr x1 = one / x, x2 = x1 * x1, x3 = x2 * x1;
    ddr ym = -(cx * x2) - sx * x1;
    Y[0] = ym;
    ddr yc = (x1 - ddr_of(3.0) * x3) * cx - ddr_of(3.0) * x2 * sx;
    if (nmax >= 2) Y[1] = yc;
    for (int i = 2; i <= nmax - 1; i++) {
      const ddr yn = ddr_i(2 * i + 1) * x1 * yc - ym;
      Y[i] = yn;
      ym = yc;
      yc = yn;
    }
    DY[0] = -(x1 * (cx + Y[0]));
    for (int i = 2; i <= nmax; i++) DY[i - 1] = Y[i - 2] - ddr_i(i) * x1 * Y[i - 1];
  }
  {  // CJB: RJB for the complex argument m k r
    const int L = nmax + nnmax2;
    const ddc cxx = ddc_inv(ddc_of(xr, xi));
    ddc z = ddc_of(xr / ddr_i(2 * L + 1), xi / ddr_i(2 * L + 1));
    if (L <= nmax) { JR[L - 1] = z.re; JI[L - 1] = z.im; }
    for (int i1 = L - 1; i1 >= 1; i1--) {
      const ddr qf = ddr_i(2 * i1 + 1);
      z = ddc_inv(ddc_of(qf * cxx.re - z.re, qf * cxx.im - z.im));
      if (i1 <= nmax) { JR[i1 - 1] = z.re; JI[i1 - 1] = z.im; }
    }
    const ddc z0 = ddc_inv(cxx - ddc_of(JR[0], JI[0]));
    ddr sr, cr;
    ddr_sincos(xr, sr, cr);
    const ddc cosz = ddc_of(cr * ddr_cosh(xi), -(sr * ddr_sinh(xi)));
    const ddc y0 = (z0 * cosz) * cxx;
    ddc yp = y0 * ddc_of(JR[0], JI[0]);
    const ddc u1 = y0 - yp * cxx;
    DJR[0] = u1.re;
    DJI[0] = u1.im;
    JR[0] = yp.re;
    JI[0] = yp.im;
    for (int i = 2; i <= nmax; i++) {
      const ddc yv = yp * ddc_of(JR[i - 1], JI[i - 1]);
      const ddc a = yv * cxx;
      DJR[i - 1] = yp.re - ddr_i(i) * a.re;
      DJI[i - 1] = yp.im - ddr_i(i) * a.im;
      JR[i - 1] = yv.re;
      JI[i - 1] = yv.im;
      yp = yv;
    }
  }
}

// VIG at node ngauss + t and its mirror ngauss - 1 - t (t < ngauss): Wigner
// d^n_{0m} and the theta-derivative; the m-factor in single precision as
// the reference's float() forms it.
DDR_FN void tdd_vig_node(double* sd, int t, int ngauss, int nmax, int m) {
  ddr *D1 = tdd_d(sd, 0), *D2 = tdd_d(sd, 1);
  const ddr one = ddr_of(1.0);
  const int i1 = ngauss + t, i2 = ngauss - 1 - t;
  const ddr x = tdd_node(sd, TDN_X)[i1], qs = ddr_sqrt(one - x * x), qs1 = one / qs;
  auto put = [&](int k, ddr d1, ddr d2) {
    const double si = ((k + 1 + m) & 1) ? -1.0 : 1.0;
    D1[(size_t)i1 * TM_NMAX + k] = d1;
    D2[(size_t)i1 * TM_NMAX + k] = d2;
    D1[(size_t)i2 * TM_NMAX + k] = d1 * si;
    D2[(size_t)i2 * TM_NMAX + k] = -(d2 * si);
  };
  if (m == 0) {
    ddr d1 = one, d2 = x;
    for (int n = 1; n <= nmax; n++) {
      const ddr qn = ddr_i(n), qn1 = ddr_i(n + 1), qn2 = ddr_i(2 * n + 1);
      const ddr d3 = (qn2 * x * d2 - qn * d1) / qn1;
      const ddr der = qs1 * (qn1 * qn / qn2) * (d3 - d1);
      put(n - 1, d2, der);
      d1 = d2;
      d2 = d3;
    }
    return;
  }
  for (int n = 1; n < m && n <= nmax; n++) put(n - 1, ddr_of(0.0), ddr_of(0.0));
  const ddr qmm = ddr_i(m * m);
  ddr a = one;
  for (int i = 1; i <= m; i++) a = a * (double)sqrtf((float)(2 * i - 1) / (float)(2 * i)) * qs;
  ddr d1 = ddr_of(0.0), d2 = a;
  for (int n = m; n <= nmax; n++) {
    const ddr qn = ddr_i(n), qn2 = ddr_i(2 * n + 1), qn1 = ddr_i(n + 1);
    const ddr qnm = ddr_sqrt(qn * qn - qmm), qnm1 = ddr_sqrt(qn1 * qn1 - qmm);
    const ddr d3 = (qn2 * x * d2 - qnm * d1) / qnm1;
    const ddr der = qs1 * (qn * qnm1 * d3 - qn1 * qnm * d1) / qn2;
    put(n - 1, d2, der);
    d1 = d2;
    d2 = d3;
  }
}

// TMATR0 / TMATR (NCHECK = 1) for pair pr of order m: the surface integrals
// of (n1, n2) over the ngauss nodes of one half, the block phases, and the
// entries of [Q | I] (rows k1, K1) and RgQ.
DDR_FN void tdd_pair(double* sd, int pr, int m, int nmax, int ngauss, double lam, double mrr_d, double mri_d) {
  const int mm1 = (m == 0) ? 1 : m, nm = nmax - mm1 + 1, n2m = 2 * nm, ldw = 2 * n2m;
  const int n1 = mm1 + pr / nm, n2 = mm1 + pr % nm;
  const ddr *W = tdd_node(sd, TDN_W), *S = tdd_node(sd, TDN_S), *SS = tdd_node(sd, TDN_SS),
            *R = tdd_node(sd, TDN_R), *DR = tdd_node(sd, TDN_DR), *DDR = tdd_node(sd, TDN_DDR),
            *DRR = tdd_node(sd, TDN_DRR), *DRI = tdd_node(sd, TDN_DRI);
  const ddr *J = tdd_bes(sd, 0), *Y = tdd_bes(sd, 1), *JR = tdd_bes(sd, 2), *JI = tdd_bes(sd, 3),
            *DJ = tdd_bes(sd, 4), *DY = tdd_bes(sd, 5), *DJR = tdd_bes(sd, 6), *DJI = tdd_bes(sd, 7);
  const ddr *D1 = tdd_d(sd, 0), *D2 = tdd_d(sd, 1);
  const ddr kq = tdd_k(lam);
  const ddr ppi = kq * kq, pir = ppi * ddr_of(mrr_d), pii = ppi * ddr_of(mri_d);
  const ddr qm = ddr_i(m), qmm = ddr_i(m * m);
  const ddr an1 = ddr_i(n1 * (n1 + 1)), an2 = ddr_i(n2 * (n2 + 1));
  const ddc zero = ddc_of(ddr_of(0.0), ddr_of(0.0));
  const bool even = ((n1 + n2) & 1) == 0;
  ddc a11 = zero, a12 = zero, a21 = zero, a22 = zero, g11 = zero, g12 = zero, g21 = zero, g22 = zero;
  auto acc = [](ddc& a, ddr f1, ddc x, ddr f2, ddc y) {
    a = ddc_of(a.re + f1 * x.re + f2 * y.re, a.im + f1 * x.im + f2 * y.im);
  };
  if (!(m == 0 && !even)) {
    for (int i = 0; i < ngauss; i++) {
      const size_t o1 = (size_t)i * TM_NMAX + n1 - 1, o2 = (size_t)i * TM_NMAX + n2 - 1;
      const ddr d1n1 = D1[o1], d2n1 = D2[o1], d1n2 = D1[o2], d2n2 = D2[o2];
      const ddr e11 = d1n1 * d1n2, e12 = d1n1 * d2n2, e21 = d2n1 * d1n2, e22 = d2n1 * d2n2;
      const ddr qj1 = J[o1], qy1 = Y[o1], qdj1 = DJ[o1], qdy1 = DY[o1];
      const ddr qjr2 = JR[o2], qji2 = JI[o2], qdjr2 = DJR[o2], qdji2 = DJI[o2];
      // c: j_n(kr) j_n(mkr); b: h_n(kr) j_n(mkr)
      const ddc c1 = ddc_of(qjr2 * qj1, qji2 * qj1), b1 = ddc_of(c1.re - qji2 * qy1, c1.im + qjr2 * qy1);
      const ddc c2 = ddc_of(qjr2 * qdj1, qji2 * qdj1), b2 = ddc_of(c2.re - qji2 * qdy1, c2.im + qjr2 * qdy1);
      const ddr ddri = DDR[i];
      const ddc c3 = ddc_of(ddri * c1.re, ddri * c1.im), b3 = ddc_of(ddri * b1.re, ddri * b1.im);
      const ddc c4 = ddc_of(qdjr2 * qj1, qdji2 * qj1), b4 = ddc_of(c4.re - qdji2 * qy1, c4.im + qdjr2 * qy1);
      const ddc dm = ddc_of(DRR[i], DRI[i]);
      const ddc c5 = c1 * dm, b5 = b1 * dm;
      const ddr uri = DR[i], wr = W[i] * R[i];
      if (m == 0 || even) {
        const ddr f1 = (m == 0) ? wr * e22 : wr * (e11 * (SS[i] * qmm) + e22);
        acc(a12, f1, b2, wr * uri * an1 * e12, b3);
        acc(g12, f1, c2, wr * uri * an1 * e12, c3);
        acc(a21, f1, b4, wr * uri * an2 * e21, b5);
        acc(g21, f1, c4, wr * uri * an2 * e21, c5);
      } else {
        const ddc c6 = ddc_of(qdjr2 * qdj1, qdji2 * qdj1), b6 = ddc_of(c6.re - qdji2 * qdy1, c6.im + qdjr2 * qdy1);
        const ddc c7 = ddc_of(c4.re * ddri, c4.im * ddri), b7 = ddc_of(b4.re * ddri, b4.im * ddri);
        const ddc c8 = c2 * dm, b8 = b2 * dm;
        const ddr dsi = S[i] * qm * wr;
        const ddr e1 = dsi * (e12 + e21);
        a11 = ddc_of(a11.re + e1 * b1.re, a11.im + e1 * b1.im);
        g11 = ddc_of(g11.re + e1 * c1.re, g11.im + e1 * c1.im);
        const ddr e2b = dsi * uri * e11;
        const ddr e3 = e2b * an2, e2 = e2b * an1;
        a22 = ddc_of(a22.re + e1 * b6.re + e2 * b7.re + e3 * b8.re, a22.im + e1 * b6.im + e2 * b7.im + e3 * b8.im);
        g22 = ddc_of(g22.re + e1 * c6.re + e2 * c7.re + e3 * c8.re, g22.im + e1 * c6.im + e2 * c7.im + e3 * c8.im);
      }
    }
  }
  const double dd1 = (double)sqrtf((float)(2 * n1 + 1) / (float)(n1 * (n1 + 1)));
  const double dd2 = (double)sqrtf((float)(2 * n2 + 1) / (float)(n2 * (n2 + 1)));
  const ddr an12 = ddr_two_prod(dd1, dd2);  // ANN(n1, n2) * 2 = d(n1) d(n2) * 0.5 * 2
  auto sc = [&](ddc v) { return ddc_of(v.re * an12, v.im * an12); };
  // block phases: T11 = -X11, T12 = -i X12, T21 = i X21, T22 = -X22
  auto ph = [](int blk, ddc v) -> ddc {
    if (blk == 0 || blk == 3) return ddc_of(-v.re, -v.im);
    if (blk == 1) return ddc_of(v.im, -v.re);
    return ddc_of(-v.im, v.re);
  };
  const ddc t11 = ph(0, sc(a11)), t12 = ph(1, sc(a12)), t21 = ph(2, sc(a21)), t22 = ph(3, sc(a22));
  const ddc q11 = ph(0, sc(g11)), q12 = ph(1, sc(g12)), q21 = ph(2, sc(g21)), q22 = ph(3, sc(g22));
  auto comb = [&](ddc x, ddc y) {
    return ddc_of(pir * x.re - pii * x.im + ppi * y.re, pir * x.im + pii * x.re + ppi * y.im);
  };
  ddc* aug = tdd_aug(sd);
  ddc* rg = tdd_rg(sd);
  const int k1 = n1 - mm1, k2 = n2 - mm1, K1 = k1 + nm, K2 = k2 + nm;
  auto put = [&](int r, int c, ddc qv, ddc gv) {
    aug[(size_t)r * ldw + c] = qv;
    rg[(size_t)r * n2m + c] = gv;
  };
  put(k1, k2, comb(t21, t12), comb(q21, q12));
  put(K1, K2, comb(t12, t21), comb(q12, q21));
  if (m == 0) {
    put(k1, K2, zero, zero);
    put(K1, k2, zero, zero);
  } else {
    put(k1, K2, comb(t11, t22), comb(q11, q22));
    put(K1, k2, comb(t22, t11), comb(q22, q11));
  }
}

// The identity half of [Q | I], element e < n2m^2.
DDR_FN void tdd_identity(double* sd, int e, int n2m) {
  const int r = e / n2m, c = e % n2m;
  tdd_aug(sd)[(size_t)r * (2 * n2m) + n2m + c] = ddc_of(ddr_of(r == c ? 1.0 : 0.0), ddr_of(0.0));
}
// Pivot key of row r in column c (the largest |re| + |im| is chosen, the lowest row on ties).
DDR_FN double tdd_pivot_key(double* sd, int r, int c, int n2m) {
  const ddc v = tdd_aug(sd)[(size_t)r * (2 * n2m) + c];
  return fabs(v.re.hi) + fabs(v.im.hi);
}
DDR_FN ddc tdd_pivot_inverse(double* sd, int pr, int c, int n2m) {
  return ddc_inv(tdd_aug(sd)[(size_t)pr * (2 * n2m) + c]);
}
// Swap rows c and pr and scale the pivot row, column j >= c.
DDR_FN void tdd_swap_scale(double* sd, int c, int pr, int j, int n2m, ddc ip) {
  ddc* aug = tdd_aug(sd);
  const size_t ldw = 2 * (size_t)n2m;
  const ddc vp = aug[(size_t)pr * ldw + j];
  if (pr != c) aug[(size_t)pr * ldw + j] = aug[(size_t)c * ldw + j];
  aug[(size_t)c * ldw + j] = vp * ip;
}
// Eliminate column c from row r, element e of the (rows) x (columns > c) update.
DDR_FN void tdd_elim(double* sd, int c, int e, int n2m) {
  ddc* aug = tdd_aug(sd);
  const int ldw = 2 * n2m, wcols = ldw - c - 1;
  const int r = e / wcols, j = c + 1 + e % wcols;
  if (r == c) return;
  const ddc f = aug[(size_t)r * ldw + c];
  if (f.re.hi == 0.0 && f.im.hi == 0.0) return;
  aug[(size_t)r * ldw + j] = aug[(size_t)r * ldw + j] - f * aug[(size_t)c * ldw + j];
}
// TT: T(i, j) = -sum_k RgQ(i, k) Q^-1(k, j) accumulated in double over k in
// order, element e < n2m^2; T(i, j) goes to tout[2 (j 2 n2m + n2m + i)] (re, im),
// where the FP64 solve of tmatrix.cuh leaves it.
DDR_FN void tdd_product(double* sd, double* tout, int e, int n2m) {
  const ddc* aug = tdd_aug(sd);
  const ddc* rg = tdd_rg(sd);
  const int i = e / n2m, j = e % n2m;
  double tr = 0.0, ti = 0.0;
  for (int k = 0; k < n2m; k++) {
    const ddc g = rg[(size_t)i * n2m + k], q = aug[(size_t)k * (2 * n2m) + n2m + j];
    const double arr = ddr_to_double(g.re), ari = ddr_to_double(g.im);
    const double ar = ddr_to_double(q.re), ai = ddr_to_double(q.im);
    tr = tr - arr * ar + ari * ai;
    ti = ti - arr * ai - ari * ar;
  }
  const size_t o = 2 * ((size_t)j * (2 * n2m) + n2m + i);
  tout[o] = tr;
  tout[o + 1] = ti;
}

}  // namespace pb
