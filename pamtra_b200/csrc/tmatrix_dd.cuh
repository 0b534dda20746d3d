// Double-double solve of the T-matrix for bins outside the FP64 envelope
// (large, strongly aspherical liquid drops), following the reference's
// REAL*16 tmatrix_amplq (src/tmatrix_amplq.lp.f): nodes, surface, Bessel
// tables, surface integrals and the inverse of Q in double-double
// (ddreal.cuh), then T = -RgQ Q^-1 accumulated in double over k = 1..2 nm as
// the reference's TT (:2107-2153) does.  Same CTA organisation as the FP64
// solve in tmatrix.cuh (one bin per CTA, 256 threads, one node or (n1, n2)
// pair per thread, Gauss-Jordan with warp 0 choosing the pivot); the working
// set takes twice the doubles in the CTA's scratch slot.
//
// Not yet included in the library: it joins k_tmatrix (per bin, chosen by
// size parameter, index and aspect ratio) together with its GPU parity run
// against the REAL*16 oracle.  Its double-double twin on the CPU
// (oracle/dd.h) reproduces the REAL*16 single-precision T-matrix where FP64
// fails.
#pragma once
#include "common.cuh"
#include "ddreal.cuh"
#include "tmatrix.cuh"

namespace pb {

struct ddc {
  ddr re, im;
};
__device__ __forceinline__ ddc ddc_of(ddr r, ddr i) { return ddc{r, i}; }
__device__ __forceinline__ ddc operator+(ddc a, ddc b) { return ddc{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ ddc operator-(ddc a, ddc b) { return ddc{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ ddc operator*(ddc a, ddc b) {
  return ddc{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ ddc ddc_inv(ddc b) {
  const ddr d = b.re * b.re + b.im * b.im;
  return ddc{b.re / d, (-b.im) / d};
}
__device__ __forceinline__ ddr ddr_i(int v) { return ddr_of((double)v); }

// Scratch of the double-double solve, in doubles (a ddr is two), after the
// CTA's FP64 slot (which keeps the single-precision T and the angular work):
// nodes x w s ss r dr ddr drr dri [TM_NG], Bessel tables J Y JR JI DJ DY DJR
// DJI [TM_NG][TM_NMAX], Wigner d1 d2 [TM_NG][TM_NMAX], the augmented system
// [Q^T | I] and -RgQ [TM_N2][TM_N2] as ddc.
constexpr size_t TDO_NODE = 0;
constexpr size_t TDO_BES = TDO_NODE + 2 * 9 * (size_t)TM_NG;
constexpr size_t TDO_D = TDO_BES + 2 * 8 * (size_t)TM_NG * TM_NMAX;
constexpr size_t TDO_AUG = TDO_D + 2 * 2 * (size_t)TM_NG * TM_NMAX;
constexpr size_t TDO_RG = TDO_AUG + 4 * (size_t)TM_N2 * 2 * TM_N2;
constexpr size_t TDO_END = TDO_RG + 4 * (size_t)TM_N2 * TM_N2;

__device__ __forceinline__ ddr* tdd_node(double* s, int k) {
  return reinterpret_cast<ddr*>(s + TDO_NODE) + (size_t)k * TM_NG;
}
__device__ __forceinline__ ddr* tdd_bes(double* s, int k) {
  return reinterpret_cast<ddr*>(s + TDO_BES) + (size_t)k * TM_NG * TM_NMAX;
}
__device__ __forceinline__ ddr* tdd_d(double* s, int k) {
  return reinterpret_cast<ddr*>(s + TDO_D) + (size_t)k * TM_NG * TM_NMAX;
}
__device__ __forceinline__ ddc* tdd_aug(double* s) { return reinterpret_cast<ddc*>(s + TDO_AUG); }
__device__ __forceinline__ ddc* tdd_rg(double* s) { return reinterpret_cast<ddc*>(s + TDO_RG); }

// Gauss-Legendre root pair k of order n by Newton in double-double from the
// double estimate (QGAUSS, tmatrix_amplq.lp.f:1025-1112).
__device__ void tdd_gauss_pair(int n, int k, ddr* x_out, ddr* w_out) {
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
  x_out[n - 1 - k] = x;
  w_out[n - 1 - k] = wk;
  x_out[k] = -x;
  w_out[k] = wk;
}

// CONST + RSP1 + VARY + BESS in double-double (tmatrix_amplq.lp.f:972-1023,
// :1194-1225, :1114-1192, :1342-1524).  sd: the double-double scratch.
// Whole CTA; false when the reference would stop (NMAX + NNMAX2 >= 1200).
__device__ bool tdd_setup(double* sd, TmShared& sh, int nmax, int ngauss, double lam, double mrr_d, double mri_d,
                          double rev_d, double eps_d) {
  const int t = threadIdx.x, ng = 2 * ngauss;
  ddr *X = tdd_node(sd, 0), *W = tdd_node(sd, 1), *S = tdd_node(sd, 2), *SS = tdd_node(sd, 3), *R = tdd_node(sd, 4),
      *DR = tdd_node(sd, 5), *DDR = tdd_node(sd, 6), *DRR = tdd_node(sd, 7), *DRI = tdd_node(sd, 8);
  if (t < (ng + 1) / 2) tdd_gauss_pair(ng, t, X, W);
  __syncthreads();
  const ddr one = ddr_of(1.0);
  const ddr mrr = ddr_of(mrr_d), mri = ddr_of(mri_d), eps = ddr_of(eps_d);
  const ddr kq = ddr_half_pi() * 4.0 / ddr_of(lam);  // P * 2 / LAM
  if (t < ngauss) {
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
  __syncthreads();
  const ddr v0 = one / (mrr * mrr + mri * mri);
  const ddr prr = mrr * v0, pri = -(mri * v0);
  ddr vt = ddr_of(0.0);
  if (t < ng) {
    vt = ddr_sqrt(R[t]) * kq;
    const ddr iv = one / vt;
    DDR[t] = iv;
    DRR[t] = prr * iv;
    DRI[t] = pri * iv;
  }
  // the recurrence lengths only need double
  double ta = ddr_to_double(vt);
  for (int o = 16; o > 0; o >>= 1) ta = fmax(ta, __shfl_xor_sync(0xffffffffu, ta, o));
  if ((t & 31) == 0) sh.accs[t >> 5] = ta;
  __syncthreads();
  ta = 0.0;
  for (int w = 0; w < TM_THREADS / 32; w++) ta = fmax(ta, sh.accs[w]);
  double tb = ta * sqrt(mrr_d * mrr_d + mri_d * mri_d);
  tb = fmax(tb, (double)nmax);
  if (!(ta > 0.0) || !(tb < (double)TM_LBES)) {
    __syncthreads();
    return false;
  }
  const int nnmax1 = (int)(8.0 * sqrt(fmax(ta, (double)nmax)) + 3.0);
  int nnmax2 = (int)(tb + 4.0 * pow(tb, 0.33333) + 8.0 * sqrt(tb));
  nnmax2 = nnmax2 - nmax + 5;
  __syncthreads();
  if (nmax + nnmax2 >= TM_LBES) return false;
  if (t < ng) {
    ddr *J = tdd_bes(sd, 0) + (size_t)t * TM_NMAX, *Y = tdd_bes(sd, 1) + (size_t)t * TM_NMAX;
    ddr *JR = tdd_bes(sd, 2) + (size_t)t * TM_NMAX, *JI = tdd_bes(sd, 3) + (size_t)t * TM_NMAX;
    ddr *DJ = tdd_bes(sd, 4) + (size_t)t * TM_NMAX, *DY = tdd_bes(sd, 5) + (size_t)t * TM_NMAX;
    ddr *DJR = tdd_bes(sd, 6) + (size_t)t * TM_NMAX, *DJI = tdd_bes(sd, 7) + (size_t)t * TM_NMAX;
    const ddr x = vt, xr = vt * mrr, xi = vt * mri;
    ddr sx, cx;
    ddr_sincos(x, sx, cx);
    // RJB: ratios j_n / j_{n-1} downward; those of orders <= nmax wait in J
    {
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
    // RYB: y_n upward
    {
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
    // CJB: RJB for the complex argument m k r
    {
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
  __syncthreads();
  return true;
}

// TMATR0 / TMATR with NCHECK = 1 and TT in double-double for order m
// (tmatrix_amplq.lp.f:1526-2153): Wigner tables, surface integrals, Q and
// RgQ, the inverse of Q by Gauss-Jordan on [Q | I], and T = -RgQ Q^-1
// accumulated in double over k = 1..2 nm (the reference's TT).  T goes where
// the FP64 solve leaves it (tm_tget of the FP64 slot s), so the convergence
// sums and the single-precision storage of k_tmatrix read it unchanged.
// Whole CTA; returns 2 nm, or 0 when a pivot vanishes.
__device__ int tdd_solve(double* s, double* sd, TmShared& sh, int m, int nmax, int ngauss, double lam, double mrr_d,
                         double mri_d) {
  const int t = threadIdx.x;
  const int mm1 = (m == 0) ? 1 : m, nm = nmax - mm1 + 1, n2m = 2 * nm, ldw = 2 * n2m;
  const ddr one = ddr_of(1.0);
  const ddr* X = tdd_node(sd, 0);
  ddr *D1 = tdd_d(sd, 0), *D2 = tdd_d(sd, 1);
  if (t < ngauss) {
    // VIG (:2049-2105) in double-double; the m-factor in single precision as float() forms it
    const int i1 = ngauss + t, i2 = ngauss - 1 - t;
    const ddr x = X[i1], qs = ddr_sqrt(one - x * x), qs1 = one / qs;
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
    } else {
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
  }
  __syncthreads();
  const ddr *W = tdd_node(sd, 1), *S = tdd_node(sd, 2), *SS = tdd_node(sd, 3), *R = tdd_node(sd, 4),
            *DR = tdd_node(sd, 5), *DDR = tdd_node(sd, 6), *DRR = tdd_node(sd, 7), *DRI = tdd_node(sd, 8);
  const ddr *J = tdd_bes(sd, 0), *Y = tdd_bes(sd, 1), *JR = tdd_bes(sd, 2), *JI = tdd_bes(sd, 3),
            *DJ = tdd_bes(sd, 4), *DY = tdd_bes(sd, 5), *DJR = tdd_bes(sd, 6), *DJI = tdd_bes(sd, 7);
  ddc* aug = tdd_aug(sd);
  ddc* rg = tdd_rg(sd);
  const ddr kq = ddr_half_pi() * 4.0 / ddr_of(lam);
  const ddr ppi = kq * kq, pir = ppi * ddr_of(mrr_d), pii = ppi * ddr_of(mri_d);
  const ddr qm = ddr_i(m), qmm = ddr_i(m * m);
  const ddc zero = ddc_of(ddr_of(0.0), ddr_of(0.0));
  for (int pr = t; pr < nm * nm; pr += TM_THREADS) {
    const int n1 = mm1 + pr / nm, n2 = mm1 + pr % nm;
    const ddr an1 = ddr_i(n1 * (n1 + 1)), an2 = ddr_i(n2 * (n2 + 1));
    const bool even = ((n1 + n2) & 1) == 0;
    ddc a11 = zero, a12 = zero, a21 = zero, a22 = zero, g11 = zero, g12 = zero, g21 = zero, g22 = zero;
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
        auto acc = [](ddc& a, ddr f1, ddc x, ddr f2, ddc y) {
          a = ddc_of(a.re + f1 * x.re + f2 * y.re, a.im + f1 * x.im + f2 * y.im);
        };
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
    const int k1 = n1 - mm1, k2 = n2 - mm1, K1 = k1 + nm, K2 = k2 + nm;
    // aug row r = [Q(r, :) | I(r, :)]; rg row-major RgQ
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
  for (int e = t; e < n2m * n2m; e += TM_THREADS) {
    const int r = e / n2m, c = e % n2m;
    aug[(size_t)r * ldw + n2m + c] = ddc_of(ddr_of(r == c ? 1.0 : 0.0), ddr_of(0.0));
  }
  __syncthreads();
  // Gauss-Jordan on [Q | I]: the right half becomes Q^-1
  for (int c = 0; c < n2m; c++) {
    if (t < 32) {
      double best = -1.0;
      int br = c;
      for (int r = c + t; r < n2m; r += 32) {
        const ddc v = aug[(size_t)r * ldw + c];
        const double a = fabs(v.re.hi) + fabs(v.im.hi);
        if (a > best) { best = a; br = r; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int orr = __shfl_xor_sync(0xffffffffu, br, o);
        if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
      }
      if (t == 0) sh.pivrow = (best > 0.0) ? br : -1;
    }
    __syncthreads();
    const int pr = sh.pivrow;
    if (pr < 0) return 0;
    const ddc ip = ddc_inv(aug[(size_t)pr * ldw + c]);
    __syncthreads();
    for (int j = c + t; j < ldw; j += TM_THREADS) {
      const ddc vp = aug[(size_t)pr * ldw + j];
      if (pr != c) aug[(size_t)pr * ldw + j] = aug[(size_t)c * ldw + j];
      aug[(size_t)c * ldw + j] = vp * ip;
    }
    __syncthreads();
    const int wcols = ldw - c - 1;
    for (int e = t; e < n2m * wcols; e += TM_THREADS) {
      const int r = e / wcols, j = c + 1 + e % wcols;
      if (r == c) continue;
      const ddc f = aug[(size_t)r * ldw + c];
      if (f.re.hi == 0.0 && f.im.hi == 0.0) continue;
      aug[(size_t)r * ldw + j] = aug[(size_t)r * ldw + j] - f * aug[(size_t)c * ldw + j];
    }
    __syncthreads();
  }
  // T(i, j) = -sum_k RgQ(i, k) Q^-1(k, j), accumulated in double as TT does
  cplx* tout = tm_aug(s);
  for (int e = t; e < n2m * n2m; e += TM_THREADS) {
    const int i = e / n2m, j = e % n2m;
    double tr = 0.0, ti = 0.0;
    for (int k = 0; k < n2m; k++) {
      const ddc g = rg[(size_t)i * n2m + k], q = aug[(size_t)k * ldw + n2m + j];
      const double arr = ddr_to_double(g.re), ari = ddr_to_double(g.im);
      const double ar = ddr_to_double(q.re), ai = ddr_to_double(q.im);
      tr = tr - arr * ar + ari * ai;
      ti = ti - arr * ai - ari * ar;
    }
    tout[(size_t)j * (2 * n2m) + n2m + i] = cmk(tr, ti);  // where tm_tget(s, n2m, i, j) reads
  }
  __syncthreads();
  return n2m;
}

}  // namespace pb
