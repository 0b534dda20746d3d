// T-matrix scattering of spheroids (scat_name 'tmatrix', src/tmatrix.f90 and
// the extended-precision EBCM code src/tmatrix_amplq.lp.f of the reference).
//
// One persistent CTA (256 threads) carries one particle (bin) at a time
// through the whole computation, in FP64, with its working set in a slot of
// global scratch that stays in L1 / L2:
//   1. the convergence of NMAX and then of the Gauss points on the m = 0
//      extinction and scattering sums (tmatrix_amplq.lp.f:386-470), each
//      step a full m = 0 solve: Gauss-Legendre nodes (one root pair per
//      thread), spheroid surface and spherical Bessel tables (one node per
//      thread, downward ratio recurrences), the EBCM surface integrals (one
//      (n1, n2) pair per thread) assembled into [Q^T | -RgQ^T], and a
//      Gauss-Jordan elimination with partial pivoting that leaves T^T;
//   2. the m >= 1 blocks (TMATR, :1765-2047), each one more solve;
//   3. the T-matrix stored in single precision, as the reference stores it
//      (REAL*4 common /TMAT/), and the amplitude matrices of 30 scattering
//      azimuths for every pair of Lobatto angles (calc_single_tmatrix,
//      src/tmatrix.f90:436-684).  For an upright particle (canting 0) the
//      polar parts of the amplitude sum do not depend on the azimuth: per
//      incident angle and order m the kernel forms the eight vectors
//      (CAL o T_xy) d0 once, dots them with the scattered angles' Wigner
//      vectors, and sums the 30 azimuths from those (30x fewer products than
//      evaluating AMPL per azimuth).  A canted particle takes the AMPL
//      evaluation per (incident angle, scattered angle, azimuth).
// The reference computes the solve in REAL*16; FP64 here agrees with it to
// about 1e-12 relative on microwave hydrometeors, below the single-precision
// storage of T.  The normalisation factors the reference forms in
// single-precision float() arithmetic (CONST, VIG) are formed the same way.
#pragma once
#include "common.cuh"
#include "mie.cuh"  // eps_mix_m
#include "tmatrix_limits.cuh"

namespace pb {
static_assert(TM_NG <= TM_THREADS, "one Gauss node per thread");

// Scratch slot of one CTA, in doubles.
constexpr size_t TMO_NODE = 0;                                   // x w s ss r dr ddr drr dri [TM_NG]
constexpr size_t TMO_BES = TMO_NODE + 9 * (size_t)TM_NG;          // J Y JR JI DJ DY DJR DJI [TM_NG][TM_NMAX]
constexpr size_t TMO_D = TMO_BES + 8 * (size_t)TM_NG * TM_NMAX;   // d1 d2 [TM_NG][TM_NMAX]
constexpr size_t TMO_AUG = TMO_D + 2 * (size_t)TM_NG * TM_NMAX;   // [TM_N2][2 TM_N2] complex
constexpr size_t TMO_P = TMO_AUG + 2 * (size_t)TM_N2 * 2 * TM_N2; // [TM_NMAX+1][TM_NA][4] complex
constexpr size_t TMO_DVA = TMO_P + 2 * (size_t)(TM_NMAX + 1) * TM_NA * 4;  // [TM_NA][2][TM_NMAX]
constexpr size_t TMO_Z = TMO_DVA + (size_t)TM_NA * 2 * TM_NMAX;   // [TM_NA][TM_NAZ][4]
constexpr size_t TM_DIRD = 7;                                     // doubles of one direction record
constexpr size_t TMO_G = TMO_Z + (size_t)TM_NA * TM_NAZ * 4;      // incident [32], scattered [TM_NA][TM_NAZ]
constexpr size_t TMO_T = TMO_G + (32 + (size_t)TM_NA * TM_NAZ) * TM_DIRD;  // float2 [TM_NMAX+1][4][TM_NMAX][TM_NMAX]
constexpr size_t TM_T_FLOAT2 = (size_t)(TM_NMAX + 1) * 4 * TM_NMAX * TM_NMAX;
constexpr size_t TM_SLOT_DOUBLES = TMO_T + TM_T_FLOAT2;          // a float2 is one double wide

// Inputs and outputs of one launch: particle p = item * nbins + bin.
struct TmArgs {
  int n_items, nbins, nummu;
  const double* freq;      // [item] Hz
  const double* mrr;       // [item * nbins + bin] real part of the index used
  const double* mri;       // [item * nbins + bin] |imaginary part|
  const double* axi;       // [particle] equal-volume-sphere radius (m)
  const double* asr;       // [particle] aspect ratio
  const double* beta;      // [particle] canting angle (deg)
  const double* ndens;     // [particle] 0 = no particle
  const double* mu;        // Lobatto angles [nummu]
  const double* wq;        // Lobatto weights [nummu]
  double* scat;            // [particle][2 nummu 2 nummu 2] (Fortran order of scatter_matrix)
  double* ext;             // [particle][2 2 nummu]
  double* emis;            // [particle][2 nummu]
  double* sback;           // [particle][2 2]
  int* nmax;               // [particle] converged NMAX (0 when skipped)
  int* status;             // [particle]
  double* scratch;         // [slots][TM_SLOT_DOUBLES]
  int* counter;            // persistent work counter (zeroed before the launch)
};

struct TmShared {
  double accs[8];
  int iv[8];
  double u[8][TM_NMAX][2];   // (CAL o T_xy) p0 / q0 of the current incident angle and m
  double dv0[2][TM_NMAX];    // m d0/sin and d0' at the incident angle
  double piv[2];
  double cth[TM_NA];         // particle-frame polar cosines of the scattered angles
  double thet[TM_NA];        // scattered polar angles (deg) as calc_single_tmatrix forms them
  int pivrow;
  int particle;
};

__device__ __forceinline__ double* tm_node(double* s, int k) { return s + TMO_NODE + (size_t)k * TM_NG; }
__device__ __forceinline__ double* tm_bes(double* s, int k) { return s + TMO_BES + (size_t)k * TM_NG * TM_NMAX; }
__device__ __forceinline__ double* tm_d(double* s, int k) { return s + TMO_D + (size_t)k * TM_NG * TM_NMAX; }
__device__ __forceinline__ cplx* tm_aug(double* s) { return reinterpret_cast<cplx*>(s + TMO_AUG); }
__device__ __forceinline__ float2* tm_t(double* s) { return reinterpret_cast<float2*>(s + TMO_T); }
__device__ __forceinline__ size_t tm_tidx(int nmax, int m, int blk, int n1, int n2) {
  return (((size_t)m * 4 + blk) * nmax + (n1 - 1)) * nmax + (n2 - 1);
}

// Gauss-Legendre root pair k of order n (ascending nodes on [-1, 1], weights
// summing to 2) by Newton iteration on the three-term recurrence (QGAUSS,
// tmatrix_amplq.lp.f:1025-1112).
__device__ void tm_gauss_pair(int n, int k, double* x_out, double* w_out) {
  double x = cos(3.141592653589793 * ((double)k + 0.75) / ((double)n + 0.5));
  double dp = 1.0;
  for (int it = 0; it < 100; it++) {
    double p0 = 1.0, p1 = x;
    for (int j = 2; j <= n; j++) {
      const double p2 = ((double)(2 * j - 1) * x * p1 - (double)(j - 1) * p0) / (double)j;
      p0 = p1;
      p1 = p2;
    }
    dp = (double)n * (x * p1 - p0) / (x * x - 1.0);
    const double dx = p1 / dp;
    x -= dx;
    if (fabs(dx) <= 1.0e-16 * fabs(x) || fabs(dx) < 1.0e-300) break;
  }
  double p0 = 1.0, p1 = x;
  for (int j = 2; j <= n; j++) {
    const double p2 = ((double)(2 * j - 1) * x * p1 - (double)(j - 1) * p0) / (double)j;
    p0 = p1;
    p1 = p2;
  }
  dp = (double)n * (x * p1 - p0) / (x * x - 1.0);
  if ((n & 1) && k == (n - 1) / 2) x = 0.0;
  const double wk = 2.0 / ((1.0 - x * x) * dp * dp);
  x_out[n - 1 - k] = x;
  w_out[n - 1 - k] = wk;
  x_out[k] = -x;
  w_out[k] = wk;
}

// VIG (tmatrix_amplq.lp.f:2049-2105): d^n_{0m}(x) and its theta-derivative
// for n = 1..nmax, written through the callback at n - 1.  The m-factor
// prod sqrt((2i-1)/(2i)) is formed in single precision as the reference's
// float() does.
template <class F>
__device__ __forceinline__ void tm_vig(double x, int nmax, int m, F&& put) {
  const double qs = sqrt(1.0 - x * x), qs1 = 1.0 / qs;
  if (m == 0) {
    double d1 = 1.0, d2 = x;
    for (int n = 1; n <= nmax; n++) {
      const double qn = n, qn1 = n + 1, qn2 = 2 * n + 1;
      const double d3 = (qn2 * x * d2 - qn * d1) / qn1;
      const double der = qs1 * (qn1 * qn / qn2) * (-d1 + d3);
      put(n - 1, d2, der);
      d1 = d2;
      d2 = d3;
    }
    return;
  }
  for (int n = 1; n < m && n <= nmax; n++) put(n - 1, 0.0, 0.0);
  const double qmm = (double)(m * m);
  double a = 1.0;
  for (int i = 1; i <= m; i++) a = a * (double)sqrtf((float)(2 * i - 1) / (float)(2 * i)) * qs;
  double d1 = 0.0, d2 = a;
  for (int n = m; n <= nmax; n++) {
    const double qn = n, qn2 = 2 * n + 1, qn1 = n + 1;
    const double qnm = sqrt(qn * qn - qmm), qnm1 = sqrt(qn1 * qn1 - qmm);
    const double d3 = (qn2 * x * d2 - qnm * d1) / qnm1;
    const double der = qs1 * (-qn1 * qnm * d1 + qn * qnm1 * d3) / qn2;
    put(n - 1, d2, der);
    d1 = d2;
    d2 = d3;
  }
}

// CONST + RSP1 + VARY + BESS (tmatrix_amplq.lp.f:972-1023, :1194-1225,
// :1114-1192, :1342-1524) for NP = -1: nodes, surface, size parameters and
// the Bessel tables.  Whole CTA; returns false when the reference would stop
// (NMAX + NNMAX2 >= 1200).
__device__ bool tm_setup(double* s, TmShared& sh, int nmax, int ngauss, double lam, double mrr, double mri, double rev,
                         double eps) {
  const int t = threadIdx.x, ng = 2 * ngauss;
  double *X = tm_node(s, 0), *W = tm_node(s, 1), *S = tm_node(s, 2), *SS = tm_node(s, 3), *R = tm_node(s, 4),
         *DR = tm_node(s, 5), *DDR = tm_node(s, 6), *DRR = tm_node(s, 7), *DRI = tm_node(s, 8);
  if (t < (ng + 1) / 2) tm_gauss_pair(ng, t, X, W);
  __syncthreads();
  const double pi = 2.0 * 3.141592653589793 / lam;  // k (P * 2 / LAM)
  if (t < ngauss) {
    const double c = X[t], cc = c * c, ssv = 1.0 - cc, sv = sqrt(ssv);
    double y = 1.0 / (1.0 - c * c);
    SS[t] = y;
    SS[ng - 1 - t] = y;
    y = sqrt(y);
    S[t] = y;
    S[ng - 1 - t] = y;
    const double a = rev * pow(eps, 1.0 / 3.0);
    const double aa = a * a, ee = eps * eps, ee1 = ee - 1.0;
    const double rr = 1.0 / (ssv + ee * cc);
    R[t] = aa * rr;
    R[ng - 1 - t] = aa * rr;
    DR[t] = rr * c * sv * ee1;
    DR[ng - 1 - t] = -(rr * c * sv * ee1);
  }
  __syncthreads();
  // size parameters and the recurrence lengths (max over the nodes)
  const double v0 = 1.0 / (mrr * mrr + mri * mri);
  const double prr = mrr * v0, pri = -mri * v0;
  double vt = 0.0;
  if (t < ng) {
    vt = sqrt(R[t]) * pi;
    const double iv = 1.0 / vt;
    DDR[t] = iv;
    DRR[t] = prr * iv;
    DRI[t] = pri * iv;
  }
  double ta = vt;
  for (int o = 16; o > 0; o >>= 1) ta = fmax(ta, __shfl_xor_sync(0xffffffffu, ta, o));
  if ((t & 31) == 0) sh.accs[t >> 5] = ta;
  __syncthreads();
  ta = 0.0;
  for (int w = 0; w < TM_THREADS / 32; w++) ta = fmax(ta, sh.accs[w]);
  double tb = ta * sqrt(mrr * mrr + mri * mri);
  tb = fmax(tb, (double)nmax);
  // bounded recurrence lengths for any input (the reference stops at 1200)
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
    double *J = tm_bes(s, 0) + (size_t)t * TM_NMAX, *Y = tm_bes(s, 1) + (size_t)t * TM_NMAX;
    double *JR = tm_bes(s, 2) + (size_t)t * TM_NMAX, *JI = tm_bes(s, 3) + (size_t)t * TM_NMAX;
    double *DJ = tm_bes(s, 4) + (size_t)t * TM_NMAX, *DY = tm_bes(s, 5) + (size_t)t * TM_NMAX;
    double *DJR = tm_bes(s, 6) + (size_t)t * TM_NMAX, *DJI = tm_bes(s, 7) + (size_t)t * TM_NMAX;
    const double x = vt, xr = vt * mrr, xi = vt * mri;
    // RJB: z_n = j_n / j_{n-1} downward from nmax + nnmax1; the ratios of
    // orders <= nmax wait in J until the upward pass replaces them
    {
      const int L = nmax + nnmax1;
      const double xx = 1.0 / x;
      double z = 1.0 / ((double)(2 * L + 1) * xx);
      if (L <= nmax) J[L - 1] = z;
      for (int i1 = L - 1; i1 >= 1; i1--) {
        z = 1.0 / ((double)(2 * i1 + 1) * xx - z);
        if (i1 <= nmax) J[i1 - 1] = z;
      }
      const double z0 = 1.0 / (xx - J[0]);
      const double y0 = z0 * cos(x) * xx;
      double yp = y0 * J[0];
      DJ[0] = y0 - yp * xx;
      J[0] = yp;
      for (int i = 2; i <= nmax; i++) {
        const double yi = yp * J[i - 1];
        DJ[i - 1] = yp - (double)i * yi * xx;
        J[i - 1] = yi;
        yp = yi;
      }
    }
    // RYB: y_n upward
    {
      const double c = cos(x), sn = sin(x), x1 = 1.0 / x, x2 = x1 * x1, x3 = x2 * x1;
      double ym = -c * x2 - sn * x1;
      Y[0] = ym;
      double yc = (-3.0 * x3 + x1) * c - 3.0 * x2 * sn;
      if (nmax >= 2) Y[1] = yc;
      for (int i = 2; i <= nmax - 1; i++) {
        const double yn = (double)(2 * i + 1) * x1 * yc - ym;
        Y[i] = yn;
        ym = yc;
        yc = yn;
      }
      DY[0] = -x1 * (c + Y[0]);
      for (int i = 2; i <= nmax; i++) DY[i - 1] = Y[i - 2] - (double)i * x1 * Y[i - 1];
    }
    // CJB: RJB for the complex argument m k r
    {
      const int L = nmax + nnmax2;
      const double xrxi = 1.0 / (xr * xr + xi * xi);
      const double cxr = xr * xrxi, cxi = -xi * xrxi;
      double zr = xr / (double)(2 * L + 1), zi = xi / (double)(2 * L + 1);
      if (L <= nmax) { JR[L - 1] = zr; JI[L - 1] = zi; }
      for (int i1 = L - 1; i1 >= 1; i1--) {
        const double qf = (double)(2 * i1 + 1);
        const double ar = qf * cxr - zr, ai = qf * cxi - zi;
        const double ari = 1.0 / (ar * ar + ai * ai);
        zr = ar * ari;
        zi = -ai * ari;
        if (i1 <= nmax) { JR[i1 - 1] = zr; JI[i1 - 1] = zi; }
      }
      double ar = cxr - JR[0], ai = cxi - JI[0];
      double ari = 1.0 / (ar * ar + ai * ai);
      const double z0r = ar * ari, z0i = -ai * ari;
      const double cr = cos(xr) * cosh(xi), ci = -sin(xr) * sinh(xi);
      ar = z0r * cr - z0i * ci;
      ai = z0i * cr + z0r * ci;
      const double y0r = ar * cxr - ai * cxi, y0i = ai * cxr + ar * cxi;
      double ypr = y0r * JR[0] - y0i * JI[0], ypi = y0i * JR[0] + y0r * JI[0];
      ar = ypr * cxr - ypi * cxi;
      ai = ypi * cxr + ypr * cxi;
      DJR[0] = y0r - ar;
      DJI[0] = y0i - ai;
      JR[0] = ypr;
      JI[0] = ypi;
      for (int i = 2; i <= nmax; i++) {
        const double zr2 = JR[i - 1], zi2 = JI[i - 1];
        const double yr = ypr * zr2 - ypi * zi2, yi = ypi * zr2 + ypr * zi2;
        ar = yr * cxr - yi * cxi;
        ai = yi * cxr + yr * cxi;
        DJR[i - 1] = ypr - (double)i * ar;
        DJI[i - 1] = ypi - (double)i * ai;
        JR[i - 1] = yr;
        JI[i - 1] = yi;
        ypr = yr;
        ypi = yi;
      }
    }
  }
  __syncthreads();
  return true;
}

// TMATR0 / TMATR (tmatrix_amplq.lp.f:1526-2047) with NCHECK = 1 for order m:
// Wigner tables on the nodes, the surface integrals of every (n1, n2) pair
// (the blocks of one (n1 + n2) parity only), Q and RgQ assembled transposed
// into [Q^T | -RgQ^T], and T = -RgQ Q^-1 (TT, :2107-2153) by Gauss-Jordan
// elimination with partial pivoting: afterwards row j of the right half
// holds column j of T.  Whole CTA; returns the order of the system (2 nm),
// or 0 when a pivot vanishes.
__device__ int tm_solve(double* s, TmShared& sh, int m, int nmax, int ngauss, double ppi, double pir, double pii) {
  const int t = threadIdx.x;
  const int mm1 = (m == 0) ? 1 : m, nm = nmax - mm1 + 1, n2m = 2 * nm, ldw = 2 * n2m;
  const double* X = tm_node(s, 0);
  double *D1 = tm_d(s, 0), *D2 = tm_d(s, 1);
  if (t < ngauss) {
    const int i1 = ngauss + t, i2 = ngauss - 1 - t;
    tm_vig(X[i1], nmax, m, [&](int k, double d1, double d2) {
      const double si = ((k + 1 + m) & 1) ? -1.0 : 1.0;
      D1[(size_t)i1 * TM_NMAX + k] = d1;
      D2[(size_t)i1 * TM_NMAX + k] = d2;
      D1[(size_t)i2 * TM_NMAX + k] = d1 * si;
      D2[(size_t)i2 * TM_NMAX + k] = -d2 * si;
    });
  }
  __syncthreads();
  const double *W = tm_node(s, 1), *S = tm_node(s, 2), *SS = tm_node(s, 3), *R = tm_node(s, 4), *DR = tm_node(s, 5),
               *DDR = tm_node(s, 6), *DRR = tm_node(s, 7), *DRI = tm_node(s, 8);
  const double *J = tm_bes(s, 0), *Y = tm_bes(s, 1), *JR = tm_bes(s, 2), *JI = tm_bes(s, 3), *DJ = tm_bes(s, 4),
               *DY = tm_bes(s, 5), *DJR = tm_bes(s, 6), *DJI = tm_bes(s, 7);
  cplx* aug = tm_aug(s);
  const double qm = m, qmm = (double)(m * m);
  for (int pr = t; pr < nm * nm; pr += TM_THREADS) {
    const int n1 = mm1 + pr / nm, n2 = mm1 + pr % nm;
    const double an1 = (double)(n1 * (n1 + 1)), an2 = (double)(n2 * (n2 + 1));
    const bool even = ((n1 + n2) & 1) == 0;
    double a11r = 0, a11i = 0, a12r = 0, a12i = 0, a21r = 0, a21i = 0, a22r = 0, a22i = 0;
    double g11r = 0, g11i = 0, g12r = 0, g12i = 0, g21r = 0, g21i = 0, g22r = 0, g22i = 0;
    if (!(m == 0 && !even)) {
      for (int i = 0; i < ngauss; i++) {
        const size_t o1 = (size_t)i * TM_NMAX + n1 - 1, o2 = (size_t)i * TM_NMAX + n2 - 1;
        const double d1n1 = D1[o1], d2n1 = D2[o1], d1n2 = D1[o2], d2n2 = D2[o2];
        const double e11 = d1n1 * d1n2, e12 = d1n1 * d2n2, e21 = d2n1 * d1n2, e22 = d2n1 * d2n2;
        const double qj1 = J[o1], qy1 = Y[o1], qdj1 = DJ[o1], qdy1 = DY[o1];
        const double qjr2 = JR[o2], qji2 = JI[o2], qdjr2 = DJR[o2], qdji2 = DJI[o2];
        const double c1r = qjr2 * qj1, c1i = qji2 * qj1, b1r = c1r - qji2 * qy1, b1i = c1i + qjr2 * qy1;
        const double c2r = qjr2 * qdj1, c2i = qji2 * qdj1, b2r = c2r - qji2 * qdy1, b2i = c2i + qjr2 * qdy1;
        const double ddri = DDR[i];
        const double c3r = ddri * c1r, c3i = ddri * c1i, b3r = ddri * b1r, b3i = ddri * b1i;
        const double c4r = qdjr2 * qj1, c4i = qdji2 * qj1, b4r = c4r - qdji2 * qy1, b4i = c4i + qdjr2 * qy1;
        const double drri = DRR[i], drii = DRI[i];
        const double c5r = c1r * drri - c1i * drii, c5i = c1i * drri + c1r * drii;
        const double b5r = b1r * drri - b1i * drii, b5i = b1i * drri + b1r * drii;
        const double uri = DR[i], wr = W[i] * R[i];
        if (m == 0 || even) {
          const double f1 = (m == 0) ? wr * e22 : wr * (e11 * (SS[i] * qmm) + e22);
          double f2 = wr * uri * an1 * e12;
          a12r = a12r + f1 * b2r + f2 * b3r;
          a12i = a12i + f1 * b2i + f2 * b3i;
          g12r = g12r + f1 * c2r + f2 * c3r;
          g12i = g12i + f1 * c2i + f2 * c3i;
          f2 = wr * uri * an2 * e21;
          a21r = a21r + f1 * b4r + f2 * b5r;
          a21i = a21i + f1 * b4i + f2 * b5i;
          g21r = g21r + f1 * c4r + f2 * c5r;
          g21i = g21i + f1 * c4i + f2 * c5i;
        } else {
          const double c6r = qdjr2 * qdj1, c6i = qdji2 * qdj1, b6r = c6r - qdji2 * qdy1, b6i = c6i + qdjr2 * qdy1;
          const double c7r = c4r * ddri, c7i = c4i * ddri, b7r = b4r * ddri, b7i = b4i * ddri;
          const double c8r = c2r * drri - c2i * drii, c8i = c2i * drri + c2r * drii;
          const double b8r = b2r * drri - b2i * drii, b8i = b2i * drri + b2r * drii;
          const double dsi = S[i] * qm * wr;
          const double e1 = dsi * (e12 + e21);
          a11r = a11r + e1 * b1r;
          a11i = a11i + e1 * b1i;
          g11r = g11r + e1 * c1r;
          g11i = g11i + e1 * c1i;
          double e2 = dsi * uri * e11;
          const double e3 = e2 * an2;
          e2 = e2 * an1;
          a22r = a22r + e1 * b6r + e2 * b7r + e3 * b8r;
          a22i = a22i + e1 * b6i + e2 * b7i + e3 * b8i;
          g22r = g22r + e1 * c6r + e2 * c7r + e3 * c8r;
          g22i = g22i + e1 * c6i + e2 * c7i + e3 * c8i;
        }
      }
    }
    // ANN(n1, n2) * 2 with the single-precision normalisation of CONST
    const double dd1 = (double)sqrtf((float)(2 * n1 + 1) / (float)(n1 * (n1 + 1)));
    const double dd2 = (double)sqrtf((float)(2 * n2 + 1) / (float)(n2 * (n2 + 1)));
    const double an12 = dd1 * dd2 * 0.5 * 2.0;
    // block phases: T11 = -X11, T12 = -i X12, T21 = i X21, T22 = -X22
    const cplx t11 = cmk(-a11r * an12, -a11i * an12), g11 = cmk(-g11r * an12, -g11i * an12);
    const cplx t12 = cmk(a12i * an12, -a12r * an12), g12 = cmk(g12i * an12, -g12r * an12);
    const cplx t21 = cmk(-a21i * an12, a21r * an12), g21 = cmk(-g21i * an12, g21r * an12);
    const cplx t22 = cmk(-a22r * an12, -a22i * an12), g22 = cmk(-g22r * an12, -g22i * an12);
    auto comb = [&](cplx x, cplx y) {
      return cmk(pir * x.re - pii * x.im + ppi * y.re, pir * x.im + pii * x.re + ppi * y.im);
    };
    const int k1 = n1 - mm1, k2 = n2 - mm1, K1 = k1 + nm, K2 = k2 + nm;
    // Q(r, c) goes to aug[c][r]; -RgQ(r, c) to aug[c][n2m + r]
    auto put = [&](int r, int c, cplx qv, cplx gv) {
      aug[(size_t)c * ldw + r] = qv;
      aug[(size_t)c * ldw + n2m + r] = cmk(-gv.re, -gv.im);
    };
    put(k1, k2, comb(t21, t12), comb(g21, g12));
    put(K1, K2, comb(t12, t21), comb(g12, g21));
    if (m == 0) {
      put(k1, K2, cmk(0, 0), cmk(0, 0));
      put(K1, k2, cmk(0, 0), cmk(0, 0));
    } else {
      put(k1, K2, comb(t11, t22), comb(g11, g22));
      put(K1, k2, comb(t22, t11), comb(g22, g11));
    }
  }
  __syncthreads();
  // Gauss-Jordan on the n2m x 2 n2m augmented system
  for (int c = 0; c < n2m; c++) {
    if (t < 32) {
      double best = -1.0;
      int br = c;
      for (int r = c + t; r < n2m; r += 32) {
        const cplx v = aug[(size_t)r * ldw + c];
        const double a = fabs(v.re) + fabs(v.im);
        if (a > best) { best = a; br = r; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int orr = __shfl_xor_sync(0xffffffffu, br, o);
        if (ob > best || (ob == best && orr < br)) { best = ob; br = orr; }
      }
      if (t == 0) {
        sh.pivrow = (best > 0.0) ? br : -1;
        if (best > 0.0) {
          const cplx p = aug[(size_t)br * ldw + c];
          const double d = p.re * p.re + p.im * p.im;
          sh.piv[0] = p.re / d;
          sh.piv[1] = -p.im / d;
        }
      }
    }
    __syncthreads();
    const int pr = sh.pivrow;
    if (pr < 0) return 0;
    const cplx ip = cmk(sh.piv[0], sh.piv[1]);
    // swap rows c and pr and scale the pivot row (columns >= c)
    for (int j = c + t; j < ldw; j += TM_THREADS) {
      const cplx vp = aug[(size_t)pr * ldw + j];
      if (pr != c) aug[(size_t)pr * ldw + j] = aug[(size_t)c * ldw + j];
      aug[(size_t)c * ldw + j] = cmul(vp, ip);
    }
    __syncthreads();
    // eliminate column c from every other row (columns > c)
    const int wcols = ldw - c - 1;
    for (int e = t; e < n2m * wcols; e += TM_THREADS) {
      const int r = e / wcols, j = c + 1 + e % wcols;
      if (r == c) continue;
      const cplx f = aug[(size_t)r * ldw + c];
      if (f.re == 0.0 && f.im == 0.0) continue;
      const cplx v = aug[(size_t)c * ldw + j];
      cplx& a = aug[(size_t)r * ldw + j];
      a = csub(a, cmul(f, v));
    }
    __syncthreads();
  }
  return n2m;
}

// T(r, c) of the last solve (r, c 0-based in [0, 2 nm)).
__device__ __forceinline__ cplx tm_tget(double* s, int n2m, int r, int c) {
  return tm_aug(s)[(size_t)c * (2 * n2m) + n2m + r];
}

// VIGAMPL (tmatrix_amplq.lp.f:890-970): d^n_{0m}(x) / sin (dv1) and the
// theta-derivative (dv2) in double, with the pole values for m = 1.
template <class F>
__device__ __forceinline__ void tm_vigampl(double x, int nmax, int m, F&& put) {
  if (fabs(1.0 - fabs(x)) <= 1e-10) {
    for (int n = 1; n <= nmax; n++) {
      if (m != 1) { put(n - 1, 0.0, 0.0); continue; }
      double dn = 0.5 * sqrt((double)(n * (n + 1)));
      if (x < 0.0) dn = dn * (((n + 1) & 1) ? -1.0 : 1.0);
      const double v1 = dn;
      if (x < 0.0) dn = -dn;
      put(n - 1, v1, dn);
    }
    return;
  }
  const double qs = sqrt(1.0 - x * x), qs1 = 1.0 / qs, dsi = qs1;
  if (m == 0) {
    double d1 = 1.0, d2 = x;
    for (int n = 1; n <= nmax; n++) {
      const double qn = n, qn1 = n + 1, qn2 = 2 * n + 1;
      const double d3 = (qn2 * x * d2 - qn * d1) / qn1;
      const double der = qs1 * (qn1 * qn / qn2) * (-d1 + d3);
      put(n - 1, d2 * dsi, der);
      d1 = d2;
      d2 = d3;
    }
    return;
  }
  for (int n = 1; n < m && n <= nmax; n++) put(n - 1, 0.0, 0.0);
  const double qmm = (double)(m * m);
  double a = 1.0;
  for (int i = 1; i <= m; i++) a = a * sqrt((double)(2 * i - 1) / (double)(2 * i)) * qs;
  double d1 = 0.0, d2 = a;
  for (int n = m; n <= nmax; n++) {
    const double qn = n, qn2 = 2 * n + 1, qn1 = n + 1;
    const double qnm = sqrt(qn * qn - qmm), qnm1 = sqrt(qn1 * qn1 - qmm);
    const double d3 = (qn2 * x * d2 - qnm * d1) / qnm1;
    const double der = qs1 * (-qn1 * qnm * d1 + qn * qnm1 * d3) / qn2;
    put(n - 1, d2 * dsi, der);
    d1 = d2;
    d2 = d3;
  }
}

// Geometry of AMPL (tmatrix_amplq.lp.f:618-795) for one direction (polar tl,
// azimuth pl in degrees, with the reference's 1e-8 offsets away from the
// singular values): the particle-frame polar cosine, the particle-frame
// azimuth and the lab -> particle polarisation rotation, inverted for the
// scattered direction.  The incident and the scattered direction go through
// the same steps in the reference, so a table of each (per incident angle,
// per scattered angle and azimuth) gives the values of every AMPL call.
struct TmDir {
  double ctp, phip, M[2][2];
};
__device__ void tm_dir(double tl, double pl, double alpha, double beta, bool invert, TmDir& d) {
  const double pin = 3.141592653589793, pin2 = pin * 0.5, pi = pin / 180.0;
  const double alph = alpha * pi;
  double bet = beta * pi, thetl = tl * pi, phil = pl * pi;
  const double eps = 1e-8;
  if (thetl < pin2) thetl = thetl + eps;
  if (thetl > pin2) thetl = thetl - eps;
  if (phil < pin) phil = phil + eps;
  if (phil > pin) phil = phil - eps;
  if (bet <= pin2 && pin2 - bet <= eps) bet = bet - eps;
  if (bet > pin2 && bet - pin2 <= eps) bet = bet + eps;
  const double cb = cos(bet), sb = sin(bet);
  double ct = cos(thetl), st = sin(thetl), cp = cos(phil - alph), sp = sin(phil - alph);
  const double ctp = ct * cb + st * sb * cp, thetp = acos(ctp);
  const double cpp = cb * st * cp - sb * ct, spp = st * sp;
  double phip = atan(spp / cpp);
  if (phip > 0.0 && sp < 0.0) phip = phip + pin;
  if (phip < 0.0 && sp > 0.0) phip = phip + pin;
  if (phip < 0.0) phip = phip + 2.0 * pin;
  const double ca = cos(alph), sa = sin(alph);
  const double B[3][3] = {{ca * cb, sa * cb, -sb}, {-sa, ca, 0.0}, {ca * sb, sa * sb, cb}};
  cp = cos(phil);
  sp = sin(phil);
  const double AL[3][2] = {{ct * cp, -sp}, {ct * sp, cp}, {-st, 0.0}};
  ct = ctp;
  st = sin(thetp);
  cp = cos(phip);
  sp = sin(phip);
  const double AP[2][3] = {{ct * cp, ct * sp, -st}, {-sp, cp, 0.0}};
  double C[3][2], R[2][2];
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      double x = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) x = x + B[i][k] * AL[k][j];
      C[i][j] = x;
    }
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      double x = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) x = x + AP[i][k] * C[k][j];
      R[i][j] = x;
    }
  if (invert) {
    const double dd = 1.0 / (R[0][0] * R[1][1] - R[0][1] * R[1][0]);
    d.M[0][0] = R[1][1] * dd;
    d.M[0][1] = -R[0][1] * dd;
    d.M[1][0] = -R[1][0] * dd;
    d.M[1][1] = R[0][0] * dd;
  } else {
    d.M[0][0] = R[0][0];
    d.M[0][1] = R[0][1];
    d.M[1][0] = R[1][0];
    d.M[1][1] = R[1][1];
  }
  d.ctp = ctp;
  d.phip = phip;
}

struct TmGeom {
  double ctp, ctp1, ph, R[2][2], R1[2][2];
};
__device__ __forceinline__ void tm_geom_of(const TmDir& in, const TmDir& sc, TmGeom& g) {
  g.ctp = in.ctp;
  g.ctp1 = sc.ctp;
  g.ph = sc.phip - in.phip;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++) {
      g.R[i][j] = in.M[i][j];
      g.R1[i][j] = sc.M[i][j];
    }
}

// The particle-frame amplitudes (VV, VH, HV, HH) / k rotated to the lab
// frame (tmatrix_amplq.lp.f:868-885).
__device__ __forceinline__ void tm_rotate(const TmGeom& g, double dk, cplx& vv, cplx& vh, cplx& hv, cplx& hh) {
  vv = cmk(vv.re / dk, vv.im / dk);
  vh = cmk(vh.re / dk, vh.im / dk);
  hv = cmk(hv.re / dk, hv.im / dk);
  hh = cmk(hh.re / dk, hh.im / dk);
  const cplx cvv = cadd(cscale(vv, g.R[0][0]), cscale(vh, g.R[1][0]));
  const cplx cvh = cadd(cscale(vv, g.R[0][1]), cscale(vh, g.R[1][1]));
  const cplx chv = cadd(cscale(hv, g.R[0][0]), cscale(hh, g.R[1][0]));
  const cplx chh = cadd(cscale(hv, g.R[0][1]), cscale(hh, g.R[1][1]));
  vv = cadd(cscale(cvv, g.R1[0][0]), cscale(chv, g.R1[0][1]));
  vh = cadd(cscale(cvh, g.R1[0][0]), cscale(chh, g.R1[0][1]));
  hv = cadd(cscale(cvv, g.R1[1][0]), cscale(chv, g.R1[1][1]));
  hh = cadd(cscale(cvh, g.R1[1][0]), cscale(chh, g.R1[1][1]));
}

// CAL(n, nn) = i^(nn - n - 1) sqrt((2n+1)(2nn+1) / (n nn (n+1)(nn+1))).
__device__ __forceinline__ cplx tm_cal(int n, int nn) {
  double dnn = (double)((2 * n + 1) * (2 * nn + 1));
  dnn = dnn / (double)(n * nn * (n + 1) * (nn + 1));
  const double rn = sqrt(dnn);
  switch (((nn - n - 1) % 4 + 4) % 4) {
    case 0: return cmk(rn, 0.0);
    case 1: return cmk(0.0, rn);
    case 2: return cmk(-rn, 0.0);
    default: return cmk(0.0, -rn);
  }
}

// AMPL (tmatrix_amplq.lp.f:602-888) evaluated in full for one geometry from
// the single-precision T-matrix: the path of canted particles.
__device__ void tm_ampl_full(const float2* T, int nmax, const TmGeom& g, double dk, cplx& vv, cplx& vh, cplx& hv,
                             cplx& hh) {
  double dv1[TM_NMAX], dv2[TM_NMAX], dv01[TM_NMAX], dv02[TM_NMAX];
  vv = vh = hv = hh = cmk(0.0, 0.0);
  for (int m = 0; m <= nmax; m++) {
    const int nmin = max(m, 1);
    tm_vigampl(g.ctp1, nmax, m, [&](int k, double a, double b) { dv1[k] = a; dv2[k] = b; });
    tm_vigampl(g.ctp, nmax, m, [&](int k, double a, double b) { dv01[k] = a; dv02[k] = b; });
    const double fc = 2.0 * cos(m * g.ph), fs = 2.0 * sin(m * g.ph);
    for (int nn = nmin; nn <= nmax; nn++) {
      const double dv1nn = m * dv01[nn - 1], dv2nn = dv02[nn - 1];
      for (int n = nmin; n <= nmax; n++) {
        const double dv1n = m * dv1[n - 1], dv2n = dv2[n - 1];
        const float2 f11 = T[tm_tidx(nmax, m, 0, n, nn)], f22 = T[tm_tidx(nmax, m, 3, n, nn)];
        const cplx ct11 = cmk(f11.x, f11.y), ct22 = cmk(f22.x, f22.y);
        const cplx cl = tm_cal(n, nn);
        if (m == 0) {
          const cplx cn = cscale(cscale(cl, dv2n), dv2nn);
          vv = cadd(vv, cmul(cn, ct22));
          hh = cadd(hh, cmul(cn, ct11));
        } else {
          const float2 f12 = T[tm_tidx(nmax, m, 1, n, nn)], f21 = T[tm_tidx(nmax, m, 2, n, nn)];
          const cplx ct12 = cmk(f12.x, f12.y), ct21 = cmk(f21.x, f21.y);
          const cplx cn1 = cscale(cl, fc), cn2 = cscale(cl, fs);
          const double d11 = dv1n * dv1nn, d12 = dv1n * dv2nn, d21 = dv2n * dv1nn, d22 = dv2n * dv2nn;
          auto q4 = [&](double x11, double x21, double x12, double x22) {
            return cadd(cadd(cadd(cscale(ct11, x11), cscale(ct21, x21)), cscale(ct12, x12)), cscale(ct22, x22));
          };
          vv = cadd(vv, cmul(q4(d11, d21, d12, d22), cn1));
          vh = cadd(vh, cmul(q4(d12, d22, d11, d21), cn2));
          hv = csub(hv, cmul(q4(d21, d11, d22, d12), cn2));
          hh = cadd(hh, cmul(q4(d22, d12, d21, d11), cn1));
        }
      }
    }
  }
  tm_rotate(g, dk, vv, vh, hv, hh);
}

// One particle: the converged T-matrix, then calc_single_tmatrix's angular
// sums into this particle's slices of the outputs.  Whole CTA.
__device__ void tm_particle(const TmArgs& A, double* s, TmShared& sh, int p) {
  const int t = threadIdx.x, nummu = A.nummu, na = 2 * nummu;
  const size_t NS = (size_t)2 * nummu * 2 * nummu * 2;
  double* scat = A.scat + (size_t)p * NS;
  double* ext = A.ext + (size_t)p * 4 * nummu;
  double* emis = A.emis + (size_t)p * 2 * nummu;
  double* sback = A.sback + (size_t)p * 4;
  for (size_t e = t; e < NS; e += TM_THREADS) scat[e] = 0.0;
  for (int e = t; e < 4 * nummu; e += TM_THREADS) ext[e] = 0.0;
  for (int e = t; e < 2 * nummu; e += TM_THREADS) emis[e] = 0.0;
  if (t < 4) sback[t] = 0.0;
  if (A.ndens[p] == 0.0) {
    if (t == 0) A.nmax[p] = 0;
    return;
  }
  const int item = p / A.nbins;
  const double lam = C_LIGHT / A.freq[item];
  const double wave_num = 2.0 * PI / lam;
  const double mrr = A.mrr[p], mri = A.mri[p], axi = A.axi[p], asr = A.asr[p], beta = A.beta[p];
  const double eps = 1.0 / asr, rev = 1.0 * axi;
  const double kq = 2.0 * 3.141592653589793 / lam, ppi = kq * kq, pir = ppi * mrr, pii = ppi * mri;
  const double xev = 2.0 * 3.141592653589793 * rev / lam;
  const int inm1 = max(4, (int)(xev + 4.05 * pow(xev, 0.333333)));
  int fail = 0, nmax = 0, ngauss = 0, n2m = 0;
  double qext1 = 0.0, qsca1 = 0.0;
  auto conv_sums = [&](double& qext, double& qsca) {
    if (t == 0) {
      double qe = 0.0, qs = 0.0;
      for (int k = 1; k <= nmax; k++) {
        const cplx a = tm_tget(s, n2m, k - 1, k - 1), b = tm_tget(s, n2m, k - 1 + nmax, k - 1 + nmax);
        const double dn1 = (double)(2 * k + 1);
        qs = qs + dn1 * (a.re * a.re + a.im * a.im + b.re * b.re + b.im * b.im);
        qe = qe + (a.re + b.re) * dn1;
      }
      sh.accs[0] = qe;
      sh.accs[1] = qs;
    }
    __syncthreads();
    qext = sh.accs[0];
    qsca = sh.accs[1];
    __syncthreads();
  };
  // NMAX convergence (tmatrix_amplq.lp.f:386-431)
  bool conv = false;
  for (nmax = inm1; nmax <= TM_NMAX; nmax++) {
    ngauss = 2 * nmax;
    if (ngauss > TM_NGAUSS || !tm_setup(s, sh, nmax, ngauss, lam, mrr, mri, rev, eps)) { fail = 1; break; }
    n2m = tm_solve(s, sh, 0, nmax, ngauss, ppi, pir, pii);
    if (!n2m) { fail = 1; break; }
    double qext, qsca;
    conv_sums(qext, qsca);
    const double dsca = fabs((qsca1 - qsca) / qsca), dext = fabs((qext1 - qext) / qext);
    qext1 = qext;
    qsca1 = qsca;
    if (dsca <= 0.001 && dext <= 0.001) { conv = true; break; }
  }
  if (!conv) fail = 1;
  // Gauss-point convergence (:432-470): at least one more node pair
  if (!fail) {
    for (int ng2 = ngauss + 1;; ng2++) {
      if (ng2 > TM_NGAUSS) { fail = 1; break; }
      ngauss = ng2;
      if (!tm_setup(s, sh, nmax, ngauss, lam, mrr, mri, rev, eps)) { fail = 1; break; }
      n2m = tm_solve(s, sh, 0, nmax, ngauss, ppi, pir, pii);
      if (!n2m) { fail = 1; break; }
      double qext, qsca;
      conv_sums(qext, qsca);
      const double dsca = fabs((qsca1 - qsca) / qsca), dext = fabs((qext1 - qext) / qext);
      qext1 = qext;
      qsca1 = qsca;
      if (dsca <= 0.001 && dext <= 0.001) break;
    }
  }
  if (fail) {
    if (t == 0) { A.nmax[p] = -nmax; A.status[p] |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_RANGE; }
    return;
  }
  // single-precision T of every order m (:472-556)
  float2* T = tm_t(s);
  for (int m = 0; m <= nmax; m++) {
    if (m > 0) {
      n2m = tm_solve(s, sh, m, nmax, ngauss, ppi, pir, pii);
      if (!n2m) { fail = 1; break; }
    }
    const int nm = n2m / 2, off = (m == 0) ? 0 : m - 1;
    for (int e = t; e < nm * nm; e += TM_THREADS) {
      const int n1 = e / nm, n2 = e % nm;
      const int r[4] = {n1, n1, n1 + nm, n1 + nm}, c[4] = {n2, n2 + nm, n2, n2 + nm};
#pragma unroll
      for (int b = 0; b < 4; b++) {
        const cplx v = tm_tget(s, n2m, r[b], c[b]);
        T[tm_tidx(nmax, m, b, n1 + 1 + off, n2 + 1 + off)] = make_float2((float)v.re, (float)v.im);
      }
    }
    __syncthreads();
  }
  if (fail) {
    if (t == 0) { A.nmax[p] = -nmax; A.status[p] |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_RANGE; }
    return;
  }
  // ---------------- calc_single_tmatrix angular sums (tmatrix.f90:560-680)
  const double fact_sca = 0.5 / (wave_num * wave_num);
  const double fext = 2.0 * PI / (wave_num * wave_num);
  const double phi_weights = 1.0 / 360.0 * (360.0 / TM_NAZ);
  const bool upright = (beta == 0.0);
  const double dk = 2.0 * 3.141592653589793 / lam;
  double* Zb = s + TMO_Z;
  cplx* P = reinterpret_cast<cplx*>(s + TMO_P);
  double* DVA = s + TMO_DVA;
  TmDir* Gin = reinterpret_cast<TmDir*>(s + TMO_G);
  TmDir* Gsc = Gin + 32;
  if (t < na) {
    const int kk = t / nummu, ll = t % nummu;
    double th = acos(A.mu[ll] * (kk == 0 ? 1.0 : -1.0)) * 180.0 / PI;
    if (th > 179.9999) th = 180.0;
    sh.thet[t] = th;
  }
  __syncthreads();
  // direction tables: incident (phi0 = 0) per Lobatto angle, scattered per (angle, azimuth)
  for (int e = t; e < nummu + na * TM_NAZ; e += TM_THREADS) {
    if (e < nummu) {
      double th0 = acos(A.mu[e] * 1.0) * 180.0 / PI;
      if (th0 > 179.9999) th0 = 180.0;
      tm_dir(th0, 0.0, 0.0, beta, false, Gin[e]);
    } else {
      const int a = (e - nummu) / TM_NAZ, k = (e - nummu) % TM_NAZ;
      const double phi = 360.0 / (double)TM_NAZ * ((double)(k + 1) - 1.0);
      tm_dir(sh.thet[a], phi, 0.0, beta, true, Gsc[(size_t)a * TM_NAZ + k]);
    }
  }
  __syncthreads();
  for (int jj = 0; jj < nummu; jj++) {
    double thet0 = acos(A.mu[jj] * 1.0) * 180.0 / PI;
    if (thet0 > 179.9999) thet0 = 180.0;
    if (upright) {
      // polar parts per order m: P_m(a) for the four amplitudes
      // upright: the scattered polar cosine does not depend on the azimuth
      if (t < na) {
        sh.cth[t] = Gsc[(size_t)t * TM_NAZ].ctp;
        if (t == 0) sh.accs[2] = Gin[jj].ctp;
      }
      __syncthreads();
      const double cth0 = sh.accs[2];
      for (int m = 0; m <= nmax; m++) {
        const int nmin = max(m, 1);
        if (t == na) tm_vigampl(cth0, nmax, m, [&](int k, double a, double b) { sh.dv0[0][k] = m * a; sh.dv0[1][k] = b; });
        if (t < na)
          tm_vigampl(sh.cth[t], nmax, m, [&](int k, double a, double b) {
            DVA[((size_t)t * 2 + 0) * TM_NMAX + k] = m * a;
            DVA[((size_t)t * 2 + 1) * TM_NMAX + k] = b;
          });
        __syncthreads();
        // U[b][v][n] = sum_nn CAL(n, nn) T_b(m, n, nn) v0[nn], v0 = p0 (m d0/sin), q0 (d0')
        const int nmv = nmax - nmin + 1;
        for (int e = t; e < 8 * nmv; e += TM_THREADS) {
          const int bv = e / nmv, n = nmin + e % nmv, b = bv >> 1, v = bv & 1;
          double ur = 0.0, ui = 0.0;
          for (int nn = nmin; nn <= nmax; nn++) {
            const float2 f = T[tm_tidx(nmax, m, b, n, nn)];
            const cplx ct = cmul(tm_cal(n, nn), cmk(f.x, f.y));
            const double w0 = sh.dv0[v][nn - 1];
            ur = ur + ct.re * w0;
            ui = ui + ct.im * w0;
          }
          sh.u[bv][n - 1][0] = ur;
          sh.u[bv][n - 1][1] = ui;
        }
        __syncthreads();
        // P_m(a) = sum_n (p, q)_n . U: VV, VH, HV, HH (the HV sign included)
        for (int e = t; e < 4 * na; e += TM_THREADS) {
          const int a = e >> 2, q = e & 3;
          const double* pa = DVA + (size_t)a * 2 * TM_NMAX;
          const double* qa = pa + TM_NMAX;
          double xr = 0.0, xi = 0.0;
          // (first factor vector, U index) x 4, U index = block * 2 + (0: p0, 1: q0);
          // blocks 0..3 = 11, 12, 21, 22
          int u0, u1, u2, u3;
          bool f0p, f1p, f2p, f3p;
          switch (q) {
            case 0: u0 = 0; f0p = true; u1 = 4; f1p = false; u2 = 3; f2p = true; u3 = 7; f3p = false; break;   // VV
            case 1: u0 = 1; f0p = true; u1 = 5; f1p = false; u2 = 2; f2p = true; u3 = 6; f3p = false; break;   // VH
            case 2: u0 = 0; f0p = false; u1 = 4; f1p = true; u2 = 3; f2p = false; u3 = 7; f3p = true; break;   // HV
            default: u0 = 1; f0p = false; u1 = 5; f1p = true; u2 = 2; f2p = false; u3 = 6; f3p = true; break;  // HH
          }
          if (m == 0) {
            // M = 0: VV = q . U22q0, HH = q . U11q0 (tmatrix_amplq.lp.f:842-846)
            if (q == 0 || q == 3) {
              const int ui = (q == 0) ? 7 : 1;
              for (int n = nmin; n <= nmax; n++) {
                xr = xr + qa[n - 1] * sh.u[ui][n - 1][0];
                xi = xi + qa[n - 1] * sh.u[ui][n - 1][1];
              }
            }
          } else {
            for (int n = nmin; n <= nmax; n++) {
              const double a0 = f0p ? pa[n - 1] : qa[n - 1], a1 = f1p ? pa[n - 1] : qa[n - 1];
              const double a2 = f2p ? pa[n - 1] : qa[n - 1], a3 = f3p ? pa[n - 1] : qa[n - 1];
              xr = xr + a0 * sh.u[u0][n - 1][0] + a1 * sh.u[u1][n - 1][0] + a2 * sh.u[u2][n - 1][0] + a3 * sh.u[u3][n - 1][0];
              xi = xi + a0 * sh.u[u0][n - 1][1] + a1 * sh.u[u1][n - 1][1] + a2 * sh.u[u2][n - 1][1] + a3 * sh.u[u3][n - 1][1];
            }
            if (q == 2) { xr = -xr; xi = -xi; }
          }
          P[((size_t)m * TM_NA + a) * 4 + q] = cmk(xr, xi);
        }
        __syncthreads();
      }
    }
    // amplitudes per (scattered angle, azimuth) and their quadratic forms
    for (int e = t; e < na * TM_NAZ; e += TM_THREADS) {
      const int a = e / TM_NAZ, k = e % TM_NAZ;
      TmGeom g;
      tm_geom_of(Gin[jj], Gsc[(size_t)a * TM_NAZ + k], g);
      cplx vv, vh, hv, hh;
      if (upright) {
        vv = P[((size_t)0 * TM_NA + a) * 4 + 0];
        hh = P[((size_t)0 * TM_NA + a) * 4 + 3];
        vh = hv = cmk(0.0, 0.0);
        // cos(m ph), sin(m ph) by the angle-addition recurrence
        double s1, c1;
        sincos(g.ph, &s1, &c1);
        double cm = 1.0, sm = 0.0;
        for (int m = 1; m <= nmax; m++) {
          const double cn = cm * c1 - sm * s1;
          sm = sm * c1 + cm * s1;
          cm = cn;
          const double fc = 2.0 * cm, fs = 2.0 * sm;
          const cplx* pm = P + ((size_t)m * TM_NA + a) * 4;
          vv = cadd(vv, cscale(pm[0], fc));
          vh = cadd(vh, cscale(pm[1], fs));
          hv = cadd(hv, cscale(pm[2], fs));
          hh = cadd(hh, cscale(pm[3], fc));
        }
        tm_rotate(g, dk, vv, vh, hv, hh);
      } else {
        tm_ampl_full(T, nmax, g, dk, vv, vh, hv, hh);
      }
      const cplx s11 = cscale(vv, wave_num), s12 = cscale(vh, wave_num), s21 = cscale(hv, wave_num),
                 s22 = cscale(hh, wave_num);
      const double a11 = s11.re * s11.re + s11.im * s11.im, a12 = s12.re * s12.re + s12.im * s12.im;
      const double a21 = s21.re * s21.re + s21.im * s21.im, a22 = s22.re * s22.re + s22.im * s22.im;
      double* z = Zb + ((size_t)a * TM_NAZ + k) * 4;
      z[0] = (fact_sca * (a11 + a12 + a21 + a22)) * phi_weights;
      z[1] = (fact_sca * (a11 - a12 + a21 - a22)) * phi_weights;
      z[2] = (fact_sca * (a11 + a12 - a21 - a22)) * phi_weights;
      z[3] = (fact_sca * (a11 - a12 - a21 + a22)) * phi_weights;
      if (k == 0 && sh.thet[a] == 180.0 && jj == nummu - 1) {
        sback[0] = fact_sca * (a11 + a12 + a21 + a22);
        sback[2] = fact_sca * (a11 - a12 + a21 - a22);
        sback[1] = fact_sca * (a11 + a12 - a21 - a22);
        sback[3] = fact_sca * (a11 - a12 - a21 + a22);
      }
      if (k == 0 && sh.thet[a] == thet0) {
        const double sp = s11.im + s22.im, sm = s11.im - s22.im;
        ext[0 + 2 * (0 + 2 * jj)] += 1.0 * (fext * sp);
        ext[0 + 2 * (1 + 2 * jj)] += 1.0 * (fext * sm);
        ext[1 + 2 * (0 + 2 * jj)] += 1.0 * (fext * sm);
        ext[1 + 2 * (1 + 2 * jj)] += 1.0 * (fext * sp);
      }
    }
    __syncthreads();
    // azimuth sums in the reference's order, the scattering matrix of this incident angle
    if (t < na) {
      const int kk = t / nummu, ll = t % nummu;
      double z11 = 0.0, z12 = 0.0, z21 = 0.0, z22 = 0.0;
      for (int k = 0; k < TM_NAZ; k++) {
        const double* z = Zb + ((size_t)t * TM_NAZ + k) * 4;
        z11 = z11 + z[0];
        z12 = z12 + z[1];
        z21 = z21 + z[2];
        z22 = z22 + z[3];
      }
      auto S_ = [&](int i2, int i1) -> double& {
        return scat[i2 + 2 * (ll + nummu * (i1 + 2 * (jj + nummu * kk)))];
      };
      S_(0, 0) = 0.0 + z11 * 1.0;
      S_(0, 1) = 0.0 + z12 * 1.0;
      S_(1, 0) = 0.0 + z21 * 1.0;
      S_(1, 1) = 0.0 + z22 * 1.0;
    }
    __syncthreads();
    // emission vector: extinction minus the scattering integrated over the sphere
    if (t == 0) {
      double e11 = 0.0, e12 = 0.0;
      for (int kk = 0; kk < 2; kk++)
        for (int ll = 0; ll < nummu; ll++) {
          const size_t b0 = 2 * (ll + nummu * (0 + 2 * (jj + nummu * kk)));
          const size_t b1 = 2 * (ll + nummu * (1 + 2 * (jj + nummu * kk)));
          e11 = e11 + scat[b0] * A.wq[ll] * 2.0 * PI;
          e12 = e12 + scat[b1] * A.wq[ll] * 2.0 * PI;
        }
      emis[0 + 2 * jj] = ext[0 + 2 * (0 + 2 * jj)] - e11;
      emis[1 + 2 * jj] = ext[0 + 2 * (1 + 2 * jj)] - e12;
    }
    __syncthreads();
  }
  if (t == 0) A.nmax[p] = nmax;
}

// Persistent CTAs over the particles of a launch, one scratch slot each.
__global__ void __launch_bounds__(TM_THREADS, 2) k_tmatrix(TmArgs A) {
  __shared__ TmShared sh;
  double* s = A.scratch + (size_t)blockIdx.x * TM_SLOT_DOUBLES;
  const int np = A.n_items * A.nbins;
  for (;;) {
    if (threadIdx.x == 0) sh.particle = atomicAdd(A.counter, 1);
    __syncthreads();
    const int p = sh.particle;
    __syncthreads();
    if (p >= np) break;
    tm_particle(A, s, sh, p);
    __syncthreads();
  }
}

// Per-bin set-up of calc_tmatrix (src/tmatrix.f90:124-183): input checks,
// the soft-spheroid index of ice bins (eps_mix with air), the equal-volume
// radius from the maximum dimension and the aspect ratio.  A bin that fails
// a check gets FATAL | ST_RANGE and no particle.
__global__ void k_tmat_prep(int n_items, int nbins, const double* freq, const double* ref_re, const double* ref_im, const int* phase,
                            const double* dmax, const double* del_d, const double* ndens, const double* density,
                            const double* asr, const double* canting, double* mrr, double* mri, double* axi,
                            double* nd_eff, int* status) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n_items * nbins) return;
  const int item = p / nbins;
  const double nd = ndens[p];
  status[p] = 0;
  nd_eff[p] = 0.0;
  mrr[p] = mri[p] = axi[p] = 0.0;
  if (nd == 0.0) return;
  const bool bad = !(nd > 0.0) || !(del_d[p] > 0.0) || !(density[p] > 0.0) || !(asr[p] > 0.0) ||
                   !(dmax[p] > 0.0) || !(canting[p] >= 0.0) || canting[p] > 180.0 ||
                   (phase[item] != 1 && phase[item] != -1) || !(freq[item] > 0.0) || !isfinite(freq[item]) ||
                   !isfinite(ref_re[item]) || !isfinite(ref_im[item]) || !isfinite(dmax[p]) || !isfinite(asr[p]);
  if (bad) {
    status[p] = PAMTRA_B200_FATAL | PAMTRA_B200_ST_RANGE;
    return;
  }
  cplx m = cmk(ref_re[item], ref_im[item]);
  if (phase[item] == -1 && density[p] != 917.0) m = eps_mix_m(m, density[p]);
  mrr[p] = m.re;
  mri[p] = fabs(-m.im);  // mindex = conjg(mMix); the solve takes |Im|
  const double a = asr[p];
  axi[p] = (a <= 1.0) ? 0.5 * dmax[p] * pow(a, 1.0 / 3.0) : 0.5 * dmax[p] / pow(a, 2.0 / 3.0);
  nd_eff[p] = nd;
}

// Species sums of calc_tmatrix (src/tmatrix.f90:413-416) in bin order, and
// the per-bin "NN" backscattering 4 pi ndens Sback(1,1) (:383).
__global__ void k_tmat_sum(int n_items, int nbins, int nummu, const double* ndens, const double* del_d,
                           const double* pscat, const double* pext, const double* pemis, const double* psback,
                           const int* pstatus, double* scat, double* ext, double* emis, double* sback, double* back_spec,
                           int* status) {
  const int item = blockIdx.x;
  const size_t NS = (size_t)2 * nummu * 2 * nummu * 2, NE = 4 * (size_t)nummu, NM = 2 * (size_t)nummu;
  const size_t tot = NS + NE + NM + 4;
  for (size_t e = threadIdx.x; e < tot; e += blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < nbins; b++) {
      const size_t p = (size_t)item * nbins + b;
      const double nd = ndens[p];
      if (nd == 0.0 || pstatus[p]) continue;
      double v;
      if (e < NS) v = pscat[p * NS + e];
      else if (e < NS + NE) v = pext[p * NE + (e - NS)];
      else if (e < NS + NE + NM) v = pemis[p * NM + (e - NS - NE)];
      else v = psback[p * 4 + (e - NS - NE - NM)];
      acc = acc + v * nd * del_d[p];
    }
    if (e < NS) scat[(size_t)item * NS + e] = acc;
    else if (e < NS + NE) ext[(size_t)item * NE + (e - NS)] = acc;
    else if (e < NS + NE + NM) emis[(size_t)item * NM + (e - NS - NE)] = acc;
    else sback[(size_t)item * 4 + (e - NS - NE - NM)] = acc;
  }
  for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
    const size_t p = (size_t)item * nbins + b;
    back_spec[p] = (ndens[p] == 0.0 || pstatus[p]) ? 0.0 : 4.0 * PI * ndens[p] * psback[p * 4];
  }
  if (threadIdx.x == 0) {
    int st = 0;
    for (int b = 0; b < nbins; b++) st |= pstatus[(size_t)item * nbins + b];
    status[item] = st;
  }
}

}  // namespace pb
