// Shared device helpers for the B200 passive path.
//
// Arithmetic conventions: the library is compiled with --fmad=false so that
// every a*b+c written out in the restated formulas rounds twice, as the
// reference's gfortran x86-64 build does.  Hot loops (matrix products,
// Legendre and Mie series sums) call fma() explicitly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pamtra_b200.h"

namespace pb {

constexpr double PI = 3.141592653589793;           // constants.f90 pi
constexpr double C_LIGHT = 299792458.0;             // constants.f90 c
constexpr double R_D = 287.0596736665907;           // constants.f90 r_d
constexpr double R_V = 461.5249933083879;           // constants.f90 r_v
constexpr double RHO_WATER = 1000.0;
constexpr double RHO_ICE = 917.0;
constexpr double SKY_TEMP = 2.73;
constexpr double DELTA_D_MONO = 1.0e-8;
constexpr int MAXNLEG = PAMTRA_B200_MAXNLEG;
constexpr int MAXBIN = PAMTRA_B200_MAXBIN;

// Fortran default-REAL literal promoted to double.
__host__ __device__ __forceinline__ double F(float v) { return (double)v; }

// gfortran powi chains for constant integer exponents.
__device__ __forceinline__ double p2(double x) { return x * x; }
__device__ __forceinline__ double p3(double x) { double x2 = x * x; return x2 * x; }
__device__ __forceinline__ double p5(double x) { double x2 = x * x; double x3 = x2 * x; return x3 * x2; }

// ------------------------------------------------------------------ complex
struct cplx {
  double re, im;
};
__device__ __forceinline__ cplx cmk(double r, double i) { return cplx{r, i}; }
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ cplx cmul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ cplx cscale(cplx a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ cplx cconj(cplx a) { return {a.re, -a.im}; }
// Smith-style division as gfortran emits it (-fcx-fortran-rules).
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  double tr, ti, ratio, div;
  if (fabs(b.re) < fabs(b.im)) {
    ratio = b.re / b.im;
    div = (b.re * ratio) + b.im;
    tr = (a.re * ratio) + a.im;
    ti = (a.im * ratio) - a.re;
  } else {
    ratio = b.im / b.re;
    div = (b.im * ratio) + b.re;
    tr = (a.im * ratio) + a.re;
    ti = a.im - (a.re * ratio);
  }
  return {tr / div, ti / div};
}
// Principal square root: r = sqrt((|z|+x)/2), s = y/(2r) (x > 0), else the
// mirrored form; avoids cancellation in |z| - x.
__device__ __forceinline__ cplx csqrt_(cplx z) {
  double d = hypot(z.re, z.im);
  double r, s;
  if (z.re > 0) {
    r = sqrt(0.5 * (d + z.re));
    s = 0.5 * (z.im / r);
  } else {
    s = sqrt(0.5 * (d - z.re));
    r = fabs(0.5 * (z.im / s));
  }
  return {r, copysign(s, z.im)};
}
// CMPLX(x, y) without KIND: rounds both parts to REAL(4).
__device__ __forceinline__ cplx cmplx4(double x, double y) { return {(double)(float)x, (double)(float)y}; }

// ------------------------------------------------------------------ warp helpers
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ------------------------------------------------------------------ team linear algebra
// A "team" is one CTA of T = n*RS threads working on n x n FP64 matrices held
// in shared memory, column-major with leading dimension LD = n + 2 (even, so a
// column is 16-byte aligned for vector loads; two-way bank conflicts at most
// on strided column reads).  Thread t owns column t % n and the row block
// [(t/n)*R, (t/n)*R + R), R = n/RS.
template <int n, int RS>
struct TeamCfg {
  static constexpr int T = n * RS;
  static constexpr int LD = n + 2;
  static constexpr int R = n / RS;
  static constexpr int MAT = n * LD;  // doubles per matrix
};

__device__ __forceinline__ void team_sync() { __syncthreads(); }

// C = A * B (C must not alias A or B).  k-ascending accumulation with FMA.
template <int n, int RS>
__device__ __forceinline__ void mm(const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ C) {
  constexpr int LD = TeamCfg<n, RS>::LD, R = TeamCfg<n, RS>::R;
  const int t = threadIdx.x, j = t % n, r0 = (t / n) * R;
  double acc[R];
#pragma unroll
  for (int i = 0; i < R; i++) acc[i] = 0.0;
#pragma unroll 4
  for (int k = 0; k < n; k++) {
    const double b = B[j * LD + k];
    const double2* a2 = reinterpret_cast<const double2*>(A + k * LD + r0);
#pragma unroll
    for (int i = 0; i < R / 2; i++) {
      const double2 a = a2[i];
      acc[2 * i] = fma(a.x, b, acc[2 * i]);
      acc[2 * i + 1] = fma(a.y, b, acc[2 * i + 1]);
    }
  }
#pragma unroll
  for (int i = 0; i < R; i++) C[j * LD + r0 + i] = acc[i];
}

// y = M * x for vectors in shared memory (threads t < n compute row t).
template <int n, int RS>
__device__ __forceinline__ double mv_row(const double* __restrict__ M, const double* __restrict__ x, int row) {
  constexpr int LD = TeamCfg<n, RS>::LD;
  double s = 0.0;
#pragma unroll 8
  for (int k = 0; k < n; k++) s = fma(M[k * LD + row], x[k], s);
  return s;
}

// In-place Gauss-Jordan inverse with partial (row) pivoting of A (n x n).
// scratch: f[n] doubles, piv[n] ints, redv[8] doubles, redi[8] ints.
// Returns nonzero (to every thread) if a pivot was exactly zero.
template <int n, int RS>
__device__ int ginv(double* A, double* f, int* piv, double* redv, int* redi) {
  constexpr int LD = TeamCfg<n, RS>::LD, R = TeamCfg<n, RS>::R, T = TeamCfg<n, RS>::T;
  constexpr int NW = (n + 31) / 32;  // warps that hold one row each for the pivot search
  const int t = threadIdx.x, j = t % n, r0 = (t / n) * R;
  const int lane = t & 31, warp = t >> 5;
  int singular = 0;
  for (int k = 0; k < n; k++) {
    // pivot search: thread t < n examines row t of column k
    if (t < n) {
      double v = (t >= k) ? fabs(A[k * LD + t]) : -1.0;
      int idx = t;
      const unsigned mask = (n >= 32) ? 0xffffffffu : ((1u << n) - 1u);
#pragma unroll
      for (int o = (n >= 32 ? 16 : n / 2); o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(mask, v, o);
        int oi = __shfl_xor_sync(mask, idx, o);
        if (ov > v || (ov == v && oi < idx)) { v = ov; idx = oi; }
      }
      if (lane == 0) { redv[warp] = v; redi[warp] = idx; }
    }
    team_sync();
    int p = redi[0];
    if (NW > 1) {
      double bv = redv[0];
#pragma unroll
      for (int w = 1; w < NW; w++)
        if (redv[w] > bv) { bv = redv[w]; p = redi[w]; }
    }
    // row interchange k <-> p (threads of row block 0 own the whole column)
    if (t < n && p != k) {
      double tmp = A[j * LD + k];
      A[j * LD + k] = A[j * LD + p];
      A[j * LD + p] = tmp;
    }
    if (t == 0) piv[k] = p;
    team_sync();
    if (t < n) f[t] = A[k * LD + t];
    team_sync();
    const double pv = f[k];
    if (pv == 0.0) singular = 1;
    const double rp = 1.0 / pv;
    const double akj = (j == k) ? rp : A[j * LD + k] * rp;
    if (RS > 1) team_sync();
#pragma unroll 4
    for (int ii = 0; ii < R; ii++) {
      const int i = r0 + ii;
      double v;
      if (i == k) v = akj;
      else if (j == k) v = -f[i] * rp;
      else v = A[j * LD + i] - f[i] * akj;
      A[j * LD + i] = v;
    }
    team_sync();
  }
  // undo the row interchanges as column interchanges, applied in reverse
  if (t == 0) {
    for (int q = 0; q < n; q++) redi[8 + q] = q;  // caller provides redi[8 + n]
    for (int k = n - 1; k >= 0; k--) {
      int p = piv[k];
      int tmp = redi[8 + k];
      redi[8 + k] = redi[8 + p];
      redi[8 + p] = tmp;
    }
  }
  team_sync();
  double col[R];
  const int src = redi[8 + j];
#pragma unroll
  for (int ii = 0; ii < R; ii++) col[ii] = A[src * LD + r0 + ii];
  team_sync();
#pragma unroll
  for (int ii = 0; ii < R; ii++) A[j * LD + r0 + ii] = col[ii];
  team_sync();
  (void)T;
  return singular;
}

}  // namespace pb
