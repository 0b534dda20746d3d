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
// A "team" is one CTA working on n x n FP64 matrices (n = 16, 32, 64) held in
// shared memory, column-major with leading dimension LD = n + 4 (LD = 4 mod
// 16 doubles makes the DMMA fragment loads below bank-conflict free).  The
// team has one warp per 16 x 16 output tile: T = 32 (n/16)^2 threads.
template <int n>
struct Team {
  static constexpr int T = 32 * (n / 16) * (n / 16);
  static constexpr int LD = n + 4;
  static constexpr int MAT = n * LD;  // doubles per matrix
  static constexpr int RG = T / n;    // threads per column in element-wise phases
};

__device__ __forceinline__ void team_sync() { __syncthreads(); }

// FP64 tensor-core MMA, D(8x8) += A(8x4) * B(4x8); fragments: a = A[g][q],
// b = B[q][g], d = D[g][2q], D[g][2q+1] with g = lane/4, q = lane%4.
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

enum MMMode { MM_SET = 0, MM_ACC = 1, MM_IMINUS = 2, MM_IPLUS = 3 };

// C = A*B (MM_SET), C = D + A*B (MM_ACC), C = I - A*B (MM_IMINUS) or
// C = I + A*B (MM_IPLUS).
// Each warp computes one 16 x 16 tile with 2 x 2 DMMA fragments per k-step
// of 4.  Without INPLACE, C must not alias A or B; with INPLACE the team
// synchronises between reading the operands and writing C, so C may be A,
// B or D.
template <int n, int MODE, bool INPLACE = false>
__device__ __forceinline__ void mm(const double* A, const double* B, double* C, const double* D = nullptr) {
  constexpr int LD = Team<n>::LD, WT = n / 16;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row0 = (warp / WT) * 16, col0 = (warp % WT) * 16;
  const int g = lane >> 2, q = lane & 3;
  double c[2][2][2];
#pragma unroll
  for (int rt = 0; rt < 2; rt++)
#pragma unroll
    for (int ct = 0; ct < 2; ct++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int row = row0 + rt * 8 + g, col = col0 + ct * 8 + 2 * q + i;
        c[rt][ct][i] = (MODE == MM_ACC) ? D[col * LD + row]
                                        : ((MODE == MM_IMINUS || MODE == MM_IPLUS) ? (row == col ? 1.0 : 0.0) : 0.0);
      }
  const double sgn = (MODE == MM_IMINUS) ? -1.0 : 1.0;
#pragma unroll 4
  for (int kk = 0; kk < n; kk += 4) {
    const double a0 = sgn * A[(kk + q) * LD + row0 + g];
    const double a1 = sgn * A[(kk + q) * LD + row0 + 8 + g];
    const double b0 = B[(col0 + g) * LD + kk + q];
    const double b1 = B[(col0 + 8 + g) * LD + kk + q];
    dmma(c[0][0], a0, b0);
    dmma(c[0][1], a0, b1);
    dmma(c[1][0], a1, b0);
    dmma(c[1][1], a1, b1);
  }
  if (INPLACE) team_sync();
#pragma unroll
  for (int rt = 0; rt < 2; rt++)
#pragma unroll
    for (int ct = 0; ct < 2; ct++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int row = row0 + rt * 8 + g, col = col0 + ct * 8 + 2 * q + i;
        C[col * LD + row] = c[rt][ct][i];
      }
}

// Two products with the same left factor in one pass over K:
// C1 = A B1 (+ D1) and C2 = A B2 (+ D2), modes MM_SET / MM_ACC each.  The A
// fragments are loaded once for both (six operand loads per k-step for eight
// DMMAs instead of eight), and each element accumulates in the same order as
// in mm(), so the results are bit-identical to two mm() calls.  C1 and C2
// must not alias A, B1 or B2.
template <int n, int MODE1, int MODE2>
__device__ __forceinline__ void mm2(const double* A, const double* B1, double* C1, const double* D1,
                                    const double* B2, double* C2, const double* D2) {
  constexpr int LD = Team<n>::LD, WT = n / 16;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int row0 = (warp / WT) * 16, col0 = (warp % WT) * 16;
  const int g = lane >> 2, q = lane & 3;
  double c[2][2][2], e[2][2][2];
#pragma unroll
  for (int rt = 0; rt < 2; rt++)
#pragma unroll
    for (int ct = 0; ct < 2; ct++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int row = row0 + rt * 8 + g, col = col0 + ct * 8 + 2 * q + i;
        c[rt][ct][i] = (MODE1 == MM_ACC) ? D1[col * LD + row] : 0.0;
        e[rt][ct][i] = (MODE2 == MM_ACC) ? D2[col * LD + row] : 0.0;
      }
#pragma unroll 4
  for (int kk = 0; kk < n; kk += 4) {
    const double a0 = A[(kk + q) * LD + row0 + g];
    const double a1 = A[(kk + q) * LD + row0 + 8 + g];
    const double b0 = B1[(col0 + g) * LD + kk + q];
    const double b1 = B1[(col0 + 8 + g) * LD + kk + q];
    const double f0 = B2[(col0 + g) * LD + kk + q];
    const double f1 = B2[(col0 + 8 + g) * LD + kk + q];
    dmma(c[0][0], a0, b0);
    dmma(e[0][0], a0, f0);
    dmma(c[0][1], a0, b1);
    dmma(e[0][1], a0, f1);
    dmma(c[1][0], a1, b0);
    dmma(e[1][0], a1, f0);
    dmma(c[1][1], a1, b1);
    dmma(e[1][1], a1, f1);
  }
#pragma unroll
  for (int rt = 0; rt < 2; rt++)
#pragma unroll
    for (int ct = 0; ct < 2; ct++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int row = row0 + rt * 8 + g, col = col0 + ct * 8 + 2 * q + i;
        C1[col * LD + row] = c[rt][ct][i];
        C2[col * LD + row] = e[rt][ct][i];
      }
}

// row `row` of M * x (k-ascending FMA chain)
template <int n>
__device__ __forceinline__ double mv_row(const double* __restrict__ M, const double* __restrict__ x, int row) {
  constexpr int LD = Team<n>::LD;
  double s = 0.0;
#pragma unroll 8
  for (int k = 0; k < n; k++) s = fma(M[k * LD + row], x[k], s);
  return s;
}

// Scratch of the inverse routines.
template <int n>
struct InvScratch {
  double f[n], fpre[n], prow[n];
  double cand_v[4];
  int cand_i[4];
  int piv[n], perm[n];
  double nrm;
  int sing;
};

// Pivot candidate of rows i >= k among the n/32 (or one) warps of a column
// group: the lanes hold rows i (value v of column k).
template <int n>
__device__ __forceinline__ void pivot_candidates(int i, int k, double v, InvScratch<n>& S) {
  constexpr int W = (n >= 32) ? 32 : n;
  S.fpre[i] = v;
  double best = (i >= k) ? fabs(v) : -1.0;
  int bi = i;
  const unsigned mask = (n >= 32) ? 0xffffffffu : (((1u << n) - 1u) << (threadIdx.x & 31 & ~(n - 1)));
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(mask, best, o);
    const int oi = __shfl_xor_sync(mask, bi, o);
    if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
  }
  if ((i & (W - 1)) == 0) {
    S.cand_v[i / W] = best;
    S.cand_i[i / W] = bi;
  }
}

// In-place Gauss-Jordan inverse with partial (row) pivoting of A (n x n).
// Thread t owns row t % n of the columns cg, cg + CG, ... (cg = t / n,
// CG = T / n), so every shared-memory sweep is bank-conflict free; the
// pivot search of the next column is fused into the elimination, leaving
// two team barriers per step.  Returns nonzero to every thread if a pivot
// was exactly zero.
template <int n, int T = Team<n>::T>
__device__ int ginv(double* A, InvScratch<n>& S) {
  constexpr int LD = Team<n>::LD, CG = T / n, NC = n / CG, NGW = (n + 31) / 32;
  const int t = threadIdx.x, i = t % n, cg = t / n;
  if (cg == 0) pivot_candidates<n>(i, 0, A[i], S);
  if (t == 0) S.sing = 0;
  team_sync();
  for (int k = 0; k < n; k++) {
    // (b) resolve the pivot, interchange rows k and p, scaled pivot row
    int p = S.cand_i[0];
    {
      double bv = S.cand_v[0];
#pragma unroll
      for (int w = 1; w < NGW; w++)
        if (S.cand_v[w] > bv) { bv = S.cand_v[w]; p = S.cand_i[w]; }
    }
    const double pv = S.fpre[p];
    const double rp = 1.0 / pv;
    if (t < n) {
      const int j = t;
      const double akj = A[j * LD + p];
      if (p != k) {
        A[j * LD + p] = A[j * LD + k];
        A[j * LD + k] = akj;
      }
      S.prow[j] = (j == k) ? rp : akj * rp;
      S.f[t] = (t == k) ? pv : ((t == p) ? S.fpre[k] : S.fpre[t]);
      if (t == 0) {
        S.piv[k] = p;
        if (pv == 0.0) S.sing = 1;
      }
    }
    team_sync();
    // (c) eliminate column k from every other row; the group that owns
    // column k+1 also finds the next pivot
    const double fi = S.f[i];
    double vnext = 0.0;
#pragma unroll
    for (int jj = 0; jj < NC; jj++) {
      const int j = cg + CG * jj;
      const double pj = S.prow[j];
      double v;
      if (i == k) v = pj;
      else if (j == k) v = -fi * rp;
      else v = fma(-fi, pj, A[j * LD + i]);
      A[j * LD + i] = v;
      if (j == k + 1) vnext = v;
    }
    if (k + 1 < n && cg == (k + 1) % CG) pivot_candidates<n>(i, k + 1, vnext, S);
    team_sync();
  }
  // undo the row interchanges as column interchanges in reverse order
  if (t == 0) {
    for (int q = 0; q < n; q++) S.perm[q] = q;
    for (int k = n - 1; k >= 0; k--) {
      const int p = S.piv[k];
      const int tmp = S.perm[k];
      S.perm[k] = S.perm[p];
      S.perm[p] = tmp;
    }
  }
  team_sync();
  double col[NC];
#pragma unroll
  for (int jj = 0; jj < NC; jj++) col[jj] = A[S.perm[cg + CG * jj] * LD + i];
  team_sync();
#pragma unroll
  for (int jj = 0; jj < NC; jj++) A[(cg + CG * jj) * LD + i] = col[jj];
  team_sync();
  return S.sing;
}

// G = (I - X)^-1 in FP64.  X (in buffer P) is overwritten.  When the row-sum
// norm of X is below 0.74 the inverse is a truncated Neumann series whose
// remainder is below 2^-54 relative (the FP64 rounding unit), evaluated with
// the fewer products of two forms:
//   Horner    G = I + X (I + X (... (I + X)))   k products, remainder ||X||^(k+2)
//   squaring  G = (I + X)(I + X^2)(I + X^4)...  2 (m-1) products, remainder ||X||^(2^m)
// (Horner wins for the thin layers of the first doublings, where ||X|| is
// tiny and G = I + X needs no product at all); otherwise Gauss-Jordan with
// partial pivoting.  Returns the buffer holding the inverse (P or G); *sing
// set on a zero pivot; *nprod (if given) grows by the n x n products the
// inverse took (Gauss-Jordan counted as one: n^3 multiply-adds).
template <int n>
__device__ double* inv_iminus(double* P, double* G, InvScratch<n>& S, int* sing, int* nprod = nullptr) {
  constexpr int LD = Team<n>::LD, T = Team<n>::T;
  const int t = threadIdx.x;
  // infinity norm of X
  if (t < n) {
    double r = 0.0;
#pragma unroll 8
    for (int j = 0; j < n; j++) r += fabs(P[j * LD + t]);
    const unsigned mask = (n >= 32) ? 0xffffffffu : ((1u << n) - 1u);
#pragma unroll
    for (int o = ((n >= 32) ? 16 : n / 2); o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(mask, r, o));
    if ((t & 31) == 0) S.cand_v[t >> 5] = r;
  }
  team_sync();
  double nrm = S.cand_v[0];
#pragma unroll
  for (int w = 1; w < (n + 31) / 32; w++) nrm = fmax(nrm, S.cand_v[w]);
  int m = 1;
  double pw = nrm;
  while (pw > 5.0e-17 && m < 8) {
    pw = pw * pw;
    m++;
  }
  int kh = 0;  // Horner products
  double ph = nrm * nrm;
  while (ph > 5.0e-17 && kh < 2 * (m - 1)) {
    ph = ph * nrm;
    kh++;
  }
  if (m < 8 && ph <= 5.0e-17 && kh < 2 * (m - 1)) {
    for (int e = t; e < n * n; e += T) {
      const int col = e / n, row = e % n;
      G[col * LD + row] = ((row == col) ? 1.0 : 0.0) + P[col * LD + row];
    }
    team_sync();
    for (int k = 0; k < kh; k++) {
      mm<n, MM_IPLUS, true>(P, G, G);  // G = I + X G
      team_sync();
    }
    if (nprod) *nprod += kh;
    return G;
  }
  if (m >= 8) {
    // Gauss-Jordan on I - X
    for (int e = t; e < n * n; e += T) {
      const int col = e / n, row = e % n;
      P[col * LD + row] = ((row == col) ? 1.0 : 0.0) - P[col * LD + row];
    }
    team_sync();
    if (ginv<n>(P, S)) *sing = 1;
    if (nprod) *nprod += 1;
    return P;
  }
  // G = I + X
  for (int e = t; e < n * n; e += T) {
    const int col = e / n, row = e % n;
    G[col * LD + row] = ((row == col) ? 1.0 : 0.0) + P[col * LD + row];
  }
  team_sync();
  for (int k = 1; k < m; k++) {
    mm<n, MM_SET, true>(P, P, P);     // P = P^2
    team_sync();
    mm<n, MM_ACC, true>(G, P, G, G);  // G = G + G P
    team_sync();
  }
  if (nprod) *nprod += 2 * (m - 1);
  return G;
}

}  // namespace pb
