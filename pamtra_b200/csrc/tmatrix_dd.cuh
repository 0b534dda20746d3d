// Double-double solve of the T-matrix for bins outside the FP64 envelope
// (large, strongly aspherical liquid drops), following the reference's
// REAL*16 tmatrix_amplq (src/tmatrix_amplq.lp.f): nodes, surface, Bessel
// tables, surface integrals and the inverse of Q in double-double
// (ddreal.cuh), then T = -RgQ Q^-1 accumulated in double over k = 1..2 nm as
// the reference's TT (:2107-2153) does.  The steps are in
// tmatrix_dd_core.cuh, shared with a serial host driver that the CPU tests
// run against the REAL*16 oracle; here are the CTA drivers (one bin per CTA,
// 256 threads, one node, pair or element per thread, warp 0 choosing the
// pivot), with the same organisation as the FP64 solve of tmatrix.cuh.  The
// double-double scratch (TDO_END doubles) follows the CTA's FP64 slot, which
// keeps the single-precision T and the angular work.
//
// Not yet included in the library: it joins k_tmatrix (per bin, chosen by
// size parameter, index and aspect ratio) together with its GPU parity run
// against the REAL*16 oracle.
#pragma once
#include "common.cuh"
#include "tmatrix.cuh"
#include "tmatrix_dd_core.cuh"

namespace pb {

// CONST + RSP1 + VARY + BESS (tmatrix_amplq.lp.f:972-1524) in double-double.
// Whole CTA; false when the reference would stop.
__device__ bool tdd_setup(double* sd, TmShared& sh, int nmax, int ngauss, double lam, double mrr, double mri,
                          double rev, double eps) {
  const int t = threadIdx.x, ng = 2 * ngauss;
  if (t < (ng + 1) / 2) tdd_gauss_pair(sd, ng, t);
  __syncthreads();
  if (t < ngauss) tdd_surface_node(sd, t, ngauss, rev, eps);
  __syncthreads();
  double ta = (t < ng) ? tdd_size_node(sd, t, lam, mrr, mri) : 0.0;
  for (int o = 16; o > 0; o >>= 1) ta = fmax(ta, __shfl_xor_sync(0xffffffffu, ta, o));
  if ((t & 31) == 0) sh.accs[t >> 5] = ta;
  __syncthreads();
  ta = 0.0;
  for (int w = 0; w < TM_THREADS / 32; w++) ta = fmax(ta, sh.accs[w]);
  int nnmax1 = 0, nnmax2 = 0;
  const bool ok = tdd_lengths(ta, nmax, mrr, mri, &nnmax1, &nnmax2);
  __syncthreads();
  if (!ok) return false;
  if (t < ng) tdd_bessel_node(sd, t, nmax, nnmax1, nnmax2, mrr, mri);
  __syncthreads();
  return true;
}

// TMATR0 / TMATR + TT (tmatrix_amplq.lp.f:1526-2153) in double-double for
// order m; T goes where tm_tget of the FP64 slot s reads it.  Whole CTA;
// returns 2 nm, or 0 when a pivot vanishes.
__device__ int tdd_solve(double* s, double* sd, TmShared& sh, int m, int nmax, int ngauss, double lam, double mrr,
                         double mri) {
  const int t = threadIdx.x;
  const int mm1 = (m == 0) ? 1 : m, nm = nmax - mm1 + 1, n2m = 2 * nm, ldw = 2 * n2m;
  if (t < ngauss) tdd_vig_node(sd, t, ngauss, nmax, m);
  __syncthreads();
  for (int pr = t; pr < nm * nm; pr += TM_THREADS) tdd_pair(sd, pr, m, nmax, ngauss, lam, mrr, mri);
  for (int e = t; e < n2m * n2m; e += TM_THREADS) tdd_identity(sd, e, n2m);
  __syncthreads();
  for (int c = 0; c < n2m; c++) {
    if (t < 32) {
      double best = -1.0;
      int br = c;
      for (int r = c + t; r < n2m; r += 32) {
        const double a = tdd_pivot_key(sd, r, c, n2m);
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
    const ddc ip = tdd_pivot_inverse(sd, pr, c, n2m);
    __syncthreads();
    for (int j = c + t; j < ldw; j += TM_THREADS) tdd_swap_scale(sd, c, pr, j, n2m, ip);
    __syncthreads();
    const int wcols = ldw - c - 1;
    for (int e = t; e < n2m * wcols; e += TM_THREADS) tdd_elim(sd, c, e, n2m);
    __syncthreads();
  }
  double* tout = reinterpret_cast<double*>(tm_aug(s));
  for (int e = t; e < n2m * n2m; e += TM_THREADS) tdd_product(sd, tout, e, n2m);
  __syncthreads();
  return n2m;
}

}  // namespace pb
