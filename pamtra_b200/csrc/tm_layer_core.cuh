// The start of a scattering layer that holds T-matrix species, element by
// element, in the storage of the layer set-up (rt.cuh layer_setup: P1 and
// P2 column-major with leading dimension LD, element (row i2 + 2 j2,
// column i1 + 2 j1) at column * LD + row).  With T-matrix species the
// reference adds their scattering matrix, angle-dependent extinction matrix
// and two-component emission vector to scatcnv's
// (src/hydrometeor_extinction.f90:329-342), and the layer start reads them in
// full: CHECK_NORM4 (src/radscat4.f90:87-136), the number of doublings from
// extinct_matrix(1) + gas (src/radtran4.f90:319-329), INITIALIZE4
// (src/radintg4.f90:1-45) and INITIAL_SOURCE4 (:51-73).  Without T-matrix
// arrays (null pointers) every function reduces to the set-up's Mie-only
// arithmetic.
//
// Host and device code: the CPU tests check it against the oracle's layer
// start; layer_setup takes it up with the GPU forward run of T-matrix
// species.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define TML_FN __host__ __device__ __forceinline__
#else
#define TML_FN inline
#endif

namespace pb {

// T-matrix quadrants are stored row-major: tmq[q][row * n + col], q = 0 for
// L = 1 (and 4), q = 1 for L = 2 (and 3).  Element e = row * n + col.
TML_FN void tml_add_scatter(int e, int n, int LD, const double* tmq, double* Tb, double* Rb) {
  const int row = e / n, col = e % n;
  const size_t o = (size_t)col * LD + row;
  Tb[o] = tmq[e] + Tb[o];                       // P1: T-matrix species + scatcnv
  Rb[o] = tmq[(size_t)n * n + e] + Rb[o];       // P2
}

// CHECK_NORM4 of quadrature row t < N on P1 / P2 (before INITIALIZE4):
// |emis(1, t) - ext(1, 1, t) + 2 pi sum_j2 w(j2) (P1 + P2)(1, j2; 1, t)|.
TML_FN double tml_norm(int t, int N, int LD, const double* wq, double ext, double emis, const double* tm_ext,
                       const double* tm_emis, const double* Tb, const double* Rb) {
  double sum = tm_ext ? (tm_emis[0 + 2 * t] + emis) - (tm_ext[0 + 2 * (0 + 2 * t)] + ext) : emis - ext;
  for (int j2 = 0; j2 < N; j2++)
    sum = sum + 2.0 * 3.1415926535897932384 * wq[j2] * (Tb[(2 * t) * LD + 2 * j2] + Rb[(2 * t) * LD + 2 * j2]);
  return fabs(sum);
}

// Number of doublings and the thin-layer thickness from extinct_matrix(1,1,1) + gas.
TML_FN int tml_doublings(double ext, const double* tm_ext, double gas, double zdiff, double* delta_z) {
  const double extinct = (tm_ext ? tm_ext[0] + ext : ext) + gas;
  const double fl = log(fmax(extinct * zdiff, 1.0e-7) / 1.0e-6) / 0.693147182464599609375;  // log(2.) in REAL(4)
  int nd = 0;
  if (fl > 0.0) nd = (int)fl + 1;
  *delta_z = zdiff / ldexp(1.0, nd);
  return nd;
}

// INITIALIZE4 element e = col * n + row, in place: P2 -> R, P1 -> T.
TML_FN void tml_init4(int e, int n, int LD, const double* mu, const double* wq, double delta_z, double gas, double ext,
                      const double* tm_ext, double* Rb, double* Tb) {
  const double C = 2.0 * 3.1415926535897932384;
  const int col = e / n, row = e % n;
  const int i1 = col & 1, j1 = col >> 1, i2 = row & 1, j2 = row >> 1;
  const double wj1 = wq[j1];
  const double tmp = delta_z / mu[j2];
  const double gext = (i1 == i2) ? gas : 0.0;
  const double diag = (row == col) ? 1.0 : 0.0;
  // EXTINCT_MATRIX(I2, I1, J2, L)
  const double em = tm_ext ? tm_ext[i2 + 2 * (i1 + 2 * j2)] + ((i1 == i2) ? ext : 0.0) : ((i1 == i2) ? ext : 0.0);
  double ex = 0.0;
  if (j1 == j2) ex = em + gext;
  const size_t o = (size_t)col * LD + row;
  Rb[o] = C * tmp * wj1 * Rb[o];
  Tb[o] = diag - tmp * (ex - C * wj1 * Tb[o]);
}

// INITIAL_SOURCE4 entry t < 2 N (Stokes i = t & 1, angle t >> 1), the same for both halves.
TML_FN double tml_source(int t, const double* mu, double planck0, double delta_z, double gas, double emis,
                         const double* tm_emis) {
  const int i = t & 1, jj = t >> 1;
  const double tmp = planck0 * delta_z / mu[jj];
  const double ev = tm_emis ? tm_emis[i + 2 * jj] + ((i == 0) ? emis : 0.0) : ((i == 0) ? emis : 0.0);
  const double e = (i == 0) ? gas : 0.0;
  return tmp * (ev + e);
}

}  // namespace pb
