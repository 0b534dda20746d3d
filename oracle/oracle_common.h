// Test infrastructure only: CPU FP64 restatement ("oracle") of the reference
// PAMTRA passive forward path.  It is linked by nothing in the product; only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
//
// Parity status: pinned against the reference's golden end-to-end fixture
// (tests/golden/rain_snow_reference.npz from the reference's test-suite,
// tests/test_regression.py:42-43, rtol 1e-5) and the TKC water permittivity
// known answer (tests/test_fortran_functions.py:23-33).
//
// Every function names the reference file:line it restates.  Single-precision
// rounding points of the Fortran (default-REAL literals, CMPLX without KIND)
// are reproduced with (double)(float) casts and commented where they occur.
#pragma once
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

namespace orc {

// Fortran default-REAL literal promoted to double.
static inline double F(float v) { return (double)v; }

constexpr double PI = 3.141592653589793;          // constants.f90 pi
constexpr double C_LIGHT = 299792458.0;            // constants.f90 c
constexpr double R_D = 287.0596736665907;          // constants.f90 r_d
constexpr double R_V = 461.5249933083879;          // constants.f90 r_v
constexpr double RHO_WATER = 1000.0;               // constants.f90 rho_water
constexpr double RHO_ICE = 917.0;                  // constants.f90 rho_ice
constexpr double SKY_TEMP = 2.73;                  // constants.f90 sky_temp
constexpr double DELTA_D_MONO = 1.0e-8;            // constants.f90 delta_d_mono
constexpr int MAXNLEG = 200;                       // settings.f90 maxnleg

// gfortran complex arithmetic (-fcx-fortran-rules): plain products and
// Smith-style ("wide") division without NaN recovery.
struct cplx {
  double re, im;
};
static inline cplx cmk(double r, double i) { return cplx{r, i}; }
static inline cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
static inline cplx csub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
static inline cplx cmul(cplx a, cplx b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
static inline cplx cscale(cplx a, double s) { return {a.re * s, a.im * s}; }
static inline cplx cdiv(cplx a, cplx b) {
  double ar = a.re, ai = a.im, br = b.re, bi = b.im;
  double tr, ti, ratio, div;
  if (std::fabs(br) < std::fabs(bi)) {
    ratio = br / bi;
    div = (br * ratio) + bi;
    tr = (ar * ratio) + ai;
    ti = (ai * ratio) - ar;
  } else {
    ratio = bi / br;
    div = (bi * ratio) + br;
    tr = (ai * ratio) + ar;
    ti = ai - (ar * ratio);
  }
  return {tr / div, ti / div};
}
static inline cplx cconj(cplx a) { return {a.re, -a.im}; }
static inline double cabs_(cplx a) { return std::hypot(a.re, a.im); }
static inline cplx csqrt_(cplx a) {
  std::complex<double> z(a.re, a.im);
  std::complex<double> r = std::sqrt(z);
  return {r.real(), r.imag()};
}
// CMPLX(x,y) without KIND: COMPLEX(4)
static inline cplx cmplx4(double x, double y) { return {(double)(float)x, (double)(float)y}; }

// distribution names (make_dist_param.f90)
enum Dist { D_EXP = 0, D_EXP_FIELD_T = 1, D_MGAMMA = 2, D_MONO = 3, D_EXP_COSMO_SNOW = 4,
            D_EXP_RYAN = 5, D_LOGN = 6, D_DISABLED = 7 };

}  // namespace orc

extern "C" {

// nmlSet keys used on the passive Mie path (settings.f90:454-573 defaults,
// python/pyPamtra/core.py:89-157 Python defaults).
typedef struct {
  double emissivity;
  double hydro_threshold;
  double hydro_softsphere_min_density;
  int32_t lgas_extinction;
  int32_t lhyd_absorption;
  int32_t lhyd_scattering;
  int32_t lhyd_emission;
  int32_t hydro_includehydroinrhoair;
  int32_t hydro_adaptive_grid;
  int32_t conserve_mass_rescale_dsd;
  int32_t hydro_limit_density_area;
  int32_t outpol_vh;
  int32_t nummu;
  int32_t active;             // nmlSet['active'] (simple radar)
  int32_t radar_attenuation;  // 0 disabled, 1 bottom-up, 2 top-down
  double radar_k2;            // nmlSet['radar_k2']
  int32_t liq_mod;            // 0 TKC, 1 Ell, 2 Lie, 3 Ray, 4 Sto (src/eps_water.f90:39-63)
  int32_t gas_mod;            // 0 R98, 1 L93 (src/get_gasabs.f90:78-102)
} orc_settings;

// One descriptor-file row (python/pyPamtra/descriptorFile.py:19-20).
typedef struct {
  int32_t liq_ice;
  int32_t moment_in;
  int32_t nbin;
  int32_t dist;
  double as_ratio, rho_ms, a_ms, b_ms, alpha_as, beta_as;
  double p_1, p_2, p_3, p_4, d_1, d_2;
} orc_species;

// Full size spectra (nmlSet['hydro_fullspec'], src/hydrometeor_extinction.f90:122-151)
// of one column: [L][nhydro][nbin], d_bound [L][nhydro][nbin + 1].
typedef struct {
  int32_t nbin;
  const double *d, *d_bound, *n, *rho, *mass;
  const double *as_ratio, *canting;  // per bin, T-matrix species only (may be NULL)
} orc_fullspec;

// Optional per-(layer,freq) intermediates for parity tests.
typedef struct {
  double* kextatmo;        // [nfreq][L]            Np/m, bottom-up layer order
  double* kexttot;         // [nfreq][L]
  double* salbedo;         // [nfreq][L]
  int32_t* nlegen;         // [nfreq][L]
  double* legen;           // [nfreq][L][3][MAXNLEG] normalised coefficients (rows 1..3)
  int32_t* present;        // [L]
  double* scatter_matrix;  // [nfreq][L][4][n][n] quadrant-major, row=(i2,j2), col=(i1,j1), row-major
  double* ext;             // [nfreq][L]            extinction matrix diagonal
  double* emis;            // [nfreq][L]            emission vector I component
  int32_t* num_doubles;    // [nfreq][L]            bottom-up order
  double* back;            // [nfreq][L]            volumetric backscattering cross section, m^2/m^3
  double* ze;              // [nfreq][L]            simple radar, dBZ (-9999 without hydrometeors)
  double* att_hydro;       // [nfreq][L]            dB
  double* att_atmo;        // [nfreq][L]            dB
  // save_psd bins [L][nhydro][psd_nbin] of the moment-based distributions
  // (left untouched where none is computed; the caller fills -9999)
  int32_t psd_nbin;
  double *psd_d, *psd_deltad, *psd_n, *psd_mass, *psd_area;
  double* psd_bscat;       // [L][nhydro][psd_nbin] m2 per particle, last frequency (also for full spectra)
} orc_debug;

}
