// Single scattering of Mie spheres, integrated over the size distribution,
// summed over species into normalised Legendre coefficients per
// (column, layer, frequency).
#pragma once
#include "common.cuh"
#include "work.cuh"
#include "ray_table.cuh"

namespace pb {

#ifndef MIE_MAXNREG
#define MIE_MAXNREG 128  // registers per k_mie thread: four 4-warp CTAs per SM
#endif
constexpr int MIE_WARPS = 4;      // default warps per CTA
constexpr int MIE_MAX_WARPS = 8;  // largest launch shape (pamtra_b200_set_launch)
constexpr int NQ_MAX = 256;   // Gauss points per series (nquad)
constexpr int NT_MAX = 128;   // Mie terms per bin

// Shared memory of one warp of k_mie: the phase-function sums of the
// current species per quadrature point (P11, P12, P33) and the weights and
// term counts of the bins of the current pass.
struct MieSmem {
  double sump[3][NQ_MAX];
  double bw[32], bd[32];
  int bn[32];
};
// Coefficient slab of one warp in global scratch: up to 32 bins x kmax rows
// of (a_n, b_n); 4096 doubles hold 32 bins up to 32 terms (size parameters
// up to about 20), fewer bins per pass beyond that (8 at the 127-term limit).
constexpr int MIE_SLAB = 4096;
// each warp's slab region: the coefficients, then the item's species sums of
// the Legendre coefficients [3][MAXNLEG] (FP64 whatever the storage of the result)
constexpr int MIE_SLAB_STRIDE = MIE_SLAB + 3 * MAXNLEG;
constexpr int MIE_SLAB_WARPS_PER_SM = 16;  // slabs reserved per SM (caps the k_mie grid; the resident maximum)

// Per-term constants: c_n = (2n+1) / (n(n+1)) of mieangle evaluated in REAL(4)
// as the reference does (mie_scat_utilities.f90:139), and 1/n, which replaces
// the divisions by n in the pi_n and Legendre recurrences (the reference
// divides; the products differ from the quotients in the last bit only).
// c_mie_inv covers the Legendre orders too (l <= MAXNLEG - 1 > NT_MAX).
__constant__ double c_mie_c[NT_MAX + 1], c_mie_inv[MAXNLEG];

// src/eps_water.f90:653-757 eps_water_tkc (T in degC, f in GHz)
__device__ cplx eps_water_tkc(double T, double f) {
  const double a_1 = 8.169396e+01, b_1 = 4.410555e-03, c_1 = 1.208992e-13, d_1 = 6.768869e+02;
  const double a_2 = 1.597733e+00, b_2 = 1.060228e-02, c_2 = 9.982113e-15, d_2 = 5.720517e+02;
  const double t_c = 1.351758e+02;
  const double frq = f * 1e9;
  double eps_s = 87.9144 - 0.404399 * T + 9.58726e-4 * (T * T) - 1.32802e-6 * pow(T, 3.0);
  double delta_1 = a_1 * exp(-b_1 * T), tau_1 = c_1 * exp(d_1 / (T + t_c));
  double delta_2 = a_2 * exp(-b_2 * T), tau_2 = c_2 * exp(d_2 / (T + t_c));
  double wv = 2.0 * PI * frq;
  double x1 = wv * tau_1, x2 = wv * tau_2;
  double t1 = ((tau_1 * tau_1) * delta_1) / (1.0 + x1 * x1);
  double t2 = ((tau_2 * tau_2) * delta_2) / (1.0 + x2 * x2);
  double eps1 = eps_s - (wv * wv) * (t1 + t2);
  t1 = (tau_1 * delta_1) / (1.0 + x1 * x1);
  t2 = (tau_2 * delta_2) / (1.0 + x2 * x2);
  double eps2 = wv * (t1 + t2);
  return cmplx4(eps1, eps2);  // CMPLX without KIND (eps_water.f90:749)
}

// The other liquid water models of src/eps_water.f90 (nmlSet['liq_mod']),
// salinity 0 as src/scatProperties.f90:228 passes it; T in degC, f in GHz.
// Literals without a kind in the reference are REAL(4) values promoted to
// REAL(8) (written as float literals here), its pi parameter is the REAL(4)
// value of 3.141592653589793, and CMPLX without KIND rounds both parts to
// REAL(4).
constexpr double PI_R4 = (double)3.141592653589793f;

// eps_water_ellison (src/eps_water.f90:85-158, after Maetzler 2006, 5.2.5.4)
__device__ __noinline__ cplx eps_water_ellison(double s, double T, double f) {
  const double a1 = 0.46606917e-02f, a2 = -0.26087876e-04f, a3 = -0.63926782e-05f, a4 = 0.63000075e+01f,
               a5 = 0.26242021e-02f, a6 = -0.42984155e-02f, a7 = 0.34414691e-04f, a8 = 0.17667420e-03f,
               a9 = -0.20491560e-06f, a10 = 0.58366888e+03f, a11 = 0.12634992e+03f, a12 = 0.69227972e-04f,
               a13 = 0.38957681e-06f, a14 = 0.30742330e+03f, a15 = 0.12634992e+03f, a16 = 0.37245044e+01f,
               a17 = 0.92609781e-02f, a18 = -0.26093754e-01f;
  const double T2 = T * T, T4 = T2 * T2;
  const double p = s * (37.5109f + 5.45216f * s + 0.014409f * (s * s)) / (1004.75f + 182.283f * s + s * s);
  const double alpha_0 = (6.9431f + 3.2841f * s - 0.099486f * (s * s)) / (84.85f + 69.024f * s + s * s);
  const double alpha_1 = 49.843f - 0.2276f * s + 0.00198f * (s * s);
  const double sig_s35 = 2.903602f + 8.607e-02f * T + 4.738817e-04f * T2 - 2.991e-06f * (T2 * T) + 4.3041e-09f * T4;
  const double eps_s = 87.85306f * exp(-0.00456992f * T - a1 * s - a2 * (s * s) - a3 * s * T);
  const double eps_1 = a4 * exp(-a5 * T - a6 * s - a7 * s * T);
  const double tau_1 = (a8 + a9 * s) * exp(a10 / (T + a11));
  const double tau_2 = (a12 + a13 * s) * exp(a14 / (T + a15));
  const double eps_inf = a16 + a17 * T + a18 * s;
  const double q = 1 + (alpha_0 * (T - 15)) / (T + alpha_1);
  const double sig = sig_s35 * p * q;
  const cplx d1 = cmk(1.0, -(2.0 * PI_R4 * f * tau_1)), d2 = cmk(1.0, -(2.0 * PI_R4 * f * tau_2));
  cplx e = cadd(cdiv(cmk(eps_s - eps_1, 0.0), d1), cdiv(cmk(eps_1 - eps_inf, 0.0), d2));
  e = cadd(e, cmk(eps_inf, 0.0));
  return cadd(e, cmk(0.0, (double)17.9751f * sig / f));
}

// eps_water_liebe (src/eps_water.f90:160-207, Liebe, Hufford and Manabe 1991)
__device__ __noinline__ cplx eps_water_liebe(double T, double f) {
  const double T_K = T + 273.15f;
  const double theta_1 = 1. - 300. / T_K;
  const double fp = 20.1f * exp(7.88f * theta_1);
  const double fs = 39.8f * fp;
  const double eps_0 = 77.66f - 103.3f * theta_1;
  const double eps_1 = 0.0671f * eps_0;
  const double eps_2 = 3.52f;
  cplx e = cadd(cdiv(cmk(eps_0 - eps_1, 0.0), cmplx4(1.0, -f / fp)), cdiv(cmk(eps_1 - eps_2, 0.0), cmplx4(1.0, -f / fs)));
  return cadd(e, cmk(eps_2, 0.0));
}

// eps_water_ray (src/eps_water.f90:215-592): below 1 mm wavelength (f above
// 299.79 GHz) linear interpolation in the tabulated optical constants of
// 0.2-1000 um (:515-537; the interval is the one ending at the first table
// wavelength >= wl, found here by bisection over the ascending table instead
// of the reference's linear scan), 1 mm - 10 cm the Ray (1972) formula;
// *bad is set outside 0.2 um - 10 cm, where the reference stops.
__device__ __noinline__ cplx eps_water_ray(double T, double f, int* bad) {
  const double wl = (double)(1.e6f * 2.99792458e8f) / (f * 1.e9f);  // microns
  if (wl < (double)0.2f || wl > 100000.0 || !(wl == wl)) {
    *bad = 1;
    return cmk(1.0, 0.0);
  }
  if (!(wl > 1000.0)) {
    // smallest i in [1, RAY_NUMWAT) with wl <= ray_wl[i]; ray_wl[last] = 1000
    int lo = 1, hi = RAY_NUMWAT - 1;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (wl > (double)ray_wl[mid]) lo = mid + 1;
      else hi = mid;
    }
    const int i1 = lo - 1, i2 = lo;
    const double w1 = ray_wl[i1], w2 = ray_wl[i2];
    const double fac = (wl - w1) / (w2 - w1);
    const double rn = (double)ray_rn[i1] + fac * ((double)ray_rn[i2] - (double)ray_rn[i1]);
    const double cn = (double)ray_cn[i1] + fac * ((double)ray_cn[i2] - (double)ray_cn[i1]);
    return cmul(cmk(rn, cn), cmk(rn, cn));
  }
  const double T1 = T + 273.0f, T2 = T - 25.0f, xl = wl / 10000.0f;
  const double sigma = 12.5664e8f;
  const double alpha = -16.8129f / T1 + 0.0609265f;
  const double eps_s = 78.54f * (1.0f - 4.579e-3f * T2 + 1.19e-5f * (T2 * T2) - 2.8e-8f * (T2 * T2 * T2));
  const double eps_inf = 5.27137f + 0.0216474f * T - 0.00131198f * (T * T);
  const double xlams = 0.00033836f * exp(2513.98f / T1);
  const double powtrm = pow(xlams / xl, 1.f - alpha);
  const double sn = sin(PI_R4 * alpha / 2), cs = cos(PI_R4 * alpha / 2);
  const double denom = 1.f + 2 * powtrm * sn + pow(xlams / xl, 2.f * (1.f - alpha));
  const double eps_r = eps_inf + (eps_s - eps_inf) * (1.0f + powtrm * sn) / denom;
  const double eps_i = (sigma * xl / (double)18.8496e10f) + (eps_s - eps_inf) * powtrm * cs / denom;
  const cplx n = csqrt_(cmk(eps_r, eps_i));
  double rn = n.re, cn = n.im;
  if (!(wl > 3000.0f)) {
    // remaining absorption bands (Ray eq. 8, table 2)
    cn = cn + 0.39f * exp(-pow(fabs(log10(wl / 17.0f) / 0.45f), (double)1.3f)) +
         0.41f * exp(-pow(fabs(log10(wl / 62.0f) / 0.35f), (double)1.7f)) +
         0.25f * exp(-pow(fabs(log10(wl / 300.0f) / 0.47f), 3.0));
  }
  return cmul(cmk(rn, cn), cmk(rn, cn));
}

// eps_water_stogryn (src/eps_water.f90:598-651, after Maetzler 2006, 5.2.4.2)
__device__ __noinline__ cplx eps_water_stogryn(double s, double T, double f) {
  const double T2 = T * T, T4 = T2 * T2;
  const double p = s * (37.5109f + 5.45216f * s + 0.014409f * (s * s)) / (1004.75f + 182.283f * s + s * s);
  const double alpha_0 = (6.9431f + 3.2841f * s - 0.099486f * (s * s)) / (84.85f + 69.024f * s + s * s);
  const double alpha_1 = 49.843f - 0.2276f * s + 0.00198f * (s * s);
  const double sig_s35 = 2.903602f + 8.607e-02f * T + 4.738817e-04f * T2 - 2.991e-06f * (T2 * T) + 4.3041e-09f * T4;
  const double a = 1.f - (s * (0.03838f + 0.00218f * s) * (79.88f + T)) / ((12.01f + s) * (52.53f + T));
  const double b = 1.f - s * ((0.03409f + 0.002817f * s) / (7.69f + s)) -
                   s * T * ((0.00246f + 0.00141f * T) / (188.f - 7.57f * T + T2));
  const double eps_s = ((37088.6f - 82.168f * T) / (421.854f + T)) * a;
  const double eps_1 = (0.0787f * ((37088.6f - 82.168f * T) / (421.854f + T))) * a;
  const double tpt1 = ((255.04f + 0.7246f * T) / ((49.25f + T) * (45.f + T))) * b;
  const double tpt2 = 0.00628f;
  const double eps_inf = 4.05f + 0.0186f * T;
  const double q = 1 + (alpha_0 * (T - 15)) / (T + alpha_1);
  const double sig = sig_s35 * p * q;
  cplx e = cadd(cdiv(cmk(eps_s - eps_1, 0.0), cmk(1.0, -(f * tpt1))), cdiv(cmk(eps_1 - eps_inf, 0.0), cmk(1.0, -(f * tpt2))));
  e = cadd(e, cmk(eps_inf, 0.0));
  return cadd(e, cmk(0.0, (double)17.9751f * sig / f));
}

// src/ref_water.f90 with src/eps_water.f90:39-63 (get_eps_water): m = sqrt(eps),
// (refre, refim) with refim > 0; *bad set where the model has no value.
__device__ cplx ref_water(double T_c, double f, int liq_mod, int* bad) {
  cplx e;
  switch (liq_mod) {
    case PAMTRA_B200_LIQ_ELL: e = eps_water_ellison(0.0, T_c, f); break;
    case PAMTRA_B200_LIQ_LIE: e = eps_water_liebe(T_c, f); break;
    case PAMTRA_B200_LIQ_RAY: e = eps_water_ray(T_c, f, bad); break;
    case PAMTRA_B200_LIQ_STO: e = eps_water_stogryn(0.0, T_c, f); break;
    default: e = eps_water_tkc(T_c, f); break;
  }
  return csqrt_(e);
}

// src/eps_ice.f90 + src/ref_ice.f90 (Maetzler ice)
__device__ cplx ref_ice(double T, double f) {
  double eps_real = (T >= 240.0) ? 3.1884 + 9.1e-4 * (T - 273.0) : 3.1884 + 9.1e-4 * (240.0 - 273.0);
  double mit = (300.0 / T) - 1.0;
  double alpha = (0.00504 + 0.0062 * mit) * exp(-22.1 * mit);
  double e = exp(335.0 / T);
  double beta_m = (0.0207 / T) * e / ((e - 1.0) * (e - 1.0));
  beta_m = beta_m + 1.16e-11 * (f * f);
  double delta_beta = exp(-9.963 + 0.0372 * (T - 273.16));
  double beta = beta_m + delta_beta;
  double eps_imag = (alpha / f) + beta * f;
  return csqrt_(cmk(eps_real, eps_imag));
}

// src/eps_mix.f90 with eps0 = 1: Sihvola mixing applied to the refractive
// index m of ice for a particle of density mix_de (mie_spheres.f90:139-144)
__device__ cplx eps_mix_m(cplx eps1, double mix_de) {
  const double v = 0.85, f = mix_de / 917.0, re1 = eps1.re, e0 = 1.0;
  double bb = re1 + 2.0 * e0 - 2.0 * v * e0 - f * (re1 - e0) * (1 + v);
  double aa = e0 * (re1 + (2.0 - v) * e0 + f * (2.0 - v) * (re1 - e0));
  double em_real = (sqrt(bb * bb + 4.0 * v * aa) - bb) / (2.0 * v);
  double em_imag = eps1.im * (-1.0 * (em_real - e0) + f * (em_real + 2.0 * e0 + v * (em_real - e0))) /
                   ((re1 + 2.0 * e0 + 2.0 * v * (em_real - e0)) - f * (1.0 + v) * (re1 - e0));
  return cmplx4(em_real, em_imag);  // CMPLX without KIND (eps_mix.f90:44)
}

// a / b as a conj(b) / |b|^2 (one division); the Mie coefficient
// denominators stay within a few hundred orders of magnitude of 1, so |b|^2
// neither overflows nor underflows.
__device__ __forceinline__ cplx cdiv_rcp(cplx a, cplx b) {
  const double s = 1.0 / (b.re * b.re + b.im * b.im);
  return cmk((a.re * b.re + a.im * b.im) * s, (a.im * b.re - a.re * b.im) * s);
}

__device__ __forceinline__ int mie_nstop(double x) { return (int)(x + 4.0 * pow(x, F(0.3334f)) + 2); }

// Refractive indices of liquid water (nmlSet['liq_mod']) and ice of every
// (present layer, frequency) item, ahead of k_mie (src/scatProperties.f90:
// 225-236): one thread per item; NaN marks a water model without a value.
__global__ void k_refr(Batch b, Work w, pamtra_b200_settings st) {
  const size_t item = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq;
  const int P = min(w.counters[0], w.pmax);
  if (item >= (size_t)P * Fm) return;
  const int p = (int)(item / Fm), f = (int)(item % Fm);
  const int cz = w.plist[p];
  const int c = cz / Lm, z = cz % Lm;
  if (f >= b.col_nfreq(c)) return;
  const double freq = b.freq(c, f);
  const double T = w.temp[(size_t)c * Lm + z];
  int bad = 0;
  const cplx mw = ref_water(T - F(273.15f), freq, st.liq_mod, &bad);
  const cplx mi = ref_ice(T, freq);
  double* o = w.m_refr + item * 4;
  o[0] = bad ? __longlong_as_double(0x7ff8000000000000ll) : mw.re;
  o[1] = mw.im;
  o[2] = mi.re;
  o[3] = mi.im;
}

// Per-bin Mie coefficients a_n, b_n of mie_scat_utilities.f90:8-116
// (miecalc + miecross) written into a column of the warp's coefficient slab
// as their sum and difference: row n-1 holds (u_n.re, u_n.im, v_n.re,
// v_n.im), u_n = a_n + b_n, v_n = a_n - b_n, rows ldc doubles apart.  The
// downward log-derivative recurrence parks d_n in the same rows first.
// Returns the efficiencies (from a_n, b_n); rows 0 .. nterms-1 are written.
__device__ __noinline__ void miecalc_slab(int nterms, double x, cplx mn, double* __restrict__ col, int ldc, double& qext,
                             double& qscat, double& qback) {
  const cplx m = cconj(mn);
  const cplx y = cscale(m, x);
  const int nn = nterms + 15;
  const cplx yinv = cdiv(cmk(1.0, 0.0), y), minv = cdiv(cmk(1.0, 0.0), m);
  // downward recurrence d(n-1) = n/y - 1/(d(n) + n/y), d(nn) = 0; keep d(1..nterms)
  cplx d = cmk(0.0, 0.0);
#pragma unroll 1
  for (int n = nn; n >= 2; n--) {
    const cplx ny = cscale(yinv, (double)n);
    // 1 / z as conj(z) / |z|^2: one division on the recurrence's critical path
    const cplx z = cadd(d, ny);
    const double s = 1.0 / (z.re * z.re + z.im * z.im);
    d = cmk(ny.re - z.re * s, ny.im + z.im * s);
    if (n - 1 <= nterms) *reinterpret_cast<double2*>(col + (size_t)(n - 2) * ldc) = make_double2(d.re, d.im);
  }
  double sx, cx;
  sincos(x, &sx, &cx);
  double psim = cx, psin = sx, chim = -sx, chin = cx;
  const double xinv = 1.0 / x;
  double sum1 = 0.0, sum2 = 0.0;
  cplx sum3 = cmk(0.0, 0.0);
#pragma unroll 1
  for (int n = 1; n <= nterms; n++) {
    double tmp = psin;
    psin = (2 * n - 1) * xinv * psin - psim;
    psim = tmp;
    tmp = chin;
    chin = (2 * n - 1) * xinv * chin - chim;
    chim = tmp;
    const cplx xin = cmplx4(psin, -chin), xim = cmplx4(psim, -chim);
    double* row = col + (size_t)(n - 1) * ldc;
    const double2 dv = *reinterpret_cast<const double2*>(row);
    const cplx dn = cmk(dv.x, dv.y);
    cplx ctmp = cmul(dn, minv);
    ctmp.re = ctmp.re + n * xinv;
    const cplx an = cdiv_rcp(cmk(ctmp.re * psin - psim, ctmp.im * psin), csub(cmul(ctmp, xin), xim));
    ctmp = cmul(m, dn);
    ctmp.re = ctmp.re + n * xinv;
    const cplx bn = cdiv_rcp(cmk(ctmp.re * psin - psim, ctmp.im * psin), csub(cmul(ctmp, xin), xim));
    *reinterpret_cast<double2*>(row) = make_double2(an.re + bn.re, an.im + bn.im);
    *reinterpret_cast<double2*>(row + 2) = make_double2(an.re - bn.re, an.im - bn.im);
    sum1 = sum1 + (2 * n + 1) * (an.re + bn.re);
    sum2 = sum2 + (2 * n + 1) * ((an.re * an.re - an.im * (-an.im)) + (bn.re * bn.re - bn.im * (-bn.im)));
    const double fac = (double)((float)(2 * n + 1) * ((n & 1) ? -1.0f : 1.0f));
    sum3 = cadd(sum3, cscale(csub(an, bn), fac));
  }
  qext = 2.0 / (x * x) * sum1;
  qscat = 2.0 / (x * x) * sum2;
  const cplx t = cscale(sum3, 1.0 / (x * x));
  qback = t.re * sum3.re - t.im * (-sum3.im);
}

// Phase-matrix elements P11, P12 (= P21) and P33 of one angle, summed over
// the bins j0 .. j0+GB-1 of a pass with their weights (mieangle,
// mie_scat_utilities.f90:119-160, and the PSD sums of mie_spheres.f90:
// 239-249).  With S+ = S1 + S2 = sum c_n u_n (pi_n + tau_n) and
// S- = S1 - S2 = sum c_n v_n (pi_n - tau_n) each term costs two complex
// multiply-adds instead of four, and
//   P11 = (|S1|^2 + |S2|^2) / 2 = (|S+|^2 + |S-|^2) / 4,
//   P12 = (|S2|^2 - |S1|^2) / 2 = -Re(S+ conj(S-)) / 2,
//   P33 = Re(S2 conj(S1))       = (|S+|^2 - |S-|^2) / 4.
// The pi_n / tau_n recurrence of the angle runs once for the group (rows
// of bins without particles, and rows past a bin's own term count, hold
// zeros).
constexpr int MIE_GROUP = 4;  // default bins per work item (the launch shape chooses 4 or 8)
template <int GB>
__device__ __forceinline__ void mie_angle_group(const double* __restrict__ slab, int ldc, int j0, int nmax, double mu,
                                                const double* __restrict__ wt, const double* __restrict__ dd, int nj,
                                                double* sum0, double* sum1, double* sum2) {
  double s[GB][4];  // S+ (re, im), S- (re, im)
#pragma unroll
  for (int j = 0; j < GB; j++) s[j][0] = s[j][1] = s[j][2] = s[j][3] = 0.0;
  double pin = 1.0, pim = 0.0;
  const double* row = slab + 4 * j0;
  for (int n = 1; n <= nmax; n++, row += ldc) {
    const double c = c_mie_c[n], rn = c_mie_inv[n];
    // tau_n = n mu pi_n - (n+1) pi_{n-1}, pi_{n+1} = ((2n+1) mu pi_n - (n+1) pi_{n-1}) / n
    const double mp = mu * pin, q = (double)(n + 1) * pim;
    const double taun = fma((double)n, mp, -q);
    const double cpl = c * (pin + taun), cmi = c * (pin - taun);
#pragma unroll
    for (int j = 0; j < GB; j++) {
      const double2 u = *reinterpret_cast<const double2*>(row + 4 * j);
      const double2 v = *reinterpret_cast<const double2*>(row + 4 * j + 2);
      s[j][0] = fma(u.x, cpl, s[j][0]);
      s[j][1] = fma(u.y, cpl, s[j][1]);
      s[j][2] = fma(v.x, cmi, s[j][2]);
      s[j][3] = fma(v.y, cmi, s[j][3]);
    }
    const double tmp = pin;
    pin = fma((double)(2 * n + 1), mp, -q) * rn;
    pim = tmp;
  }
  // add each bin's weighted elements to the angle's sums in bin order, so
  // that the sums do not depend on the number of bins per work item
  double a0 = sum0[0], a1 = sum1[0], a2 = sum2[0];
#pragma unroll
  for (int j = 0; j < GB; j++) {
    if (j >= nj || !(wt[j] > 0.0)) continue;
    const double ap = s[j][0] * s[j][0] + s[j][1] * s[j][1], am = s[j][2] * s[j][2] + s[j][3] * s[j][3];
    const double p0 = 0.25 * (ap + am), p2 = 0.25 * (ap - am);
    const double p1 = -0.5 * (s[j][0] * s[j][2] + s[j][1] * s[j][3]);
    a0 = a0 + (p0 * wt[j]) * dd[j];
    a1 = a1 + (p1 * wt[j]) * dd[j];
    a2 = a2 + (p2 * wt[j]) * dd[j];
  }
  sum0[0] = a0;
  sum1[0] = a1;
  sum2[0] = a2;
}

// Phase B of one pass (whole warp): item u = g * nquad + i is angle i over
// the bins of group g of the pass.  A round takes min(32, nquad) consecutive
// items, so its angles are distinct and each lane adds into its angle's sums
// without conflicts; rounds go in order, so every angle receives its bins in
// bin order whatever the group size.  Out of line so that the kernel's state
// is saved once per pass and the items keep the registers for their sums.
template <int GB>
__device__ __noinline__ void mie_pass_sums(MieSmem& S, const double* __restrict__ slab, int ldc, int cb, int nquad,
                                           const double* __restrict__ gx) {
  const int lane = threadIdx.x & 31;
  const int G = (cb + GB - 1) / GB;
  const int nu = G * nquad;
  const int W = min(32, nquad);
  for (int u0 = 0; u0 < nu; u0 += W) {
    const int u = u0 + lane;
    if (lane < W && u < nu) {
      const int g = u / nquad, i = u - g * nquad;
      const int j0 = GB * g, nj = min(GB, cb - j0);
      int nmax = 0;
      for (int j = 0; j < nj; j++) nmax = max(nmax, S.bn[j0 + j]);
      mie_angle_group<GB>(slab, ldc, j0, nmax, gx[i], S.bw + j0, S.bd + j0, nj, &S.sump[0][i], &S.sump[1][i],
                          &S.sump[2][i]);
    }
    __syncwarp();
  }
}

// One warp per (present layer, frequency) item; species loop in descriptor
// order.  src/scatProperties.f90:62-1002 (mie-sphere branch and the species
// sums :920-949, finalize :993) with src/mie_spheres.f90:14-345 per species.
// Per species the bins go in passes of up to 32: lanes over bins compute
// the Mie coefficients into the warp's slab (phase A), then lanes over
// (group of bins, angle) work items form the phase-function sums of
// the pass (phase B); each round of 32 items adds into the per-angle sums
// in lane order, so every result is independent of the launch shape.  The
// Legendre projection runs lanes over quadrature points with shuffle sums.
// The species sums accumulate in the item's coefficient output row.
template <int GB>
__global__ void __maxnreg__(MIE_MAXNREG) k_mie(Batch b, Work w, pamtra_b200_settings st) {
  extern __shared__ double smem_raw[];
  MieSmem& S = reinterpret_cast<MieSmem*>(smem_raw)[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const int gwarp = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (gwarp >= w.mie_nslab) return;
  double* const slab = w.mie_slab + (size_t)gwarp * MIE_SLAB_STRIDE;
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq, H = b.nhydro;
  const int P = min(w.counters[0], w.pmax);
  const int nitems = P * Fm;
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(&w.counters[1], 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nitems) break;
    const int p = item / Fm, f = item % Fm;
    const int cz = w.plist[p];
    const int c = cz / Lm, z = cz % Lm;
    if (f >= b.col_nfreq(c)) continue;
    const double freq = b.freq(c, f);
    const double wl = C_LIGHT / (freq * 1e9);
    double* const legc = slab + MIE_SLAB;  // species sums
    for (int jj = lane; jj < 3 * MAXNLEG; jj += 32) legc[jj] = 0.0;
    double kexttot = 0.0, salbedo = 0.0, backtot = 0.0;
    int nlegen_coef = 0;
    int status = 0;
    // save_psd per-bin backscatter: written at the column's last frequency
    double* const bscat = (w.psd_bscat && f == b.col_nfreq(c) - 1) ? w.psd_bscat : nullptr;
    for (int h = 0; h < H; h++) {
      const size_t s_idx = ((size_t)c * Lm + z) * H + h;
      if (w.slot_st[s_idx] != 2) continue;
      const pamtra_b200_species* spp = b.species + (size_t)c * b.species_stride + h;
      const int sp_liq_ice = spp->liq_ice;
      const double sp_as_ratio = spp->as_ratio;
      const int nb = w.slot_nb[s_idx];
      const size_t base = s_idx * (size_t)b.max_nbin;
      const double* bd = w.b_d + base;
      const double* bdd = w.b_dd + base;
      const double* bnd = w.b_nd + base;
      const double* brho = w.b_rho + base;
      const double* bmass = w.b_mass + base;
      const double* mr = w.m_refr + (size_t)item * 4 + (sp_liq_ice == 1 ? 0 : 2);
      const cplx mref = cmk(mr[0], mr[1]);
      if (isnan(mref.re)) {
        status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_RANGE;
        break;
      }
      const cplx m_ice = cmk(mref.re, -mref.im);
      // density / diameter of bin i (frequency-dependent soft spheroids of
      // make_soft_spheroid.f90:109-114 resolved here)
      auto dens_diam = [&](int i, double& rho, double& dia) {
        rho = brho[i];
        dia = bd[i];
        if (rho == -1.0) {
          const double mind = st.hydro_softsphere_min_density;
          rho = (sp_as_ratio == -20.) ? 0.863 * freq + 115.0 : 0.815 * freq + 11.2;
          if (rho < mind) rho = mind;
          dia = pow((6.0 * bmass[i]) / (PI * rho), 1.0 / 3.0);
          if (st.hydro_limit_density_area) {
            if (rho > RHO_ICE) rho = RHO_ICE;
            else if (rho < mind) rho = mind;
          }
        }
      };
      double rhoN, diaN;
      dens_diam(nb - 1, rhoN, diaN);
      const double xmax = PI * diaN / wl;
      const int nterms = mie_nstop(xmax);
      int nlegen = min(MAXNLEG - 1, 2 * nterms);
      const int nquad = (nlegen + 2 * nterms + 2) / 2;
      if (nquad > NQ_MAX || nquad > w.gq_max || nterms + 1 > NT_MAX) {
        status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE;
        break;
      }
      const double* gx = w.gq_x + (size_t)nquad * (nquad - 1) / 2;
      const double* gw = w.gq_w + (size_t)nquad * (nquad - 1) / 2;
      for (int i = lane; i < nquad; i += 32) { S.sump[0][i] = 0; S.sump[1][i] = 0; S.sump[2][i] = 0; }
      // rows the slab needs: every active bin's own series length, at least nterms
      int kmax = nterms;
      for (int ir = lane; ir < nb; ir += 32) {
        if (bnd[ir] / bdd[ir] > 0) {
          double rho, dia;
          dens_diam(ir, rho, dia);
          kmax = max(kmax, min(mie_nstop(PI * dia / wl), NT_MAX - 1));
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
      // bins per pass, a multiple of the group size so that no group runs past the slab's columns
      const int bp = min(32, MIE_SLAB / (4 * kmax)) & ~(GB - 1);
      const int ldc = 4 * bp;
      __syncwarp();
      double sqe = 0.0, sqs = 0.0, sqb = 0.0;
      for (int c0 = 0; c0 < nb; c0 += bp) {
        const int cb = min(bp, nb - c0);
        // ---- phase A: lane j < bp owns bin c0 + j (column j of the slab)
        if (lane < bp) {
          const int ir = c0 + lane;
          int nm = 0;
          double wgt = 0.0, deld = 0.0, qb_bin = 0.0, ndens = 0.0;
          double* col = slab + 4 * lane;
          if (lane < cb) {
            deld = bdd[ir];
            ndens = bnd[ir] / deld;
            if (ndens > 0) {
              double rho, dia;
              dens_diam(ir, rho, dia);
              const cplx ms = (sp_liq_ice == -1 && rho != 917.0) ? eps_mix_m(m_ice, rho) : m_ice;
              const double x = PI * dia / wl;
              int nmie = mie_nstop(x);
              if (nmie + 1 > NT_MAX) { nmie = NT_MAX - 1; status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE; }
              double qe, qs, qb;
              miecalc_slab(nmie, x, ms, col, ldc, qe, qs, qb);
              const double r2 = (dia / 2.0) * (dia / 2.0);
              qe = qe * r2 * PI;
              qs = qs * r2 * PI;
              qb = qb * r2 * PI;
              qe = qe * ndens;
              qs = qs * ndens;
              qb = qb * ndens;
              sqe = sqe + qe * deld;
              sqs = sqs + qs * deld;
              sqb = sqb + qb * deld;
              qb_bin = qb;
              nm = min(nmie, nterms);
              wgt = ndens;
            }
            // per-particle cross section as back_spec / num_density of
            // src/scatProperties.f90:916 (0 / 0 = NaN for an empty bin)
            if (bscat && ir < w.psd_nbin) bscat[s_idx * (size_t)w.psd_nbin + ir] = qb_bin / ndens;
          }
          for (int n = nm; n < nterms; n++)
            *reinterpret_cast<double4*>(col + (size_t)n * ldc) = make_double4(0.0, 0.0, 0.0, 0.0);
          S.bw[lane] = wgt;
          S.bd[lane] = deld;
          S.bn[lane] = nm;
        }
        __syncwarp();
        // ---- phase B: the phase-function sums of the pass
        mie_pass_sums<GB>(S, slab, ldc, cb, nquad, gx);
      }
      sqe = warp_sum(sqe);
      sqs = warp_sum(sqs);
      sqb = warp_sum(sqb);
      const double extinction = st.lhyd_absorption ? sqe : sqe - sqs;
      const double scatter = sqs;
      const double salb_h = scatter / extinction;
      const double tmp = (wl * wl / (PI * scatter));
      for (int i = lane; i < nquad; i += 32) {
        const double wt = gw[i];
#pragma unroll
        for (int k = 0; k < 3; k++) S.sump[k][i] = tmp * S.sump[k][i] * wt;
      }
      __syncwarp();
      // Legendre projection: coef_l = sum_i sump(i) P_l(mu_i), l = 0..nlegen,
      // in chunks of 64 quadrature points (two per lane); the chunk sums of
      // each order go into the slab (legh), in chunk order
      double* const legh = slab;  // [3][MAXNLEG]; the coefficients of the pass are no longer needed
      const double thr = F(1.0e-7f);
      for (int q0 = 0; q0 < nquad; q0 += 64) {
        const int i0 = q0 + lane, i1 = q0 + 32 + lane;
        const double mu0 = (i0 < nquad) ? gx[i0] : 0.0, mu1 = (i1 < nquad) ? gx[i1] : 0.0;
        double s0[3], s1[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
          s0[k] = (i0 < nquad) ? S.sump[k][i0] : 0.0;
          s1[k] = (i1 < nquad) ? S.sump[k][i1] : 0.0;
        }
        double pa = 1.0, pa1 = 1.0, pa2 = 0.0, pb = 1.0, pb1 = 1.0, pb2 = 0.0;
        for (int l = 0; l <= nlegen; l++) {
          if (l > 0) {
            pa = ((2 * l - 1) * mu0 * pa1 - (l - 1) * pa2) * c_mie_inv[l];
            pb = ((2 * l - 1) * mu1 * pb1 - (l - 1) * pb2) * c_mie_inv[l];
          }
          double acc[3];
#pragma unroll
          for (int k = 0; k < 3; k++) acc[k] = fma(s1[k], pb, fma(s0[k], pa, 0.0));
          pa2 = pa1;
          pa1 = pa;
          pb2 = pb1;
          pb1 = pb;
#pragma unroll
          for (int k = 0; k < 3; k++) acc[k] = warp_sum(acc[k]);
          if (lane == 0) {
#pragma unroll
            for (int k = 0; k < 3; k++) legh[k * MAXNLEG + l] = (q0 == 0) ? acc[k] : legh[k * MAXNLEG + l] + acc[k];
          }
        }
      }
      // orders past this species' series are zero in the species sums (mie_spheres.f90:309-316)
      for (int l = nlegen + 1 + lane; l < MAXNLEG; l += 32) {
#pragma unroll
        for (int k = 0; k < 3; k++) legh[k * MAXNLEG + l] = 0.0;
      }
      __syncwarp();
      int last = -1;
      for (int l = lane; l <= nlegen; l += 32) {
        const double fac = (double)((float)(2 * l + 1) / 2.0f);  // REAL(4) division, exact
#pragma unroll
        for (int k = 0; k < 3; k++) legh[k * MAXNLEG + l] = fac * legh[k * MAXNLEG + l];
        if (legh[l] > thr) last = l;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) last = max(last, __shfl_xor_sync(0xffffffffu, last, o));
      __syncwarp();
      const int nlegen_h = (last >= 0) ? last : nlegen;  // mie_spheres.f90:307-314
      if (!(extinction > 0) || !(scatter > 0) || !(sqb > 0) || isnan(extinction)) {
        status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_MIE;
        break;
      }
      // species sums (scatProperties.f90:920-949); the backscattering sum is
      // radar_simulator's input (mie_spheres.f90:263, scatProperties.f90:922)
      nlegen_coef = max(nlegen_coef, nlegen_h);
      kexttot = kexttot + extinction;
      backtot = backtot + sqb;
      if (kexttot == 0.0) salbedo = 0.0;
      else salbedo = salbedo + (salb_h * extinction);
      for (int jj = lane; jj < nlegen_coef; jj += 32) {
#pragma unroll
        for (int k = 0; k < 3; k++)
          legc[k * MAXNLEG + jj] = legc[k * MAXNLEG + jj] + (legh[k * MAXNLEG + jj] * salb_h * extinction);
      }
      __syncwarp();
      if (nlegen_coef > MAXNLEG - 1) { status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE; break; }
    }
    // finalize_rt3_scatProperties (scatProperties.f90:993-1002) into the
    // item's coefficient row: FP64, or FP32 storage in the split-precision form
    salbedo = salbedo / kexttot;
    const double den = salbedo * kexttot;
    double* const out64 = w.m_legen ? w.m_legen + (size_t)item * 3 * MAXNLEG : nullptr;
    float* const out32 = w.m_legen32 ? w.m_legen32 + (size_t)item * 3 * MAXNLEG : nullptr;
    for (int jj = lane; jj < MAXNLEG; jj += 32) {
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double v = 0.0;
        if (jj <= nlegen_coef) {
          v = legc[k * MAXNLEG + jj] / den;
          if (isnan(v) && nlegen_coef > 0) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_NAN;
        }
        if (out64) out64[k * MAXNLEG + jj] = v;
        else out32[k * MAXNLEG + jj] = (float)v;
      }
    }
    status = __reduce_or_sync(0xffffffffu, status);
    if (lane == 0) {
      w.m_kext[item] = kexttot;
      w.m_salb[item] = salbedo;
      w.m_back[item] = backtot;
      w.m_nleg[item] = nlegen_coef;
      if (w.wt_need && nlegen_coef > 0) {
        const int numpts = 2 * ((nlegen_coef + 1) / 2) + 4;
        w.wt_need[nmu_index(b.col_nummu(c)) * SCAT_NPI + (numpts - 4) / 2] = 1;
      }
      if (status) atomicOr(&w.status[(size_t)c * Fm + f], status);
    }
    __syncwarp();
  }
}

}  // namespace pb
