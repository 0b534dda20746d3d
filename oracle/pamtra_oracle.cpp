// Test infrastructure only (see oracle_common.h): CPU FP64 restatement of the
// reference PAMTRA passive forward path for one atmospheric column and a list
// of frequencies.  Product code never links or calls this file.
//
// Reference routines restated here, in call order (paths inside the reference
// project):
//   src/vars_atmosphere.f90:671-901   fillMissing_atmosphere_vars
//   src/e_sat_gg_water.f90:1-21       e_sat_gg_water
//   src/get_gasabs.f90:76-104         get_gasabs (R98 branch)
//   src/rosen98_gasabs.f90:2-153      rosen98_gasabs
//   src/gasabs_module.f90:83-333      absn2, o2abs, abh2o
//   src/hydrometeor_extinction.f90    layer x species loop
//   src/conversions.f90:5-24          q2abs
//   src/drop_size_dist.f90:107-218    run_drop_size_dist
//   src/make_mass_size.f90            make_mass_size
//   src/make_dist_param.f90           make_dist_params (exp, exp_field_t,
//                                     exp_ryan, mgamma, mono, logn)
//   src/make_dist.f90                 make_dist
//   src/make_soft_spheroid.f90        make_soft_spheroid
//   src/scatProperties.f90:62-1002    calc_scatProperties (mie-sphere branch)
//   src/ref_water.f90, eps_water.f90:653-757 (TKC), ref_ice.f90, eps_ice.f90,
//   src/eps_mix.f90                   refractive indices
//   src/mie_spheres.f90               calc_mie_spheres
//   src/mie_scat_utilities.f90:8-160  miecalc, miecross, mieangle
//   src/scat_utilities.f90            gausquad
//   src/scatcnv.f90                   scatcnv, transform_scatter, transform_ext_emis
//   src/rt_utilities.f90              PLANCK_FUNCTION, LOBATTO_QUADRATURE,
//                                     NUMBER_SUMS, SUM_LEGENDRE,
//                                     ROTATE_PHASE_MATRIX, MATRIX_SYMMETRY,
//                                     FOURIER_BASIS (order 0), CONVERT_OUTPUT
//   src/rt4.f90:185-356, radtran4.f90, radintg4.f90:1-513, radscat4.f90:87-136,
//   src/radmat.f90:137-233, sfc_matrices.f90, surface.f90:169-195,
//   src/sfc_optics.f90:79-81, collect_output.f90, run_rt.f90
//
// Matrix inversion follows LAPACK's published DGETF2 + DGETRI (unblocked)
// algorithm, which the reference reaches through OpenBLAS 0.3.34
// (radmat.f90:201-233).  gfortran MATMUL is restated as k-ascending dot
// products.
#include "oracle_common.h"
#include "ray_table.inc"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <limits>

using namespace orc;

namespace {

const double NaN = std::numeric_limits<double>::quiet_NaN();

// gfortran expands x**n (integer constant n) with GCC's powi multiplication
// chains: x**2 = x*x, x**3 = x**2*x, x**5 = x**3*x**2.
inline double p2(double x) { return x * x; }
inline double p3(double x) { double x2 = x * x; return x2 * x; }
inline double p5(double x) { double x2 = x * x; double x3 = x2 * x; return x3 * x2; }

// ---------------------------------------------------------------- atmosphere
// src/e_sat_gg_water.f90:1-21 (all constants are default REAL)
double e_sat_gg_water(double T) {
  const double a = F(1013.246f), b = F(7.90298f), t0 = F(373.16f), c = F(5.02808f), d = F(1.3816e-7f),
               e = F(11.344f), g = F(8.1328e-3f), h = F(3.49149f);
  double ex = -(b * (t0 / T - 1)) + c * std::log10(t0 / T) - d * (std::pow(10.0, e * (1 - T / t0)) - 1) +
              g * (std::pow(10.0, -(h * (t0 / T - 1))) - 1);
  return a * std::pow(10.0, ex);
}

struct Atmo {
  int L;
  std::vector<double> hgt_lev, temp_lev, press_lev, relhum_lev;
  std::vector<double> hgt, temp, press, relhum, delta_hgt, vapor_pressure, rho_vap, q_hum;
  double groundtemp;
};

// src/vars_atmosphere.f90:671-901 fillMissing_atmosphere_vars (one column)
void fill_missing(Atmo& a) {
  const int L = a.L;
  auto& hl = a.hgt_lev; auto& tl = a.temp_lev; auto& pl = a.press_lev; auto& rl = a.relhum_lev;
  auto& h = a.hgt; auto& t = a.temp; auto& p = a.press; auto& r = a.relhum;
  for (int nz = 0; nz < L; nz++)
    if (std::isnan(h[nz])) h[nz] = 0.5 * (hl[nz] + hl[nz + 1]);
  if (std::isnan(hl[0])) hl[0] = h[0] - (h[1] - h[0]) * 0.5;
  if (std::isnan(tl[0])) tl[0] = t[0] - (t[1] - t[0]) / (h[1] - h[0]) * (h[0] - hl[0]);
  if (std::isnan(rl[0])) rl[0] = r[0] - (r[1] - r[0]) / (h[1] - h[0]) * (h[0] - hl[0]);
  if (std::isnan(pl[0]))
    pl[0] = std::exp(std::log(p[0]) - (std::log(p[1]) - std::log(p[0])) / (h[1] - h[0]) * (h[0] - hl[0]));
  for (int nz = 1; nz < L; nz++) {
    if (std::isnan(tl[nz])) tl[nz] = 0.5 * (t[nz] + t[nz - 1]);
    if (std::isnan(hl[nz])) hl[nz] = 0.5 * (h[nz] + h[nz - 1]);
    if (std::isnan(rl[nz])) rl[nz] = 0.5 * (r[nz] + r[nz - 1]);
    if (std::isnan(pl[nz])) pl[nz] = std::exp(0.5 * (std::log(p[nz]) + std::log(p[nz - 1])));
  }
  {
    int nz = L;  // level L+1 (1-based)
    if (std::isnan(hl[nz])) hl[nz] = h[nz - 1] + (h[nz - 1] - h[nz - 2]) * 0.5;
    if (std::isnan(tl[nz]))
      tl[nz] = t[nz - 1] + (t[nz - 1] - t[nz - 2]) / (h[nz - 1] - h[nz - 2]) * (hl[nz] - h[nz - 1]);
    if (std::isnan(rl[nz]))
      rl[nz] = r[nz - 1] + (r[nz - 1] - r[nz - 2]) / (h[nz - 1] - h[nz - 2]) * (hl[nz] - h[nz - 1]);
    if (std::isnan(pl[nz]))
      pl[nz] = std::exp(std::log(p[nz - 1]) + (std::log(p[nz - 1]) - std::log(p[nz - 2])) /
                                                  (h[nz - 1] - h[nz - 2]) * (hl[nz] - h[nz - 1]));
  }
  a.delta_hgt.assign(L, NaN);
  a.vapor_pressure.assign(L, NaN);
  a.rho_vap.assign(L, NaN);
  a.q_hum.assign(L, NaN);
  for (int nz = 0; nz < L; nz++) {
    if (std::isnan(t[nz])) t[nz] = 0.5 * (tl[nz] + tl[nz + 1]);
    if (std::isnan(r[nz])) r[nz] = 0.5 * (rl[nz] + rl[nz + 1]);
    if (std::isnan(p[nz])) p[nz] = std::exp(0.5 * (std::log(pl[nz]) + std::log(pl[nz + 1])));
    if (std::isnan(h[nz])) h[nz] = (hl[nz] + hl[nz + 1]) * 0.5;
    a.delta_hgt[nz] = hl[nz + 1] - hl[nz];
    a.vapor_pressure[nz] = r[nz] * e_sat_gg_water(t[nz]);
    a.rho_vap[nz] = a.vapor_pressure[nz] / (t[nz] * R_V);
    a.q_hum[nz] = R_V / R_D * a.vapor_pressure[nz] / (p[nz] - (1.0 - R_V / R_D) * a.vapor_pressure[nz]);
  }
  if (std::isnan(a.groundtemp)) a.groundtemp = tl[0];
}

// ---------------------------------------------------------------- gas (R98)
// src/gasabs_module.f90:83-104 absn2
double absn2(double T, double pres, double f) {
  double th = 300.0 / T;
  return 6.4e-14 * pres * pres * f * f * std::pow(th, 3.55);
}

// src/gasabs_module.f90:106-211 o2abs (tables are default REAL)
const float O2_W300[40] = {1.63f, 1.646f, 1.468f, 1.449f, 1.382f, 1.360f, 1.319f, 1.297f, 1.266f, 1.248f,
                           1.221f, 1.207f, 1.181f, 1.171f, 1.144f, 1.139f, 1.110f, 1.108f, 1.079f, 1.078f,
                           1.05f,  1.05f,  1.02f,  1.02f,  1.0f,   1.0f,   0.97f,  0.97f,  0.94f,  0.94f,
                           0.92f,  0.92f,  0.89f,  0.89f,  1.92f,  1.92f,  1.92f,  1.81f,  1.81f,  1.81f};
const float O2_Y300[40] = {-0.0233f, 0.2408f,  -0.3486f, 0.5227f,  -0.5430f, 0.5877f,  -0.3970f, 0.3237f,
                           -0.1348f, 0.0311f,  0.0725f,  -0.1663f, 0.2832f,  -0.3629f, 0.3970f,  -0.4599f,
                           0.4695f,  -0.5199f, 0.5187f,  -0.5597f, 0.5903f,  -0.6246f, 0.6656f,  -0.6942f,
                           0.7086f,  -0.7325f, 0.7348f,  -0.7546f, 0.7702f,  -0.7864f, 0.8083f,  -0.8210f,
                           0.8439f,  -0.8529f, 0.f,      0.f,      0.f,      0.f,      0.f,      0.f};
const float O2_V[40] = {0.0079f,  -0.0978f, 0.0844f,  -0.1273f, 0.0699f,  -0.0776f, 0.2309f,  -0.2825f,
                        0.0436f,  -0.0584f, 0.6056f,  -0.6619f, 0.6451f,  -0.6759f, 0.6547f,  -0.6675f,
                        0.6135f,  -0.6139f, 0.2952f,  -0.2895f, 0.2654f,  -0.2590f, 0.3750f,  -0.3680f,
                        0.5085f,  -0.5002f, 0.6206f,  -0.6091f, 0.6526f,  -0.6393f, 0.6640f,  -0.6475f,
                        0.6729f,  -0.6545f, 0.f,      0.f,      0.f,      0.f,      0.f,      0.f};
const float O2_F[40] = {118.7503f, 56.2648f, 62.4863f, 58.4466f, 60.3061f, 59.5910f, 59.1642f, 60.4348f,
                        58.3239f,  61.1506f, 57.6125f, 61.8002f, 56.9682f, 62.4112f, 56.3634f, 62.9980f,
                        55.7838f,  63.5685f, 55.2214f, 64.1278f, 54.6712f, 64.6789f, 54.1300f, 65.2241f,
                        53.5957f,  65.7648f, 53.0669f, 66.3021f, 52.5424f, 66.8368f, 52.0214f, 67.3696f,
                        51.5034f,  67.9009f, 368.4984f, 424.7631f, 487.2494f, 715.3932f, 773.8397f, 834.1453f};
const float O2_S300[40] = {0.2936E-14f, 0.8079E-15f, 0.2480E-14f, 0.2228E-14f, 0.3351E-14f, 0.3292E-14f,
                           0.3721E-14f, 0.3891E-14f, 0.3640E-14f, 0.4005E-14f, 0.3227E-14f, 0.3715E-14f,
                           0.2627E-14f, 0.3156E-14f, 0.1982E-14f, 0.2477E-14f, 0.1391E-14f, 0.1808E-14f,
                           0.9124E-15f, 0.1230E-14f, 0.5603E-15f, 0.7842E-15f, 0.3228E-15f, 0.4689E-15f,
                           0.1748E-15f, 0.2632E-15f, 0.8898E-16f, 0.1389E-15f, 0.4264E-16f, 0.6899E-16f,
                           0.1924E-16f, 0.3229E-16f, 0.8191E-17f, 0.1423E-16f, 0.6460E-15f, 0.7047E-14f,
                           0.3011E-14f, 0.1826E-14f, 0.1152E-13f, 0.3971E-14f};
const float O2_BE[40] = {0.009f, 0.015f, 0.083f, 0.084f, 0.212f, 0.212f, 0.391f, 0.391f, 0.626f, 0.626f,
                         0.915f, 0.915f, 1.26f,  1.26f,  1.66f,  1.665f, 2.119f, 2.115f, 2.624f, 2.625f,
                         3.194f, 3.194f, 3.814f, 3.814f, 4.484f, 4.484f, 5.224f, 5.224f, 6.004f, 6.004f,
                         6.844f, 6.844f, 7.744f, 7.744f, 0.048f, 0.044f, 0.049f, 0.145f, 0.141f, 0.145f};

double o2abs(double T, double pres, double vapden, double f) {
  const double x = F(0.8f), wb300 = F(0.56f);
  double th = 300.0 / T;
  double th1 = th - 1.0;
  double b = std::pow(th, x);
  double preswv = vapden * T / 217.0;
  double presda = pres - preswv;
  double den = 0.001 * (presda * b + 1.1 * preswv * th);
  double dfnr = wb300 * den;
  double sum = 1.6e-17 * f * f * dfnr / (th * (f * f + dfnr * dfnr));
  for (int k = 0; k < 40; k++) {
    double fk = F(O2_F[k]);
    double df = F(O2_W300[k]) * den;
    double y = 0.001 * pres * b * (F(O2_Y300[k]) + F(O2_V[k]) * th1);
    double str = F(O2_S300[k]) * std::exp(-(F(O2_BE[k]) * th1));
    double sf1 = (df + (f - fk) * y) / (p2(f - fk) + df * df);
    double sf2 = (df - (f + fk) * y) / (p2(f + fk) + df * df);
    sum = sum + str * (sf1 + sf2) * p2(f / fk);
  }
  return 0.5034e12 * sum * presda * p3(th) / PI;
}

// src/gasabs_module.f90:214-333 abh2o (tables are default REAL)
const float H2O_FL[15] = {22.2351f, 183.3101f, 321.2256f, 325.1529f, 380.1974f, 439.1508f, 443.0183f, 448.0011f,
                          470.8890f, 474.6891f, 488.4911f, 556.9360f, 620.7008f, 752.0332f, 916.1712f};
const float H2O_S1[15] = {0.1310E-13f, 0.2273E-11f, 0.8036E-13f, 0.2694E-11f, 0.2438E-10f,
                          0.2179E-11f, 0.4624E-12f, 0.2562E-10f, 0.8369E-12f, 0.3263E-11f,
                          0.6659E-12f, 0.1531E-08f, 0.1707E-10f, 0.1011E-08f, 0.4227E-10f};
const float H2O_B2[15] = {2.144f, .668f, 6.179f, 1.541f, 1.048f, 3.595f, 5.048f, 1.405f,
                          3.597f, 2.379f, 2.852f, .159f,  2.391f, .396f,  1.441f};
const float H2O_W3[15] = {0.002656f, 0.00281f, 0.0023f,  0.00278f, 0.00287f, 0.0021f,  0.00186f, 0.00263f,
                          0.00215f,  0.00236f, 0.0026f,  0.00321f, 0.00244f, 0.00306f, 0.00267f};
const float H2O_X[15] = {0.69f, 0.64f, 0.67f, 0.68f, 0.54f, 0.63f, 0.60f, 0.66f,
                         0.66f, 0.65f, 0.69f, 0.69f, 0.71f, 0.68f, 0.70f};
const float H2O_WS[15] = {0.0127488f, 0.01491f, 0.0108f,  0.0135f,  0.01541f, 0.0090f,  0.00788f, 0.01275f,
                          0.00983f,   0.01095f, 0.01313f, 0.01320f, 0.01140f, 0.01253f, 0.01275f};
const float H2O_XS[15] = {0.61f, 0.85f, 0.54f, 0.74f, 0.89f, 0.52f, 0.50f, 0.67f,
                          0.65f, 0.64f, 0.72f, 1.0f,  0.68f, 0.84f, 0.78f};

double abh2o(double T, double pres, double rho, double f) {
  if (rho <= 0.0) return 0.0;
  double pvap = rho * T / 217.0;
  double pda = pres - pvap;
  double den = 3.335e16 * rho;
  double ti = 300.0 / T;
  double ti2 = std::pow(ti, 2.5);
  double con = (5.43e-10 * 1.105 * pda * p3(ti) + 1.8e-8 * 0.79 * pvap * std::pow(ti, 7.5)) * pvap * f * f;
  double sum = 0.0;
  for (int i = 0; i < 15; i++) {
    double fl = F(H2O_FL[i]);
    double width = F(H2O_W3[i]) * pda * std::pow(ti, F(H2O_X[i])) + F(H2O_WS[i]) * pvap * std::pow(ti, F(H2O_XS[i]));
    double wsq = width * width;
    double s = F(H2O_S1[i]) * ti2 * std::exp(F(H2O_B2[i]) * (1.0 - ti));
    double df[2] = {f - fl, f + fl};
    double base = width / (562500.0 + wsq);
    double res = 0.0;
    for (int j = 0; j < 2; j++)
      if (std::fabs(df[j]) < 750.0) res = res + width / (p2(df[j]) + wsq) - base;
    sum = sum + s * res * p2(f / fl);
  }
  return 0.3183e-4 * den * sum + con;
}

// src/rosen98_gasabs.f90:2-153 + src/get_gasabs.f90:88-95 -> Np/m
int gas_r98(double f, double T, double rhowv, double pres, double* kext) {
  if (f <= 0.0 || f > 800.0) return 2;
  if (T <= 100.0) return 2;
  if (pres <= 0.0 || pres > 1.2e5) return 2;
  double pmb = pres / 100.0;
  double vapden = rhowv * 1000.0;
  double absair = absn2(T, pmb, f) + o2abs(T, pmb, vapden, f);
  double abswv = abh2o(T, pmb, vapden, f);
  *kext = (absair + abswv) / 1.0e3;
  return 0;
}


// ---------------------------------------------------------------- other liquid water models
// src/eps_water.f90 (nmlSet['liq_mod']).  gfortran semantics restated: a
// literal without kind is a REAL(4) value (float literal here) promoted in
// mixed expressions; the routines' pi parameter is that REAL(4) value; a
// complex constant (0.,1.) times a real is (0, 1*x); CMPLX without KIND is
// COMPLEX(4).  Salinity is 0 (src/scatProperties.f90:228).
static const double PI4 = (double)3.141592653589793f;

// eps_water_ellison (src/eps_water.f90:85-158)
cplx eps_water_ellison(double s, double T, double f) {
  static const float a[18] = {0.46606917e-02f, -0.26087876e-04f, -0.63926782e-05f, 0.63000075e+01f,
                              0.26242021e-02f, -0.42984155e-02f, 0.34414691e-04f, 0.17667420e-03f,
                              -0.20491560e-06f, 0.58366888e+03f, 0.12634992e+03f, 0.69227972e-04f,
                              0.38957681e-06f, 0.30742330e+03f, 0.12634992e+03f, 0.37245044e+01f,
                              0.92609781e-02f, -0.26093754e-01f};
  auto A = [&](int i) { return (double)a[i - 1]; };
  double p = s * (37.5109f + 5.45216f * s + 0.014409f * p2(s)) / (1004.75f + 182.283f * s + p2(s));
  double alpha_0 = (6.9431f + 3.2841f * s - 0.099486f * p2(s)) / (84.85f + 69.024f * s + p2(s));
  double alpha_1 = 49.843f - 0.2276f * s + 0.00198f * p2(s);
  double sig_s35 = 2.903602f + 8.607e-02f * T + 4.738817e-04f * p2(T) - 2.991e-06f * p3(T) + 4.3041e-09f * (p2(T) * p2(T));
  double eps_s = 87.85306f * std::exp(-0.00456992f * T - A(1) * s - A(2) * p2(s) - A(3) * s * T);
  double eps_1 = A(4) * std::exp(-A(5) * T - A(6) * s - A(7) * s * T);
  double tau_1 = (A(8) + A(9) * s) * std::exp(A(10) / (T + A(11)));
  double tau_2 = (A(12) + A(13) * s) * std::exp(A(14) / (T + A(15)));
  double eps_inf = A(16) + A(17) * T + A(18) * s;
  double q = 1 + (alpha_0 * (T - 15)) / (T + alpha_1);
  double sig = sig_s35 * p * q;
  cplx t1 = cdiv(cmk(eps_s - eps_1, 0.0), cmk(1.0, -(2 * PI4 * f * tau_1)));
  cplx t2 = cdiv(cmk(eps_1 - eps_inf, 0.0), cmk(1.0, -(2 * PI4 * f * tau_2)));
  cplx e = cadd(cadd(t1, t2), cmk(eps_inf, 0.0));
  return cadd(e, cmk(0.0, (double)17.9751f * sig / f));
}

// eps_water_liebe (src/eps_water.f90:160-207)
cplx eps_water_liebe(double T, double f) {
  double T_K = T + 273.15f;
  double theta_1 = 1. - 300. / T_K;
  double fp = 20.1f * std::exp(7.88f * theta_1);
  double fs = 39.8f * fp;
  double eps_0 = 77.66f - 103.3f * theta_1;
  double eps_1 = 0.0671f * eps_0;
  double eps_2 = 3.52f;
  cplx e = cadd(cdiv(cmk(eps_0 - eps_1, 0.0), cmplx4(1., -f / fp)), cdiv(cmk(eps_1 - eps_2, 0.0), cmplx4(1., -f / fs)));
  return cadd(e, cmk(eps_2, 0.0));
}

// eps_water_ray (src/eps_water.f90:215-592): 0.2 um - 1 mm linear
// interpolation in the tabulated optical constants (:515-537, first table
// wavelength at or above wl, scanning from the second), 1 mm - 10 cm the
// Ray (1972) formula (:539-585); returns 2 outside 0.2 um - 10 cm (the
// reference stops there).
int eps_water_ray(double T, double f, cplx& eps) {
  double wl = (double)(1.e6f * 2.99792458e8f) / (f * 1.e9f);
  if (wl < (double)0.2f || wl > 100000.0 || wl != wl) return 2;
  if (!(wl > 1000.0)) {
    int i1 = RAY_NUMWAT - 3, i2 = RAY_NUMWAT - 2;
    for (int i = 1; i < RAY_NUMWAT; ++i) {
      if (wl > (double)ray_wl[i]) continue;
      i1 = i - 1;
      i2 = i;
      break;
    }
    double fac = (wl - (double)ray_wl[i1]) / ((double)ray_wl[i2] - (double)ray_wl[i1]);
    double rn = (double)ray_rn[i1] + fac * ((double)ray_rn[i2] - (double)ray_rn[i1]);
    double cn = (double)ray_cn[i1] + fac * ((double)ray_cn[i2] - (double)ray_cn[i1]);
    eps = cmul(cmk(rn, cn), cmk(rn, cn));
    return 0;
  }
  double T1 = T + 273.0f, T2 = T - 25.0f, xl = wl / 10000.0f;
  double sigma = 12.5664e8f;
  double alpha = -16.8129f / T1 + 0.0609265f;
  double eps_s = 78.54f * (1.0f - 4.579e-3f * T2 + 1.19e-5f * p2(T2) - 2.8e-8f * p3(T2));
  double eps_inf = 5.27137f + 0.0216474f * T - 0.00131198f * p2(T);
  double xlams = 0.00033836f * std::exp(2513.98f / T1);
  double powtrm = std::pow(xlams / xl, 1.f - alpha);
  double denom = 1.f + 2 * powtrm * std::sin(PI4 * alpha / 2) + std::pow(xlams / xl, 2.f * (1.f - alpha));
  double eps_r = eps_inf + (eps_s - eps_inf) * (1.0f + powtrm * std::sin(PI4 * alpha / 2)) / denom;
  double eps_i = (sigma * xl / (double)18.8496e10f) + (eps_s - eps_inf) * powtrm * std::cos(PI4 * alpha / 2) / denom;
  cplx n = csqrt_(cmk(eps_r, eps_i));
  double rn = n.re, cn = n.im;
  if (!(wl > 3000.0f))
    cn = cn + 0.39f * std::exp(-std::pow(std::fabs(std::log10(wl / 17.0f) / 0.45f), (double)1.3f)) +
         0.41f * std::exp(-std::pow(std::fabs(std::log10(wl / 62.0f) / 0.35f), (double)1.7f)) +
         0.25f * std::exp(-std::pow(std::fabs(std::log10(wl / 300.0f) / 0.47f), 3.0));
  eps = cmul(cmk(rn, cn), cmk(rn, cn));
  return 0;
}

// eps_water_stogryn (src/eps_water.f90:598-651)
cplx eps_water_stogryn(double s, double T, double f) {
  double p = s * (37.5109f + 5.45216f * s + 0.014409f * p2(s)) / (1004.75f + 182.283f * s + p2(s));
  double alpha_0 = (6.9431f + 3.2841f * s - 0.099486f * p2(s)) / (84.85f + 69.024f * s + p2(s));
  double alpha_1 = 49.843f - 0.2276f * s + 0.00198f * p2(s);
  double sig_s35 = 2.903602f + 8.607e-02f * T + 4.738817e-04f * p2(T) - 2.991e-06f * p3(T) + 4.3041e-09f * (p2(T) * p2(T));
  double a = 1.f - (s * (0.03838f + 0.00218f * s) * (79.88f + T)) / ((12.01f + s) * (52.53f + T));
  double b = 1.f - s * ((0.03409f + 0.002817f * s) / (7.69f + s)) -
             s * T * ((0.00246f + 0.00141f * T) / (188.f - 7.57f * T + p2(T)));
  double es = (37088.6f - 82.168f * T) / (421.854f + T);
  double eps_s = es * a;
  double eps_1 = (0.0787f * es) * a;
  double tpt1 = ((255.04f + 0.7246f * T) / ((49.25f + T) * (45.f + T))) * b;
  double tpt2 = 0.00628f;
  double eps_inf = 4.05f + 0.0186f * T;
  double q = 1 + (alpha_0 * (T - 15)) / (T + alpha_1);
  double sig = sig_s35 * p * q;
  cplx t1 = cdiv(cmk(eps_s - eps_1, 0.0), cmk(1.0, -(f * tpt1)));
  cplx t2 = cdiv(cmk(eps_1 - eps_inf, 0.0), cmk(1.0, -(f * tpt2)));
  cplx e = cadd(cadd(t1, t2), cmk(eps_inf, 0.0));
  return cadd(e, cmk(0.0, (double)17.9751f * sig / f));
}

cplx eps_water_tkc(double T, double f);

// src/ref_water.f90 + get_eps_water (src/eps_water.f90:39-63) for every liq_mod;
// returns 2 where the model has no value.
int ref_water_mod(int liq_mod, double T_c, double f, double& refre, double& refim) {
  cplx e;
  switch (liq_mod) {
    case 1: e = eps_water_ellison(0.0, T_c, f); break;
    case 2: e = eps_water_liebe(T_c, f); break;
    case 3:
      if (eps_water_ray(T_c, f, e)) return 2;
      break;
    case 4: e = eps_water_stogryn(0.0, T_c, f); break;
    default: e = eps_water_tkc(T_c, f); break;
  }
  cplx r = csqrt_(e);
  refre = r.re;
  refim = r.im;
  return 0;
}

// ---------------------------------------------------------------- gas_mod 'L93'
// src/mpm93.f90: line catalogue of Liebe, Hufford and Cotton (1993) as the
// reference declares it (REAL(4) literals, :131-222).
static const float L93_F0O2[44] = {
    50.474239f, 50.987747f, 51.503349f, 52.021412f, 52.542393f, 53.066906f, 53.595749f, 54.130001f,
    54.671158f, 55.221367f, 55.783802f, 56.264774f, 56.363388f, 56.968204f, 57.612484f, 58.323875f,
    58.446590f, 59.164207f, 59.590984f, 60.306061f, 60.434776f, 61.150558f, 61.800156f, 62.411217f,
    62.486259f, 62.997978f, 63.568520f, 64.127769f, 64.678902f, 65.224068f, 65.764771f, 66.302094f,
    66.836830f, 67.369598f, 67.900864f, 68.431007f, 68.960312f, 118.750343f, 368.498352f, 424.763123f,
    487.249359f, 715.393127f, 773.839661f, 834.145325f};
static const float L93_A1[44] = {
    0.094f, 0.246f, 0.608f, 1.414f, 3.102f, 6.410f, 12.470f, 22.800f,
    39.180f, 63.160f, 95.350f, 54.890f, 134.400f, 176.300f, 214.100f, 238.600f,
    145.700f, 240.400f, 211.200f, 212.400f, 246.100f, 250.400f, 229.800f, 193.300f,
    151.700f, 150.300f, 108.700f, 73.350f, 46.350f, 27.480f, 15.300f, 8.009f,
    3.946f, 1.832f, 0.801f, 0.330f, 0.128f, 94.500f, 6.790f, 63.800f,
    23.500f, 9.960f, 67.100f, 18.000f};
static const float L93_A2[44] = {
    9.694f, 8.694f, 7.744f, 6.844f, 6.004f, 5.224f, 4.484f, 3.814f,
    3.194f, 2.624f, 2.119f, 0.015f, 1.660f, 1.260f, 0.915f, 0.626f,
    0.084f, 0.391f, 0.212f, 0.212f, 0.391f, 0.626f, 0.915f, 1.260f,
    0.083f, 1.665f, 2.115f, 2.620f, 3.195f, 3.815f, 4.485f, 5.225f,
    6.005f, 6.845f, 7.745f, 8.695f, 9.695f, 0.009f, 0.049f, 0.044f,
    0.049f, 0.145f, 0.130f, 0.147f};
static const float L93_A3[44] = {
    0.890f, 0.910f, 0.940f, 0.970f, 0.990f, 1.020f, 1.050f, 1.070f,
    1.100f, 1.130f, 1.170f, 1.730f, 1.200f, 1.240f, 1.280f, 1.330f,
    1.520f, 1.390f, 1.430f, 1.450f, 1.360f, 1.310f, 1.270f, 1.230f,
    1.540f, 1.200f, 1.170f, 1.130f, 1.100f, 1.070f, 1.050f, 1.020f,
    0.990f, 0.970f, 0.940f, 0.920f, 0.900f, 1.630f, 1.920f, 1.930f,
    1.920f, 1.810f, 1.820f, 1.810f};
static const float L93_A4[44] = {
    0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f,
    0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f,
    0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f,
    0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f,
    0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.000f, 0.600f, 0.600f,
    0.600f, 0.600f, 0.600f, 0.600f};
static const float L93_A5[44] = {
    0.240f, 0.220f, 0.197f, 0.166f, 0.136f, 0.131f, 0.230f, 0.335f,
    0.374f, 0.258f, -0.166f, 0.390f, -0.297f, -0.416f, -0.613f, -0.205f,
    0.748f, -0.722f, 0.765f, -0.705f, 0.697f, 0.104f, 0.570f, 0.360f,
    -0.498f, 0.239f, 0.108f, -0.311f, -0.421f, -0.375f, -0.267f, -0.168f,
    -0.169f, -0.200f, -0.228f, -0.240f, -0.250f, -0.036f, 0.000f, 0.000f,
    0.000f, 0.000f, 0.000f, 0.000f};
static const float L93_A6[44] = {
    0.790f, 0.780f, 0.774f, 0.764f, 0.751f, 0.714f, 0.584f, 0.431f,
    0.305f, 0.339f, 0.705f, -0.113f, 0.753f, 0.742f, 0.697f, 0.051f,
    -0.146f, 0.266f, -0.090f, 0.081f, -0.324f, -0.067f, -0.761f, -0.777f,
    0.097f, -0.768f, -0.706f, -0.332f, -0.298f, -0.423f, -0.575f, -0.700f,
    -0.735f, -0.744f, -0.753f, -0.760f, -0.765f, 0.009f, 0.000f, 0.000f,
    0.000f, 0.000f, 0.000f, 0.000f};
static const float L93_F0H2O[35] = {
    22.235081f, 67.803963f, 119.995941f, 183.310089f, 321.225647f, 325.152924f, 336.222595f, 380.197357f,
    390.134521f, 437.346680f, 439.150818f, 443.018280f, 448.001068f, 470.888947f, 474.689117f, 488.491119f,
    503.568542f, 504.482697f, 547.676453f, 552.020935f, 556.935974f, 620.700806f, 645.866150f, 658.005310f,
    752.033203f, 841.053955f, 859.962341f, 899.306702f, 902.616150f, 906.207336f, 916.171570f, 923.118408f,
    970.315002f, 987.926758f, 1780.000000f};
static const float L93_B1[35] = {
    0.01130f, 0.00012f, 0.00008f, 0.24200f, 0.00483f, 0.14990f, 0.00011f, 1.15200f,
    0.00046f, 0.00650f, 0.09218f, 0.01976f, 1.03200f, 0.03297f, 0.12620f, 0.02520f,
    0.00390f, 0.00130f, 0.97010f, 1.47700f, 48.74000f, 0.50120f, 0.00713f, 0.03022f,
    23.96000f, 0.00140f, 0.01472f, 0.00605f, 0.00426f, 0.01876f, 0.83400f, 0.00869f,
    0.89720f, 13.21000f, 2230.00000f};
static const float L93_B2[35] = {
    2.143f, 8.735f, 8.356f, 0.668f, 6.181f, 1.540f, 9.829f, 1.048f,
    7.350f, 5.050f, 3.596f, 5.050f, 1.405f, 3.599f, 2.381f, 2.853f,
    6.733f, 6.733f, 0.114f, 0.114f, 0.159f, 2.200f, 8.580f, 7.820f,
    0.396f, 8.180f, 7.989f, 7.917f, 8.432f, 5.111f, 1.442f, 10.220f,
    1.920f, 0.258f, 0.952f};
static const float L93_B3[35] = {
    2.811f, 2.858f, 2.948f, 3.050f, 2.303f, 2.783f, 2.693f, 2.873f,
    2.152f, 1.845f, 2.100f, 1.860f, 2.632f, 2.152f, 2.355f, 2.602f,
    1.612f, 1.612f, 2.600f, 2.600f, 3.210f, 2.438f, 1.800f, 3.210f,
    3.060f, 1.590f, 3.060f, 2.985f, 2.865f, 2.408f, 2.670f, 2.900f,
    2.550f, 2.985f, 17.620f};
static const float L93_B4[35] = {
    4.80f, 4.93f, 4.78f, 5.30f, 4.69f, 4.85f, 4.74f, 5.38f,
    4.81f, 4.23f, 4.29f, 4.23f, 4.84f, 4.57f, 4.65f, 5.04f,
    3.98f, 4.01f, 4.50f, 4.50f, 4.11f, 4.68f, 4.00f, 4.14f,
    4.09f, 5.76f, 4.09f, 4.53f, 5.10f, 4.70f, 4.78f, 5.00f,
    4.94f, 4.55f, 30.50f};
static const float L93_B5[35] = {
    0.69f, 0.69f, 0.70f, 0.64f, 0.67f, 0.68f, 0.69f, 0.54f,
    0.63f, 0.60f, 0.63f, 0.60f, 0.66f, 0.66f, 0.65f, 0.69f,
    0.61f, 0.61f, 0.70f, 0.70f, 0.69f, 0.71f, 0.60f, 0.69f,
    0.68f, 0.33f, 0.68f, 0.68f, 0.70f, 0.70f, 0.70f, 0.70f,
    0.64f, 0.68f, 2.00f};
static const float L93_B6[35] = {
    1.00f, 0.82f, 0.79f, 0.85f, 0.54f, 0.74f, 0.61f, 0.89f,
    0.55f, 0.48f, 0.52f, 0.50f, 0.67f, 0.65f, 0.64f, 0.72f,
    0.43f, 0.45f, 1.00f, 1.00f, 1.00f, 0.68f, 0.50f, 1.00f,
    0.84f, 0.45f, 0.84f, 0.90f, 0.95f, 0.53f, 0.78f, 0.80f,
    0.67f, 0.90f, 5.00f};


// COMPLEX(4) division, Smith's method in single precision (gfortran
// -fcx-fortran-rules).
static void cdiv4(float ar, float ai, float br, float bi, float& qr, float& qi) {
  float tr, ti, ratio, div;
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
  qr = tr / div;
  qi = ti / div;
}

// ZF of src/mpm93.f90:269-270 and :300-301
static cplx l93_zf(double freq, double f0, double delta, double gamma) {
  float q1r, q1i, q2r, q2i;
  cdiv4(1.f, (float)(-delta), (float)(f0 - freq), (float)(-gamma), q1r, q1i);
  cdiv4(1.f, (float)delta, (float)(f0 + freq), (float)gamma, q2r, q2i);
  float dr = q1r - q2r, di = q1i - q2i;  // COMPLEX(4) difference
  double r = freq / f0;
  return cmk(r * (double)dr, r * (double)di);
}

// mpm93 (src/mpm93.f90:1-359, W = 0) called as src/get_gasabs.f90:78-86:
// Pbkpa = p / 1e3, Ekpa = e / 1e3, Tc = T - t_abs; result in Np/m.
double gas_l93(double freq, double press, double vap, double T) {
  const double t_abs = 273.15;
  double Pbkpa = press / 1.e3, Ekpa = vap / 1.e3, Tc = T - t_abs;
  double V = 300.0 / (Tc + t_abs);
  double Pb = 10.0 * Pbkpa, E = 10.0 * Ekpa;
  double P = Pb - E;
  if (P < 0) {
    P = 0.0;
    Pb = E;
  }
  cplx ZN = cmk(0.0, 0.0);
  for (int i = 0; i < 44; i++) {
    double S = (double)L93_A1[i] * P * p3(V) * std::exp((double)L93_A2[i] * (1.0 - V)) * 1.e-6;
    double GAMMA = (double)L93_A3[i] * (P * std::pow(V, 0.8 - (double)L93_A4[i]) + 1.1 * E * V) * 1.e-3;
    GAMMA = std::pow(p2(GAMMA) + p2(25.0 * 0.6e-4), 0.5);
    double DELTA = ((double)L93_A5[i] + (double)L93_A6[i] * V) * (P + E) * std::pow(V, (double)0.8f) * 1.e-3;
    cplx ZF = l93_zf(freq, L93_F0O2[i], DELTA, GAMMA);
    ZN = cadd(ZN, cscale(ZF, S));
  }
  double AT1 = 0.182 * freq * ZN.im;
  if (AT1 < 0.) AT1 = 0.0;
  double So = 6.14e-5 * P * p2(V);
  double GAMMAo = 0.56e-3 * (P + E) * std::pow(V, (double)0.8f);
  cplx ZFo = cdiv(cmk(freq, 0.0), cmplx4(freq, GAMMAo));
  ZFo = cmk(-ZFo.re, -ZFo.im);
  double Sn = 1.40e-12 * p2(P) * std::pow(V, 3.5);
  cplx ZFn = cmplx4(0., freq / (1.93e-5 * std::pow(freq, 1.5) + 1.0));
  ZN = cadd(cscale(ZFo, So), cscale(ZFn, Sn));
  double AT2 = 0.182 * freq * ZN.im;
  ZN = cmk(0.0, 0.0);
  for (int i = 0; i < 35; i++) {
    double S = (double)L93_B1[i] * E * std::pow(V, 3.5) * std::exp((double)L93_B2[i] * (1.0 - V));
    double GAMH = (double)L93_B3[i] * (P * std::pow(V, (double)L93_B5[i]) +
                                       (double)L93_B4[i] * E * std::pow(V, (double)L93_B6[i])) * 1.e-3;
    double GAMD2 = 1.e-12 / V * p2((double)1.46f * (double)L93_F0H2O[i]);
    GAMH = 0.535 * GAMH + std::pow(0.217 * p2(GAMH) + GAMD2, 0.5);
    cplx ZF = l93_zf(freq, L93_F0H2O[i], 0.0, GAMH);
    ZN = cadd(ZN, cscale(ZF, S));
  }
  double AT3 = 0.182 * freq * ZN.im;
  double AT4 = 0.0;  // cloud term, W = 0
  return 0.23026 * (AT1 + AT2 + AT3 + AT4) / 1.e3;
}

// ---------------------------------------------------------------- PSD
// src/conversions.f90:5-24
double q2abs(double spec, double t, double p, double qv, double qall) {
  return spec * p / (R_D * (1.0 + (R_V / R_D - 1.0) * qv - qall) * t);
}

struct Bins {
  int nbin = 0;
  std::vector<double> d_ds, delta_d, n_ds, dens, diam, mass;
};

struct PSDIn {
  orc_species s;
  double q_h, n_tot, r_eff, layer_t, freq;
};

// src/make_mass_size.f90
int make_mass_size(const orc_species& s, double& a_ms, double& b_ms) {
  a_ms = s.a_ms;
  b_ms = s.b_ms;
  const double rho = s.rho_ms, asr = s.as_ratio;
  const int li = s.liq_ice;
  if (b_ms > 3.5) return 2;
  if (a_ms == 0.0) return 2;
  if (rho == 0.0) return 2;
  if (asr == 0.0) return 2;
  if (li == -1 && rho > 917.0) return 2;
  if (li == 1 && (a_ms > 0.0 || b_ms > 0.0 || rho > 0.0 || (asr != 1.0 && asr > 0.0))) {
    // warning only
  } else if (li == -1 && a_ms < 0.0 && b_ms < 0.0 && rho < 0.0) {
    return 2;
  } else if ((a_ms < 0.0 && b_ms >= 0.0) || (a_ms > 0.0 && b_ms < 0.0)) {
    return 2;
  }
  if (li == 1) {
    b_ms = 3.0;
    a_ms = PI / 6.0 * RHO_WATER;
    return 0;
  }
  if (a_ms > 0.0 && b_ms >= 0 && li == -1) return 0;
  if (li == -1 && (asr < 0.0 || asr == 1.0)) {
    b_ms = 3.0;
    a_ms = PI / 6.0 * rho;
    return 0;
  } else if (li == -1 && asr > 1.0) {
    b_ms = 3.0;
    a_ms = PI / 6.0 * rho * std::pow(1.0 / asr, 2.0);
    return 0;
  } else if (li == -1 && asr > 0.0 && asr < 1.0) {
    b_ms = 3.0;
    a_ms = PI / 6.0 * rho * asr;
    return 0;
  }
  return 2;
}

struct DistPar {
  double n_0 = -99, lambda = -99, gam = NaN, mu = NaN, n_t = -99, sig = -99, d_ln = NaN, d_mono = -99;
};

// src/make_dist_param.f90 (exp, exp_field_t, exp_ryan, mgamma, mono, logn)
int make_dist_params(const PSDIn& in, double a_ms, double b_ms, DistPar& dp) {
  const orc_species& s = in.s;
  const int mi = s.moment_in;
  const double q_h = in.q_h, n_tot = in.n_tot, r_eff = in.r_eff;
  const double p_1 = s.p_1, p_2 = s.p_2, p_3 = s.p_3, p_4 = s.p_4, d_1 = s.d_1;
  if (mi == 3 && q_h <= 0.) return 2;
  if (mi == 1 && n_tot <= 0.) return 2;
  if (mi == 2 && r_eff <= 0.) return 2;
  if (mi == 13 && (q_h <= 0. || n_tot <= 0.)) return 2;
  if (mi == 23 && (q_h <= 0. || r_eff <= 0.)) return 2;
  if (mi == 12 && (n_tot <= 0. || r_eff <= 0.)) return 2;
  const int dist = s.dist;
  if (dist == D_MONO) {
    dp.lambda = 0; dp.mu = 0; dp.gam = 0;
    if (d_1 != -99. && p_1 == -99.) {
      dp.d_mono = d_1;
      if (mi == 3) dp.n_0 = q_h / (DELTA_D_MONO * a_ms * std::pow(d_1, b_ms));
      if (mi == 1) dp.n_0 = n_tot / DELTA_D_MONO;
    }
    if (p_1 != -99. && d_1 == -99.) {
      dp.n_0 = p_1 / DELTA_D_MONO;
      if (mi == 3) dp.d_mono = std::pow(q_h / (p_1 * a_ms), 1.0 / b_ms);
      if (mi == 2) dp.d_mono = r_eff * 2.0;
    }
    if (mi == 23) {
      dp.d_mono = r_eff * 2.0;
      dp.n_0 = q_h / (DELTA_D_MONO * a_ms * std::pow(dp.d_mono, b_ms));
    }
    if (dp.n_0 <= 0.0 || dp.d_mono <= 0.0) return 2;
    return 0;
  }
  if (dist == D_EXP || dist == D_EXP_FIELD_T || dist == D_EXP_RYAN) {
    dp.gam = 1.0;
    dp.mu = 0.0;
    const double gb = std::tgamma(b_ms + 1.0);
    if (dist == D_EXP) {
      if (p_1 != -99. && p_2 != -99. && mi == 0) { dp.lambda = p_1; dp.n_0 = p_2; }
      if (p_1 != -99. && p_2 != -99. && mi == 3) {
        dp.lambda = std::pow(p_1 * a_ms * gb / q_h, 1.0 / (b_ms + 1 - p_2));
        dp.n_0 = p_1 * std::pow(dp.lambda, p_2);
      }
      if (p_1 != -99. && p_2 == -99. && p_3 == -99.) {
        if (mi == 3) dp.lambda = std::pow(p_1 * a_ms * gb / q_h, 1.0 / b_ms);
        if (mi == 2) dp.lambda = 3.0 / r_eff;
        dp.n_0 = p_1 * dp.lambda;
      }
      if (p_1 == -99. && p_2 != -99. && p_3 == -99.) {
        dp.lambda = 3.0 / p_2;
        if (mi == 3) dp.n_0 = (q_h * std::pow(dp.lambda, b_ms + 1.0)) / (a_ms * gb);
        if (mi == 1) dp.n_0 = n_tot * dp.lambda;
      }
      if (p_1 == -99. && p_2 == -99. && p_3 != -99.) {
        dp.n_0 = p_3;
        if (mi == 3) dp.lambda = std::pow(dp.n_0 * a_ms * gb / q_h, 1.0 / (b_ms + 1.0));
        if (mi == 1) dp.lambda = dp.n_0 / n_tot;
        if (mi == 2) dp.lambda = 3.0 / r_eff;
      }
      if (p_1 == -99. && p_2 == -99.) {
        if (mi == 13) {
          dp.lambda = std::pow(n_tot * a_ms * gb / q_h, 1.0 / b_ms);
          dp.n_0 = n_tot * dp.lambda;
        }
        if (mi == 23) {
          dp.lambda = 3.0 / r_eff;
          dp.n_0 = (q_h * std::pow(dp.lambda, b_ms + 1)) / (a_ms * gb);
        }
        if (mi == 12) {
          dp.lambda = 3.0 / r_eff;
          dp.n_0 = n_tot * dp.lambda;
        }
      }
    }
    if (dist == D_EXP_RYAN) {
      dp.lambda = 1220.0 * std::pow(10.0, -0.0245 * (273.15 - in.layer_t));
      if (mi == 3) dp.n_0 = (q_h * std::pow(dp.lambda, b_ms + 1)) / (a_ms * gb);
      if (mi == 1) dp.n_0 = n_tot * dp.lambda;
    }
    if (dist == D_EXP_FIELD_T) {
      dp.n_0 = 7.628e6 * std::exp(0.107 * (273.15 - in.layer_t));
      if (mi == 3) dp.lambda = std::pow(a_ms * dp.n_0 * gb / q_h, 1.0 / (b_ms + 1.0));
      if (mi == 2) dp.lambda = 3.0 / r_eff;
    }
    if (dp.gam != 1.0 || dp.mu != 0.0 || dp.n_0 <= 0.0 || dp.lambda <= 0.0) return 2;
    return 0;
  }
  if (dist == D_LOGN) {
    if (p_1 != -99. && p_3 != -99.) {
      dp.n_t = p_1;
      dp.sig = p_3;
      if (mi == 3) dp.d_ln = (1.0 / b_ms) * (std::log(q_h / (a_ms * dp.n_t)) - (0.5 * std::pow(b_ms * dp.sig, 2.0)));
      if (mi == 2) dp.d_ln = std::log(2.0 * r_eff) - 2.5 * std::pow(dp.sig, 2.0);
    }
    if (p_1 != -99. && p_2 != -99. && p_3 == -99. && mi == 3) {
      dp.n_t = p_1;
      double w1 = q_h / (a_ms * dp.n_t * std::pow(2.0 * p_2, 2.0));
      double w2 = 2.0 / (b_ms * (b_ms - 5.0));
      dp.sig = std::sqrt(std::log(w1) * w2);
      dp.d_ln = std::log(2.0 * p_2) - 2.5 * std::pow(dp.sig, 2.0);
    }
    if (p_1 == -99. && p_2 != -99. && p_3 != -99.) {
      dp.sig = p_3;
      dp.d_ln = std::log(2.0 * p_2) - 2.5 * std::pow(dp.sig, 2.0);
      if (mi == 3) dp.n_t = q_h / a_ms * std::exp(-1.0 * ((b_ms * dp.d_ln) + (0.5 * std::pow(b_ms * dp.sig, 2.0))));
      if (mi == 1) dp.n_t = n_tot;
    }
    if (dp.n_t <= 0.0 || std::isnan(dp.d_ln) || dp.sig <= 0.0) return 2;
    return 0;
  }
  if (dist == D_MGAMMA) {
    if (p_3 == -99. || p_4 == -99.) return 2;
    double mu = p_3, gam = p_4;
    dp.mu = mu;
    dp.gam = gam;
    if (p_1 != -99. && p_2 == -99.) {
      if (mi == 3) {
        double w2 = std::tgamma((mu + b_ms + 1.0) / gam);
        double w3 = std::tgamma((mu + 1.0) / gam);
        dp.lambda = std::pow(a_ms / q_h * p_1 * w2 / w3, gam / b_ms);
        dp.n_0 = gam * p_1 / w3 * std::pow(dp.lambda, (mu + 1.0) / gam);
      }
      if (mi == 2) {
        double w1 = std::tgamma((mu + 4.0) / gam);
        double w2 = std::tgamma((mu + 3.0) / gam) * r_eff * 2.0;
        dp.lambda = std::pow(w1 / w2, gam);
        w1 = (mu + 1.0) / gam;
        dp.n_0 = p_1 * gam * std::pow(dp.lambda, w1) / std::tgamma(w1);
      }
    }
    if (p_1 == -99. && p_2 != -99.) {
      if (mi == 3) {
        double w1 = std::tgamma((mu + 4.0) / gam);
        double w2 = std::tgamma((mu + 3.0) / gam) * p_2 * 2.0;
        dp.lambda = std::pow(w1 / w2, gam);
        w1 = q_h * gam / a_ms;
        w2 = (mu + b_ms + 1.0) / gam;
        dp.n_0 = w1 * std::pow(dp.lambda, w2) / std::tgamma(w2);
      }
      if (mi == 1) {
        double w1 = std::tgamma((mu + 4.0) / gam);
        double w2 = std::tgamma((mu + 3.0) / gam) * p_2 * 2.0;
        dp.lambda = std::pow(w1 / w2, gam);
        w1 = (mu + 1.0) / gam;
        dp.n_0 = n_tot * gam * std::pow(dp.lambda, w1) / std::tgamma(w1);
      }
    }
    if (p_1 == -99. && p_2 == -99.) {
      if (mi == 13) {
        double w2 = std::tgamma((mu + b_ms + 1.0) / gam);
        double w3 = std::tgamma((mu + 1.0) / gam);
        dp.lambda = std::pow(a_ms / q_h * n_tot * w2 / w3, gam / b_ms);
        dp.n_0 = gam * n_tot / w3 * std::pow(dp.lambda, (mu + 1.0) / gam);
      }
      if (mi == 23) {
        double w1 = std::tgamma((mu + 4.0) / gam);
        double w2 = std::tgamma((mu + 3.0) / gam) * r_eff * 2.0;
        dp.lambda = std::pow(w1 / w2, gam);
        w1 = q_h * gam / a_ms;
        w2 = (mu + b_ms + 1.0) / gam;
        dp.n_0 = w1 * std::pow(dp.lambda, w2) / std::tgamma(w2);
      }
      if (mi == 12) {
        double w1 = std::tgamma((mu + 4.0) / gam);
        double w2 = std::tgamma((mu + 3.0) / gam) * r_eff * 2.0;
        dp.lambda = std::pow(w1 / w2, gam);
        w1 = (mu + 1.0) / gam;
        dp.n_0 = n_tot * gam * std::pow(dp.lambda, w1) / std::tgamma(w1);
      }
    }
    if (dp.lambda <= 0.0 || dp.n_0 <= 0.0 || std::isnan(mu) || std::isnan(gam)) return 2;
    return 0;
  }
  return 2;
}

// src/make_dist.f90:2-290 (gamma family, logn and mono)
int make_dist(const orc_species& s, int nbin, const DistPar& dp, double a_ms, double b_ms, double q_h,
              bool adaptive, bool conserve, std::vector<double>& d_bound, std::vector<double>& f_ds) {
  const double thres_n = 0.1;
  const double min_d = (double)(float)1.0e-7;  // `real :: min_d` (REAL(4))
  const double max_d = (double)(float)2.0e-2;  // `real :: max_d` (REAL(4))
  const double big = F(1.e30f);
  d_bound.assign(nbin + 1, 0.0);
  f_ds.assign(nbin + 1, 0.0);
  auto fdist = [&](double d) -> double {
    if (s.dist == D_LOGN)
      return dp.n_t / (d * dp.sig * std::sqrt(2.0 * PI)) *
             std::exp(-(p2(std::log(d) - dp.d_ln)) / (2.0 * p2(dp.sig)));
    return dp.n_0 * std::pow(d, dp.mu) * std::exp(-dp.lambda * std::pow(d, dp.gam));
  };
  bool skip = false;
  if (s.dist == D_MONO) {
    d_bound[0] = dp.d_mono - DELTA_D_MONO * .5;
    d_bound[1] = dp.d_mono;
    d_bound[2] = dp.d_mono + DELTA_D_MONO * .5;
    for (int i = 0; i < nbin + 1; i++) f_ds[i] = fdist(d_bound[i]);
    skip = true;
  }
  double d_1_new = 0, d_2_new = 0;
  for (int ibig = 1; ibig <= 2; ibig++) {
    if (skip) break;
    double d1w = 0, d2w = 0;
    int nw = 0;
    if (ibig == 1 && !adaptive) { d1w = s.d_1 + 1.e-8; d2w = s.d_2; nw = nbin; skip = true; }
    if (ibig == 1 && adaptive) { d1w = min_d; d2w = max_d; nw = 500; }
    if (ibig == 2) { d1w = d_1_new; d2w = d_2_new; nw = nbin; skip = true; }
    int nlin = (int)(nw / 2.0), nlog = (int)(nw / 2.0);
    if (nlin + nlog == nw) nlin = nlin - 1;
    std::vector<double> lin(nlin + 1), lg(nlog + 1), dw(nw + 1), fw(nw + 1);
    double w1 = (d2w - d1w) / (nlin + 1);
    for (int i = 1; i <= nlin + 1; i++) lin[i - 1] = d1w + w1 * i;
    w1 = (std::log(d2w) - std::log(d1w)) / (nlog + 1);
    for (int i = 1; i <= nlog + 1; i++) lg[i - 1] = std::exp(w1 * (i - 1) + std::log(d1w));
    // merge (minval/minloc with sentinel 1e30): both inputs are ascending
    for (int i = 0; i < nw + 1; i++) {
      int il = (int)(std::min_element(lin.begin(), lin.end()) - lin.begin());
      int ig = (int)(std::min_element(lg.begin(), lg.end()) - lg.begin());
      if (lg[ig] <= lin[il]) { dw[i] = lg[ig]; lg[ig] = big; }
      else { dw[i] = lin[il]; lin[il] = big; }
    }
    for (int i = 0; i < nw + 1; i++) fw[i] = fdist(dw[i]);
    if (adaptive && ibig == 1) {
      d_1_new = -1.0;
      d_2_new = -1.0;
      for (int i = nw; i >= 1; i--) {  // search_loop1 (1-based i)
        d_2_new = dw[i];
        if (fw[nw] >= thres_n) { d_2_new = dw[nw]; break; }
        if (fw[i - 1] >= thres_n && fw[i] < thres_n) break;
      }
      for (int i = 1; i <= nw; i++) {  // search_loop2
        d_1_new = dw[i - 1];
        if (fw[i - 1] >= fw[i]) { d_1_new = min_d; break; }
        if ((fw[i - 1] < thres_n && fw[i] >= thres_n) || fw[i - 1] >= fw[i]) break;
      }
      if (d_1_new < -1.e-30 || d_2_new < -1.e-30 || d_1_new > d_2_new) return 2;
    }
    if (skip) { f_ds = fw; d_bound = dw; }
  }
  (void)a_ms; (void)b_ms; (void)q_h; (void)conserve;
  return 0;
}

// src/drop_size_dist.f90:107-218 run_drop_size_dist + make_dist tail + make_soft_spheroid
int run_psd(const orc_settings& st, const PSDIn& in, Bins& out) {
  const orc_species& s = in.s;
  double a_ms, b_ms;
  if (make_mass_size(s, a_ms, b_ms) == 2) return 2;
  DistPar dp;
  if (make_dist_params(in, a_ms, b_ms, dp) == 2) return 2;
  int nbin = s.nbin;
  if (s.dist == D_MONO) nbin = 2;
  std::vector<double> d_bound, f_ds;
  if (make_dist(s, nbin, dp, a_ms, b_ms, in.q_h, st.hydro_adaptive_grid != 0, st.conserve_mass_rescale_dsd != 0,
                d_bound, f_ds) == 2)
    return 2;
  out.nbin = nbin;
  out.d_ds.assign(nbin, 0);
  out.delta_d.assign(nbin, 0);
  out.n_ds.assign(nbin, 0);
  for (int i = 0; i < nbin; i++) {
    out.d_ds[i] = (d_bound[i] + d_bound[i + 1]) * .5;
    out.delta_d[i] = d_bound[i + 1] - d_bound[i];
  }
  double mass_tot = 0.0;
  for (int i = 0; i < nbin; i++)
    mass_tot = mass_tot + a_ms * (f_ds[i] + f_ds[i + 1]) / 2.0 * out.delta_d[i] * std::pow(out.d_ds[i], b_ms);
  const int mi = s.moment_in;
  if (st.conserve_mass_rescale_dsd && (mi == 3 || mi == 23 || mi == 13))
    for (int i = 0; i < nbin + 1; i++) f_ds[i] = f_ds[i] * in.q_h / mass_tot;
  for (int i = 0; i < nbin; i++) out.n_ds[i] = (f_ds[i] + f_ds[i + 1]) / 2.0 * out.delta_d[i];
  double n_tot = 0.0;
  for (int i = 0; i < nbin; i++) n_tot += out.n_ds[i];
  for (int i = 0; i < nbin; i++)
    if (out.n_ds[i] < n_tot / nbin * 1e-60) out.n_ds[i] = 0.0;
  out.mass.assign(nbin, 0);
  for (int i = 0; i < nbin; i++) out.mass[i] = a_ms * std::pow(out.d_ds[i], b_ms);
  out.dens.assign(nbin, 0);
  out.diam.assign(nbin, 0);
  if (s.liq_ice == 1) {
    for (int i = 0; i < nbin; i++) { out.dens[i] = RHO_WATER; out.diam[i] = out.d_ds[i]; }
    return 0;
  }
  // src/make_soft_spheroid.f90
  const double rho_ms = s.rho_ms, asr = s.as_ratio, mind = st.hydro_softsphere_min_density;
  std::vector<double> mass = out.mass, rho(nbin, 0.0), dd(nbin, 0.0);
  if (rho_ms > 0.) {
    for (int i = 0; i < nbin; i++) rho[i] = rho_ms;
    if (asr <= 1.)
      for (int i = 0; i < nbin; i++) {
        if (asr < 0.) dd[i] = std::pow((6.0 * mass[i]) / (PI * rho_ms), 1.0 / 3.0);
        if (asr > 0.) dd[i] = std::pow((6.0 * mass[i]) / (PI * rho_ms * asr), 1.0 / 3.0);
      }
    if (asr > 1.)
      for (int i = 0; i < nbin; i++) dd[i] = std::pow((6.0 * mass[i] * std::pow(asr, 2.0)) / (PI * rho_ms), 1.0 / 3.0);
  } else if (rho_ms < 0.) {
    dd = out.d_ds;
    if (asr <= 1.)
      for (int i = 0; i < nbin; i++) {
        if (asr == -99.) rho[i] = (6.0 * mass[i]) / (PI * std::pow(out.d_ds[i], 3.0));
        if (asr == -10.) rho[i] = 917.0;
        if (asr == -20.) rho[i] = 0.863 * in.freq + 115.0;
        if (asr == -30.) rho[i] = 0.815 * in.freq + 11.2;
        if (asr > 0.) rho[i] = (6.0 * mass[i]) / (PI * std::pow(out.d_ds[i], 3.0) * asr);
        if (rho[i] < mind) rho[i] = mind;
        if (asr == -10. || asr == -20. || asr == -30.) dd[i] = std::pow((6.0 * mass[i]) / (PI * rho[i]), 1.0 / 3.0);
      }
    if (asr > 1.)
      for (int i = 0; i < nbin; i++) rho[i] = (6.0 * mass[i] * std::pow(asr, 2.0)) / (PI * std::pow(out.d_ds[i], 3.0));
  } else {
    return 2;
  }
  if (st.hydro_limit_density_area)
    for (int i = 0; i < nbin; i++) {
      if (rho[i] > RHO_ICE) rho[i] = RHO_ICE;
      else if (rho[i] < mind) rho[i] = mind;
    }
  for (int i = 0; i < nbin; i++)
    if (rho[i] <= 0. || dd[i] <= 0.) return 2;
  out.dens = rho;
  out.diam = dd;
  return 0;
}

// ---------------------------------------------------------------- refractive index
// src/eps_water.f90:653-757 eps_water_tkc (T in degC, f in GHz)
cplx eps_water_tkc(double T, double f) {
  const double a_1 = 8.169396e+01, b_1 = 4.410555e-03, c_1 = 1.208992e-13, d_1 = 6.768869e+02;
  const double a_2 = 1.597733e+00, b_2 = 1.060228e-02, c_2 = 9.982113e-15, d_2 = 5.720517e+02;
  const double t_c = 1.351758e+02;
  double frq = f * 1e9;
  double eps_s = 87.9144 - 0.404399 * T + 9.58726e-4 * (T * T) - 1.32802e-6 * std::pow(T, 3.0);
  double delta_1 = a_1 * std::exp(-b_1 * T);
  double tau_1 = c_1 * std::exp(d_1 / (T + t_c));
  double delta_2 = a_2 * std::exp(-b_2 * T);
  double tau_2 = c_2 * std::exp(d_2 / (T + t_c));
  double w = 2.0 * PI * frq;
  double x1 = w * tau_1, x2 = w * tau_2;
  double t1 = ((tau_1 * tau_1) * delta_1) / (1.0 + x1 * x1);
  double t2 = ((tau_2 * tau_2) * delta_2) / (1.0 + x2 * x2);
  double eps1 = eps_s - (w * w) * (t1 + t2);
  t1 = (tau_1 * delta_1) / (1.0 + x1 * x1);
  t2 = (tau_2 * delta_2) / (1.0 + x2 * x2);
  double eps2 = w * (t1 + t2);
  return cmplx4(eps1, eps2);  // CMPLX without KIND (eps_water.f90:749)
}

// src/eps_ice.f90 + src/ref_ice.f90
void ref_ice(double T, double f, double& refre, double& refim) {
  double eps_real;
  if (T >= 240.0) eps_real = 3.1884 + 9.1e-4 * (T - 273.0);
  else eps_real = 3.1884 + 9.1e-4 * (240.0 - 273.0);
  double mit = (300.0 / T) - 1.0;
  double alpha = (0.00504 + 0.0062 * mit) * std::exp(-22.1 * mit);
  double e = std::exp(335.0 / T);
  double beta_m = (0.0207 / T) * e / ((e - 1.0) * (e - 1.0));
  beta_m = beta_m + 1.16e-11 * (f * f);
  double delta_beta = std::exp(-9.963 + 0.0372 * (T - 273.16));
  double beta = beta_m + delta_beta;
  double eps_imag = (alpha / f) + beta * f;
  cplx r = csqrt_(cmk(eps_real, eps_imag));
  refre = r.re;
  refim = r.im;
}

// src/eps_mix.f90 with eps0 = (1,0): Sihvola-type mixing applied to m
cplx eps_mix_m(cplx eps1, double mix_de) {
  const double v = 0.85;
  const double f = mix_de / 917.0;
  const double re1 = eps1.re, e0 = 1.0;
  double b = re1 + 2.0 * e0 - 2.0 * v * e0 - f * (re1 - e0) * (1 + v);
  double a = e0 * (re1 + (2.0 - v) * e0 + f * (2.0 - v) * (re1 - e0));
  double em_real = (std::sqrt(b * b + 4.0 * v * a) - b) / (2.0 * v);
  double em_imag = eps1.im * (-1.0 * (em_real - e0) + f * (em_real + 2.0 * e0 + v * (em_real - e0))) /
                   ((re1 + 2.0 * e0 + 2.0 * v * (em_real - e0)) - f * (1.0 + v) * (re1 - e0));
  return cmplx4(em_real, em_imag);  // CMPLX without KIND (eps_mix.f90:44)
}

// ---------------------------------------------------------------- Mie
// src/mie_scat_utilities.f90:8-75 miecalc
int miecalc(int& nterms, double x, cplx mn, std::vector<cplx>& a, std::vector<cplx>& b) {
  int nstop = (int)(x + 4.0 * std::pow(x, F(0.3334f)) + 2);
  if (nterms <= 0) nterms = nstop;
  if (nterms > 10000) return 2;
  cplx m = cconj(mn);
  cplx y = cscale(m, x);
  int nn = nterms + 15;
  std::vector<cplx> d(nn + 1);
  d[nn] = cmk(0, 0);
  for (int n = nn; n >= 2; n--) {
    cplx ny = cdiv(cmk((double)n, 0), y);
    d[n - 1] = csub(ny, cdiv(cmk(1.0, 0), cadd(d[n], ny)));
  }
  double psim = std::cos(x), psin = std::sin(x), chim = -std::sin(x), chin = std::cos(x);
  a.assign(nterms + 1, cmk(0, 0));
  b.assign(nterms + 1, cmk(0, 0));
  for (int n = 1; n <= nterms; n++) {
    double tmp = psin;
    psin = (2 * n - 1) / x * psin - psim;
    psim = tmp;
    tmp = chin;
    chin = (2 * n - 1) / x * chin - chim;
    chim = tmp;
    cplx xin = cmplx4(psin, -chin);
    cplx xim = cmplx4(psim, -chim);
    cplx ctmp = cdiv(d[n], m);
    ctmp.re = ctmp.re + n / x;
    cplx num = cmk(ctmp.re * psin - psim, ctmp.im * psin);
    cplx den = csub(cmul(ctmp, xin), xim);
    a[n] = cdiv(num, den);
    ctmp = cmul(m, d[n]);
    ctmp.re = ctmp.re + n / x;
    num = cmk(ctmp.re * psin - psim, ctmp.im * psin);
    den = csub(cmul(ctmp, xin), xim);
    b[n] = cdiv(num, den);
  }
  return 0;
}

// src/mie_scat_utilities.f90:77-116 miecross
void miecross(int nterms, double x, const std::vector<cplx>& a, const std::vector<cplx>& b, double& qext,
              double& qscat, double& qback) {
  double sum1 = 0, sum2 = 0;
  cplx sum3 = cmk(0, 0);
  for (int n = 1; n <= nterms; n++) {
    sum1 = sum1 + (2 * n + 1) * (a[n].re + b[n].re);
    sum2 = sum2 + (2 * n + 1) * ((a[n].re * a[n].re - a[n].im * (-a[n].im)) + (b[n].re * b[n].re - b[n].im * (-b[n].im)));
    double fac = (double)((float)(2 * n + 1) * ((n & 1) ? -1.0f : 1.0f));  // REAL(4) product
    sum3 = cadd(sum3, cscale(csub(a[n], b[n]), fac));
  }
  qext = 2.0 / (x * x) * sum1;
  qscat = 2.0 / (x * x) * sum2;
  cplx t = cscale(sum3, 1.0 / (x * x));
  qback = t.re * sum3.re - t.im * (-sum3.im);
}

// src/mie_scat_utilities.f90:119-160 mieangle
void mieangle(int nterms, const std::vector<cplx>& a, const std::vector<cplx>& b, double mu, double& p1,
              double& p2_, double& p3_, double& p4) {
  cplx s1 = cmk(0, 0), s2 = cmk(0, 0);
  double pin = 1.0, pim = 0.0;
  for (int n = 1; n <= nterms; n++) {
    double taun = n * mu * pin - (n + 1) * pim;
    double c = (double)((float)(2 * n + 1) / (float)(n * (n + 1)));  // REAL(4) division
    cplx t1 = cadd(cscale(a[n], pin), cscale(b[n], taun));
    cplx t2 = cadd(cscale(b[n], pin), cscale(a[n], taun));
    s1 = cadd(s1, cscale(t1, c));
    s2 = cadd(s2, cscale(t2, c));
    double tmp = pin;
    pin = ((2 * n + 1) * mu * pin - (n + 1) * pim) / n;
    pim = tmp;
  }
  double as1 = cabs_(s1), as2 = cabs_(s2);
  p1 = 0.5 * (as2 * as2 + as1 * as1);
  p2_ = 0.5 * (as2 * as2 - as1 * as1);
  p3_ = s2.re * s1.re - (-s2.im) * s1.im;
  p4 = s1.re * s2.im + (-s1.im) * s2.re;
}

// src/scat_utilities.f90:1-44 gausquad
void gausquad(int n, std::vector<double>& xa, std::vector<double>& wt) {
  xa.assign(n, 0);
  wt.assign(n, 0);
  int k = (n + 1) / 2;
  for (int j = 1; j <= k; j++) {
    double x = std::cos(PI * (j - 0.25) / (n + 0.5));
    int i = 0;
    double pl, pl1, pl2, dpl, xp;
    do {
      pl1 = 1;
      pl = x;
      for (int l = 2; l <= n; l++) {
        pl2 = pl1;
        pl1 = pl;
        pl = ((2 * l - 1) * x * pl1 - (l - 1) * pl2) / l;
      }
      dpl = n * (x * pl - pl1) / (x * x - 1);
      xp = x;
      x = xp - pl / dpl;
      i = i + 1;
    } while (std::fabs(x - xp) > 3.0e-13 && i < 10);
    xa[j - 1] = -x;
    xa[n - j] = x;
    wt[j - 1] = 2.0 / ((1.0 - x * x) * dpl * dpl);
    wt[n - j] = wt[j - 1];
  }
}

struct MieOut {
  double kext = 0, salb = 0, back = 0;
  int nlegen = 0;
  double legen[4][MAXNLEG];
  std::vector<double> back_spec;  // per bin, m2/m4 (0 where no particles)
};

// src/mie_spheres.f90:14-345 calc_mie_spheres
int calc_mie_spheres(const orc_settings& st, double freq_hz, int liq_ice, const Bins& bn,
                     const std::vector<double>& ndens, double refre, double refim, MieOut& o) {
  std::memset(o.legen, 0, sizeof(o.legen));
  o.kext = o.salb = o.back = 0;
  o.nlegen = 0;
  const int nb = bn.nbin;
  o.back_spec.assign(nb, 0.0);
  const double wavelength = C_LIGHT / freq_hz;
  cplx msphere;
  cplx m_ice = cmk(refre, -refim);
  if (liq_ice == -1 && bn.dens[0] != 917.0) msphere = eps_mix_m(m_ice, bn.dens[nb - 1]);
  else msphere = cmk(refre, -refim);
  double x = PI * bn.diam[nb - 1] / wavelength;
  int nterms = 0;
  std::vector<cplx> a, b;
  if (miecalc(nterms, x, msphere, a, b)) return 2;
  int nlegen = 2 * nterms;
  nlegen = std::min(MAXNLEG - 1, nlegen);
  int nquad = (nlegen + 2 * nterms + 2) / 2;
  if (nquad > 5000) return 2;
  std::vector<double> mu, wts;
  gausquad(nquad, mu, wts);
  double sumqe = 0, sumqs = 0, sumqback = 0;
  std::vector<double> sump[4];
  for (int k = 0; k < 4; k++) sump[k].assign(nquad, 0.0);
  for (int ir = 0; ir < nb; ir++) {
    if (ndens[ir] <= 0) continue;
    double ndens_eff = ndens[ir], del_d_eff = bn.delta_d[ir];
    if (liq_ice == -1 && bn.dens[ir] != 917.0) msphere = eps_mix_m(m_ice, bn.dens[ir]);
    else msphere = cmk(refre, -refim);
    int nmie = 0;
    x = PI * bn.diam[ir] / wavelength;
    if (miecalc(nmie, x, msphere, a, b)) return 2;
    double qext, qscat, qback;
    miecross(nmie, x, a, b, qext, qscat, qback);
    double r2 = (bn.diam[ir] / 2.0) * (bn.diam[ir] / 2.0);
    qext = qext * r2 * PI;
    qscat = qscat * r2 * PI;
    qback = qback * r2 * PI;
    qext = qext * ndens_eff;
    qscat = qscat * ndens_eff;
    qback = qback * ndens_eff;
    sumqe = sumqe + (qext * del_d_eff);
    sumqs = sumqs + (qscat * del_d_eff);
    sumqback = sumqback + (qback * del_d_eff);
    o.back_spec[ir] = qback;
    nmie = std::min(nmie, nterms);
    for (int i = 0; i < nquad; i++) {
      double pp[4];
      mieangle(nmie, a, b, mu[i], pp[0], pp[1], pp[2], pp[3]);
      for (int k = 0; k < 4; k++) sump[k][i] = sump[k][i] + pp[k] * ndens_eff * del_d_eff;
    }
  }
  double extinction = st.lhyd_absorption ? sumqe : sumqe - sumqs;
  double scatter = sumqs;
  o.back = sumqback;
  o.kext = extinction;
  o.salb = scatter / extinction;
  double tmp = (wavelength * wavelength / (PI * scatter));
  for (int i = 0; i < nquad; i++)
    for (int k = 0; k < 4; k++) sump[k][i] = tmp * sump[k][i] * wts[i];
  std::vector<double> coef[4];
  for (int k = 0; k < 4; k++) coef[k].assign(nlegen + 1, 0.0);
  for (int i = 0; i < nquad; i++) {
    double pl1 = 1.0, pl = 1.0, pl2 = 0.0;
    for (int l = 0; l <= nlegen; l++) {
      if (l > 0) pl = (2 * l - 1) * mu[i] * pl1 / l - (l - 1) * pl2 / l;
      for (int k = 0; k < 4; k++) coef[k][l] = coef[k][l] + sump[k][i] * pl;
      pl2 = pl1;
      pl1 = pl;
    }
  }
  int nleg = nlegen;
  const double thr = F(1.0e-7f);
  for (int l = 0; l <= nleg; l++) {
    double fac = (double)((float)(2 * l + 1) / 2.0f);  // REAL(4) division, exact
    for (int k = 0; k < 4; k++) o.legen[k][l] = fac * coef[k][l];
    if (o.legen[0][l] > thr) nlegen = l;
  }
  o.nlegen = nlegen;
  for (int k = 0; k < 4; k++)
    for (int l = 0; l < MAXNLEG; l++)
      if (std::isnan(o.legen[k][l])) return 2;
  if (!(extinction > 0) || !(scatter > 0) || !(o.back > 0)) return 2;
  return 0;
}

// ---------------------------------------------------------------- quadrature / scatcnv
// src/rt_utilities.f90:165-203 LOBATTO_QUADRATURE
void lobatto(int num, std::vector<double>& ab, std::vector<double>& w) {
  ab.assign(num, 0);
  w.assign(num, 0);
  int n = 2 * num, n1 = n - 1;
  double ci = 0.50;
  if (n % 2 == 1) ci = 1.00;
  for (int j = 1; j <= num - 1; j++) {
    double x = std::sin(F(3.141592654f) * (j - ci) / (n - .5));
    int i = 0;
    double pl, pl1, pl2, dpl, d2pl, xp;
    do {
      pl1 = 1;
      pl = x;
      for (int l = 2; l <= n1; l++) {
        pl2 = pl1;
        pl1 = pl;
        pl = ((2 * l - 1) * x * pl1 - (l - 1) * pl2) / l;
      }
      dpl = n1 * (x * pl - pl1) / (x * x - 1);
      d2pl = (2.0 * x * dpl - n1 * (n1 + 1) * pl) / (1.0 - x * x);
      xp = x;
      x = xp - dpl / d2pl;
      i = i + 1;
    } while (std::fabs(x - xp) > 3.0e-14 && i < 10);
    ab[j - 1] = x;
    w[j - 1] = 2.0 / (n * n1 * pl * pl);
  }
  ab[num - 1] = 1.0;
  w[num - 1] = 2.0 / (n * n1);
}

// src/scatcnv.f90 (NSTOKES=2, AZIORDER=0).  Output scat[l][row][col] with
// row=(i2,j2) -> i2 + 2*j2, col=(i1,j1) -> i1 + 2*j1, row-major n x n.
void scatcnv(int N, int nlegen, double coef_in[3][MAXNLEG], double extinct, double albedo,
             std::vector<double>& scat, double& ext, double& emis) {
  const int n = 2 * N;
  std::vector<double> mu, wt;
  lobatto(N, mu, wt);
  double cst = extinct * albedo / (4.0 * 3.1415926535897932384);
  const double twopi = 2.0 * 3.1415926535897932384;
  int numpts = 2 * ((nlegen + 1) / 2) + 4;
  std::vector<double> coef[3];
  for (int k = 0; k < 3; k++) {
    coef[k].assign(nlegen + 1, 0.0);
    for (int i = 0; i <= nlegen; i++) coef[k][i] = cst * coef_in[k][i];
  }
  scat.assign((size_t)4 * n * n, 0.0);
  std::vector<double> S11(numpts + 2), S12(numpts + 2), S21(numpts + 2), S22(numpts + 2);
  for (int L1 = 1; L1 <= 2; L1++)
    for (int j1 = 0; j1 < N; j1++) {
      double mu1 = mu[j1];
      if (L1 == 2) mu1 = -mu1;
      for (int L2 = 1; L2 <= 2; L2++) {
        int l = 2 * (L2 - 1) + L1;
        for (int j2 = 0; j2 < N; j2++) {
          double mu2 = mu[j2];
          if (L2 == 2) mu2 = -mu2;
          for (int k = 1; k <= numpts / 2 + 1; k++) {
            double delphi = (twopi * (k - 1)) / numpts;
            double cs = mu1 * mu2 + std::sqrt((1. - mu1 * mu1) * (1. - mu2 * mu2)) * std::cos(delphi);
            // SUM_LEGENDRE with DOSUM = (1,1,1,0,0,0)
            double sm[3];
            for (int s = 0; s < 3; s++) {
              double sum = 0.0, pl1 = 1.0, pl = 1.0, pl2 = 0.0;
              for (int L = 0; L <= nlegen; L++) {
                if (L > 0) pl = (2 * L - 1) * cs * pl1 / L - (L - 1) * pl2 / L;
                sum = sum + coef[s][L] * pl;
                pl2 = pl1;
                pl1 = pl;
              }
              sm[s] = sum;
            }
            double A1 = sm[0], B1 = sm[1], A3 = sm[2], A2 = sm[0];
            // ROTATE_PHASE_MATRIX (NSTOKES=2)
            double sin_scat = std::sqrt(std::max(0.0, 1. - cs * cs));
            double sin_t1 = std::sqrt(1. - mu1 * mu1), sin_t2 = std::sqrt(1. - mu2 * mu2);
            double sinphi = std::sin(delphi), cosphi = std::cos(delphi);
            double sin1, sin2, cos1, cos2;
            if (sin_scat == 0.0) {
              sin1 = 0; sin2 = 0; cos1 = 1; cos2 = -1;
            } else {
              sin1 = sin_t2 * sinphi / sin_scat;
              sin2 = sin_t1 * sinphi / sin_scat;
              cos1 = (sin_t1 * mu2 - sin_t2 * mu1 * cosphi) / sin_scat;
              cos2 = (sin_t2 * mu1 - sin_t1 * mu2 * cosphi) / sin_scat;
            }
            double sin21 = 2.0 * sin1 * cos1, cos21 = 1.0 - 2.0 * (sin1 * sin1);
            double sin22 = 2.0 * sin2 * cos2, cos22 = 1.0 - 2.0 * (sin2 * sin2);
            S11[k] = A1;
            S12[k] = B1 * cos21;
            S21[k] = B1 * cos22;
            S22[k] = A2 * cos21 * cos22 - A3 * sin21 * sin22;
            // MATRIX_SYMMETRY onto numpts-k+2
            int km = numpts - k + 2;
            S11[km] = S11[k]; S12[km] = S12[k]; S21[km] = S21[k]; S22[km] = S22[k];
          }
          // FOURIER_BASIS, order 0: mean over numpts points in index order
          double s11 = 0, s12 = 0, s21 = 0, s22 = 0;
          for (int k = 1; k <= numpts; k++) { s11 += S11[k]; s12 += S12[k]; s21 += S21[k]; s22 += S22[k]; }
          double* q = &scat[(size_t)(l - 1) * n * n];
          q[(0 + 2 * j2) * n + (0 + 2 * j1)] = s11 / numpts;
          q[(0 + 2 * j2) * n + (1 + 2 * j1)] = s12 / numpts;
          q[(1 + 2 * j2) * n + (0 + 2 * j1)] = s21 / numpts;
          q[(1 + 2 * j2) * n + (1 + 2 * j1)] = s22 / numpts;
        }
      }
    }
  ext = extinct;
  emis = (1.0 - albedo) * extinct;
}

// ---------------------------------------------------------------- matrices
// Column-major n x n, element (r,c) at r + n*c  (Fortran layout).
typedef std::vector<double> Mat;

// gfortran MATMUL / radmat.f90 MMULT: k-ascending dot products
void matmul(int n, const double* A, const double* B, double* C) {
  std::vector<double> t((size_t)n * n);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      double s = 0.0;
      for (int k = 0; k < n; k++) s = s + A[i + n * k] * B[k + n * j];
      t[i + n * j] = s;
    }
  std::copy(t.begin(), t.end(), C);
}
void matvec(int n, const double* A, const double* x, double* y) {
  std::vector<double> t(n);
  for (int i = 0; i < n; i++) {
    double s = 0.0;
    for (int k = 0; k < n; k++) s = s + A[i + n * k] * x[k];
    t[i] = s;
  }
  std::copy(t.begin(), t.end(), y);
}

// LAPACK DGETF2 (partial pivoting, reciprocal scaling) + DGETRI (unblocked);
// radmat.f90:201-233 MINVERT_LAPACK.  Returns nonzero on a zero pivot.
int minvert(int n, const double* Ain, double* Aout) {
  std::vector<double> A(Ain, Ain + (size_t)n * n);
  std::vector<int> ipiv(n);
  auto a = [&](int r, int c) -> double& { return A[r + (size_t)n * c]; };
  const double sfmin = std::numeric_limits<double>::min();
  int info = 0;
  for (int j = 0; j < n; j++) {
    int jp = j;
    double mx = std::fabs(a(j, j));
    for (int i = j + 1; i < n; i++)
      if (std::fabs(a(i, j)) > mx) { mx = std::fabs(a(i, j)); jp = i; }
    ipiv[j] = jp;
    if (a(jp, j) != 0.0) {
      if (jp != j)
        for (int c = 0; c < n; c++) std::swap(a(j, c), a(jp, c));
      if (std::fabs(a(j, j)) >= sfmin) {
        double r = 1.0 / a(j, j);
        for (int i = j + 1; i < n; i++) a(i, j) *= r;
      } else {
        for (int i = j + 1; i < n; i++) a(i, j) = a(i, j) / a(j, j);
      }
    } else if (info == 0) {
      info = j + 1;
    }
    for (int c = j + 1; c < n; c++) {
      double t = a(j, c);
      if (t != 0.0)
        for (int i = j + 1; i < n; i++) a(i, c) = a(i, c) - a(i, j) * t;
    }
  }
  if (info) return info;
  // DTRTI2 upper, non-unit
  for (int j = 0; j < n; j++) {
    a(j, j) = 1.0 / a(j, j);
    double ajj = -a(j, j);
    // DTRMV upper, no-transpose on x = A(0:j-1, j)
    for (int jj = 0; jj < j; jj++) {
      double t = a(jj, j);
      if (t != 0.0) {
        for (int i = 0; i < jj; i++) a(i, j) = a(i, j) + t * a(i, jj);
        a(jj, j) = a(jj, j) * a(jj, jj);
      }
    }
    for (int i = 0; i < j; i++) a(i, j) = ajj * a(i, j);
  }
  // DGETRI unblocked: solve inv(A)*L = inv(U)
  std::vector<double> work(n);
  for (int j = n - 1; j >= 0; j--) {
    for (int i = j + 1; i < n; i++) { work[i] = a(i, j); a(i, j) = 0.0; }
    if (j < n - 1) {
      // DGEMV('N', n, n-j-1, -1, A(:,j+1:), work(j+1:), 1, A(:,j))
      for (int jj = j + 1; jj < n; jj++) {
        double t = -1.0 * work[jj];
        if (t != 0.0)
          for (int i = 0; i < n; i++) a(i, j) = a(i, j) + t * a(i, jj);
      }
    }
  }
  for (int j = n - 2; j >= 0; j--) {
    int jp = ipiv[j];
    if (jp != j)
      for (int r = 0; r < n; r++) std::swap(a(r, j), a(r, jp));
  }
  std::copy(A.begin(), A.end(), Aout);
  return 0;
}

// ---------------------------------------------------------------- RT4
// src/rt_utilities.f90:69-90 PLANCK_FUNCTION with UNITS='r'
double planck(double T, double wl) {
  if (T > 0.0) return 1.1911e8 / p5(wl) / (std::exp(1.4388e4 / (wl * T)) - 1);
  return 0.0;
}

struct Layer {  // R,T (n x n, two parts each), S (n, two parts)
  Mat R, T;
  std::vector<double> S;
};

// The start of a scattering layer: the number of doublings from
// extinct_matrix(1) + gas (src/radtran4.f90:319-329), INITIAL_SOURCE4
// (src/radintg4.f90:51-73) and INITIALIZE4 (:1-45).  With T-matrix species
// the extinction matrix and emission vector are theirs plus scatcnv's.
void layer_start(int N, const std::vector<double>& mu, const std::vector<double>& w, double zdiff, double gas,
                 double planck0, double planck1, const std::vector<double>& scat, double ext_k, double emis_k,
                 const double* tm_ext, const double* tm_emis, Mat& R, Mat& T, std::vector<double>& lin,
                 int& num_doubles, double& linfactor) {
  const int n = 2 * N;
  // extinct_matrix(1) + gas (src/radtran4.f90:323); with T-matrix species the
  // layer's matrices are theirs plus scatcnv's
  double extinct = (tm_ext ? tm_ext[0] + ext_k : ext_k) + gas;
  double f = std::log(std::max(extinct * zdiff, 1.0e-7) / 1.0e-6) / (double)std::log(2.0f);
  num_doubles = 0;
  if (f > 0.0) num_doubles = (int)f + 1;
  double num_sub = (double)std::ldexp(1.0f, num_doubles);
  double delta_z = zdiff / num_sub;
  // INITIAL_SOURCE4
  lin.assign(2 * n, 0.0);
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < N; j++) {
      double e = (i == 0) ? gas : 0.0;
      double tmp = planck0 * delta_z / mu[j];
      double ev = (i == 0) ? emis_k : 0.0;
      if (tm_emis) ev = tm_emis[i + 2 * j] + ((i == 0) ? emis_k : 0.0);
      lin[i + 2 * j] = tmp * (ev + e);
      lin[n + i + 2 * j] = tmp * (ev + e);
    }
  linfactor = (planck0 == 0.0) ? 0.0 : (planck1 / planck0 - 1.0) / num_sub;
  // INITIALIZE4
  const double C = 2.0 * 3.1415926535897932384;
  R.assign((size_t)2 * n * n, 0.0);
  T.assign((size_t)2 * n * n, 0.0);
  const double* Q1 = &scat[0];
  const double* Q2 = &scat[(size_t)1 * n * n];
  const double* Q3 = &scat[(size_t)2 * n * n];
  const double* Q4 = &scat[(size_t)3 * n * n];
  for (int i2 = 0; i2 < 2; i2++)
    for (int j2 = 0; j2 < N; j2++) {
      double tmp = delta_z / mu[j2];
      int row = i2 + 2 * j2;
      for (int i1 = 0; i1 < 2; i1++) {
        double gext = (i1 == i2) ? gas : 0.0;
        for (int j1 = 0; j1 < N; j1++) {
          int col = i1 + 2 * j1;
          size_t qi = (size_t)row * n + col, mi = (size_t)row + (size_t)n * col;
          R[mi] = C * tmp * w[j1] * Q2[qi];
          R[n * n + mi] = C * tmp * w[j1] * Q3[qi];
          double diag = (i1 == i2 && j1 == j2) ? 1.0 : 0.0;
          double ex = 0.0;
          // EXTINCT_MATRIX(I2, I1, J2, L) + GEXT
          const double em = tm_ext ? tm_ext[i2 + 2 * (i1 + 2 * j2)] + ((i1 == i2) ? ext_k : 0.0)
                                   : ((i1 == i2) ? ext_k : 0.0);
          if (j1 == j2) ex = em + gext;
          T[mi] = diag - tmp * (ex - C * w[j1] * Q1[qi]);
          if (j1 == j2) ex = em + gext;
          T[n * n + mi] = diag - tmp * (ex - C * w[j1] * Q4[qi]);
        }
      }
    }
}

// src/radintg4.f90:1-45 INITIALIZE4 + 51-73 INITIAL_SOURCE4 + 174-309 DOUBLING_INTEGRATION4
void scattering_layer(int N, const std::vector<double>& mu, const std::vector<double>& w, double zdiff, double gas,
                      double planck0, double planck1, const std::vector<double>& scat, double ext_k, double emis_k,
                      Layer& out, int& num_doubles, const double* tm_ext = nullptr, const double* tm_emis = nullptr) {
  const int n = 2 * N;
  Mat R, T;
  std::vector<double> lin;
  double linfactor = 0.0;
  layer_start(N, mu, w, zdiff, gas, planck0, planck1, scat, ext_k, emis_k, tm_ext, tm_emis, R, T, lin, num_doubles,
              linfactor);
  // DOUBLING_INTEGRATION4 with SYMMETRIC = .true.
  std::vector<double> cst(lin), tlin(2 * n), tcst(2 * n);
  double linfac = linfactor;
  Mat X(n * n), Y(n * n), G(n * n), TR((size_t)2 * n * n), TT((size_t)2 * n * n);
  std::vector<double> xv(n), yv(n);
  double *R1 = &R[0], *R2 = &R[n * n], *T1 = &T[0], *T2 = &T[n * n];
  for (int it = 0; it < num_doubles; it++) {
    matmul(n, R1, R2, X.data());
    for (int k = 0; k < n * n; k++) Y[k] = ((k % (n + 1)) == 0 ? 1.0 : 0.0) - X[k];
    minvert(n, Y.data(), G.data());
    matmul(n, R1, T2, X.data());
    matmul(n, G.data(), X.data(), Y.data());
    matmul(n, T1, Y.data(), X.data());
    for (int k = 0; k < n * n; k++) TR[k] = R1[k] + X[k];
    matmul(n, G.data(), T1, X.data());
    matmul(n, T1, X.data(), TT.data());
    // Sp
    for (int i = 0; i < n; i++) xv[i] = linfac * cst[n + i];
    for (int i = 0; i < n; i++) yv[i] = lin[n + i] + xv[i];
    matvec(n, R1, yv.data(), xv.data());
    for (int i = 0; i < n; i++) yv[i] = lin[i] + xv[i];
    matvec(n, G.data(), yv.data(), xv.data());
    matvec(n, T1, xv.data(), yv.data());
    for (int i = 0; i < n; i++) xv[i] = lin[i] + yv[i];
    for (int i = 0; i < n; i++) yv[i] = linfac * cst[i];
    for (int i = 0; i < n; i++) tlin[i] = xv[i] + yv[i];
    // Cp
    for (int i = 0; i < n; i++) yv[i] = cst[n + i];
    matvec(n, R1, yv.data(), xv.data());
    for (int i = 0; i < n; i++) yv[i] = cst[i] + xv[i];
    matvec(n, G.data(), yv.data(), xv.data());
    matvec(n, T1, xv.data(), yv.data());
    for (int i = 0; i < n; i++) tcst[i] = cst[i] + yv[i];
    std::copy(TR.begin(), TR.begin() + n * n, TR.begin() + n * n);
    std::copy(TT.begin(), TT.begin() + n * n, TT.begin() + n * n);
    // Sm
    for (int i = 0; i < n; i++) xv[i] = linfac * cst[n + i];
    for (int i = 0; i < n; i++) yv[i] = lin[n + i] + xv[i];
    for (int i = 0; i < n; i++) xv[i] = lin[i];
    matvec(n, R2, xv.data(), xv.data());
    for (int i = 0; i < n; i++) yv[i] = yv[i] + xv[i];
    matvec(n, G.data(), yv.data(), xv.data());
    matvec(n, T2, xv.data(), yv.data());
    for (int i = 0; i < n; i++) tlin[n + i] = lin[n + i] + yv[i];
    // Cm
    for (int i = 0; i < n; i++) xv[i] = cst[i];
    matvec(n, R2, xv.data(), xv.data());
    for (int i = 0; i < n; i++) yv[i] = cst[n + i] + xv[i];
    matvec(n, G.data(), yv.data(), xv.data());
    matvec(n, T2, xv.data(), yv.data());
    for (int i = 0; i < n; i++) tcst[n + i] = cst[n + i] + yv[i];
    lin = tlin;
    cst = tcst;
    linfac = 2.0 * linfac;
    std::copy(TR.begin(), TR.end(), R.begin());
    std::copy(TT.begin(), TT.end(), T.begin());
  }
  out.R = R;
  out.T = T;
  out.S = lin;
}

// src/radintg4.f90:79-117 NONSCATTER_LAYER4
void nonscatter_layer(int N, const std::vector<double>& mu, double dtau, double planck0, double planck1, Layer& out) {
  const int n = 2 * N;
  out.R.assign((size_t)2 * n * n, 0.0);
  out.T.assign((size_t)2 * n * n, 0.0);
  out.S.assign(2 * n, 0.0);
  for (int j = 0; j < N; j++) {
    double fac = std::exp(-dtau / mu[j]);
    for (int i = 0; i < 2; i++) {
      int r = i + 2 * j;
      out.T[r + (size_t)n * r] = fac;
      out.T[n * n + r + (size_t)n * r] = fac;
    }
  }
  if (dtau > 0.0)
    for (int j = 0; j < N; j++) {
      double path = dtau / mu[j];
      double slope = (planck1 - planck0) / path;
      out.S[0 + 2 * j] = planck1 - slope - (planck1 - slope * (1.0 + path)) * std::exp(-path);
      out.S[n + 0 + 2 * j] = planck0 + slope - (planck0 + slope * (1.0 + path)) * std::exp(-path);
    }
}

// src/radintg4.f90:447-513 COMBINE_LAYERS4 (layer 1 on top of layer 2)
void combine(int n, const Layer& L1, const Layer& L2, Layer& out) {
  const double *R1p = &L1.R[0], *R1m = &L1.R[n * n], *T1p = &L1.T[0], *T1m = &L1.T[n * n];
  const double *R2p = &L2.R[0], *R2m = &L2.R[n * n], *T2p = &L2.T[0], *T2m = &L2.T[n * n];
  const double *S1p = &L1.S[0], *S1m = &L1.S[n], *S2p = &L2.S[0], *S2m = &L2.S[n];
  Layer o;
  o.R.assign((size_t)2 * n * n, 0);
  o.T.assign((size_t)2 * n * n, 0);
  o.S.assign(2 * n, 0);
  Mat X(n * n), Y(n * n), G(n * n);
  std::vector<double> w(n);
  matmul(n, R1p, R2m, X.data());
  for (int k = 0; k < n * n; k++) Y[k] = ((k % (n + 1)) == 0 ? 1.0 : 0.0) - X[k];
  minvert(n, Y.data(), G.data());
  matmul(n, R1p, T2m, X.data());
  matmul(n, G.data(), X.data(), Y.data());
  matmul(n, T2p, Y.data(), X.data());
  for (int k = 0; k < n * n; k++) o.R[k] = R2p[k] + X[k];
  matmul(n, G.data(), T1p, X.data());
  matmul(n, T2p, X.data(), &o.T[0]);
  matvec(n, R1p, S2m, w.data());
  for (int i = 0; i < n; i++) w[i] = S1p[i] + w[i];
  matvec(n, G.data(), w.data(), w.data());
  matvec(n, T2p, w.data(), w.data());
  for (int i = 0; i < n; i++) o.S[i] = S2p[i] + w[i];
  matmul(n, R2m, R1p, X.data());
  for (int k = 0; k < n * n; k++) Y[k] = ((k % (n + 1)) == 0 ? 1.0 : 0.0) - X[k];
  minvert(n, Y.data(), G.data());
  matmul(n, R2m, T1p, X.data());
  matmul(n, G.data(), X.data(), Y.data());
  matmul(n, T1m, Y.data(), X.data());
  for (int k = 0; k < n * n; k++) o.R[n * n + k] = R1m[k] + X[k];
  matmul(n, G.data(), T2m, X.data());
  matmul(n, T1m, X.data(), &o.T[n * n]);
  matvec(n, R2m, S1p, w.data());
  for (int i = 0; i < n; i++) w[i] = S2m[i] + w[i];
  matvec(n, G.data(), w.data(), w.data());
  matvec(n, T1m, w.data(), w.data());
  for (int i = 0; i < n; i++) o.S[n + i] = S1m[i] + w[i];
  out = std::move(o);
}

// src/radintg4.f90:119-172 INTERNAL_RADIANCE4
void internal_radiance(int n, const Layer& up, const Layer& dn, const double* intop, const double* inbot,
                       double* uprad, double* dnrad) {
  const double *UR1 = &up.R[0], *UT1 = &up.T[0], *US1 = &up.S[0];
  const double *DR2 = &dn.R[n * n], *DT2 = &dn.T[n * n], *DS2 = &dn.S[n];
  Mat X(n * n), Y(n * n);
  std::vector<double> S(n), V(n);
  matmul(n, UR1, DR2, X.data());
  for (int k = 0; k < n * n; k++) Y[k] = ((k % (n + 1)) == 0 ? 1.0 : 0.0) - X[k];
  minvert(n, Y.data(), X.data());
  matvec(n, DT2, inbot, V.data());
  matvec(n, UR1, V.data(), S.data());
  matvec(n, UT1, intop, V.data());
  for (int i = 0; i < n; i++) S[i] = V[i] + S[i];
  matvec(n, UR1, DS2, V.data());
  for (int i = 0; i < n; i++) S[i] = V[i] + S[i];
  for (int i = 0; i < n; i++) S[i] = US1[i] + S[i];
  matvec(n, X.data(), S.data(), dnrad);
  matmul(n, DR2, UR1, X.data());
  for (int k = 0; k < n * n; k++) Y[k] = ((k % (n + 1)) == 0 ? 1.0 : 0.0) - X[k];
  minvert(n, Y.data(), X.data());
  matvec(n, UT1, intop, V.data());
  matvec(n, DR2, V.data(), S.data());
  matvec(n, DT2, inbot, V.data());
  for (int i = 0; i < n; i++) S[i] = V[i] + S[i];
  matvec(n, DR2, US1, V.data());
  for (int i = 0; i < n; i++) S[i] = V[i] + S[i];
  for (int i = 0; i < n; i++) S[i] = DS2[i] + S[i];
  matvec(n, X.data(), S.data(), uprad);
}

// src/rt_utilities.f90:687-735 CONVERT_OUTPUT (UNITS='T', FLUXCODE=0)
// Simple radar of one column at one frequency: src/radar_simulator.f90:123-176
// (radar_mode 'simple', polarisation NN, radar_nPeaks = 1) called per layer
// with hydrometeors in the layer order of src/hydrometeor_extinction.f90:96-106
// (top-down when radar_attenuation = 'top-down'), and the gas attenuation of
// src/run_rt.f90:119-121.  Initial values as src/vars_output.f90:150-152.
void radar_simple(const orc_settings& st, int L, double freq, const std::vector<double>& hgt_lev,
                  const std::vector<int>& present, const std::vector<double>& kexthydro,
                  const std::vector<double>& back, const std::vector<double>& kextatmo, std::vector<double>& ze,
                  std::vector<double>& att_hydro, std::vector<double>& att_atmo) {
  ze.assign(L, -9999.0);
  att_hydro.assign(L, 0.0);
  att_atmo.assign(L, 0.0);
  std::vector<double> dh(L);
  for (int z = 0; z < L; z++) {
    dh[z] = hgt_lev[z + 1] - hgt_lev[z];
    att_atmo[z] = 10.0 * std::log10(std::exp(kextatmo[z] * dh[z]));
  }
  const double K2 = st.radar_k2;
  const double wavelength = C_LIGHT / (freq * 1.e9);
  const double pi5 = (PI * PI) * (PI * PI) * PI, w2 = wavelength * wavelength, w4 = w2 * w2;
  const bool down = st.radar_attenuation == 2;
  for (int k = 0; k < L; k++) {
    const int iz = down ? L - 1 - k : k;
    if (!present[iz]) continue;
    att_hydro[iz] = 10.0 * std::log10(std::exp(kexthydro[iz] * dh[iz]));
    double ze_back = 1.e18 * (1.0 / (K2 * pi5)) * back[iz] * w4;
    double pia = 0.0;
    if (st.radar_attenuation != 0) {
      if (k > 0) {
        double sh = 0.0, sa = 0.0;
        for (int j = 0; j < k; j++) {
          const int jz = down ? L - 1 - j : j;
          sh = sh + att_hydro[jz];
          sa = sa + att_atmo[jz];
        }
        pia = 2 * (sh + sa);
      }
      pia = pia + att_hydro[iz] + att_atmo[iz];
    }
    pia = std::pow(10.0, 0.1 * pia);
    ze_back = ze_back / pia;
    ze[iz] = (ze_back == 0.0) ? -9999.0 : 10 * std::log10(ze_back);
  }
}

double rad_to_tb(double rad, double wl) {
  if (rad > 0.0) return 1.4388e4 / (wl * std::log(1.0 + 1.1911e8 / (rad * p5(wl))));
  if (rad == 0.0) return 0.0;
  return -1.4388e4 / (wl * std::log(1.0 + 1.1911e8 / (-rad * p5(wl))));
}

}  // namespace

// ======================================================================
extern "C" {

// calc_tmatrix of one species at one frequency (tmatrix_oracle.cpp)
int orc_tmatrix_species(int nummu, double frequency, double ref_re, double ref_im, int phase, int nbins,
                        const double* dmax, const double* del_d, const double* ndens, const double* density,
                        const double* as_ratio, const double* canting, double* scat, double* ext, double* emis,
                        double* back_spec, double* sback);

int orc_gas_r98(double f, double T, double rhowv, double pres, double* kext) {
  return gas_r98(f, T, rhowv, pres, kext);
}

// get_eps_water (src/eps_water.f90:6-70) for liq_mod code 0..4; returns 2
// where the model has no value.
int orc_get_eps_water(int liq_mod, double s, double T_c, double f, double* re, double* im) {
  cplx e;
  switch (liq_mod) {
    case 0: e = eps_water_tkc(T_c, f); break;
    case 1: e = eps_water_ellison(s, T_c, f); break;
    case 2: e = eps_water_liebe(T_c, f); break;
    case 3:
      if (eps_water_ray(T_c, f, e)) return 2;
      break;
    case 4: e = eps_water_stogryn(s, T_c, f); break;
    default: return 2;
  }
  *re = e.re;
  *im = e.im;
  return 0;
}

// mpm93 as get_gasabs calls it: p, e in Pa, T in K; Np/m
double orc_gas_l93(double f, double press, double vap, double T) { return gas_l93(f, press, vap, T); }

void orc_eps_water_tkc(double T_c, double f, double* re, double* im) {
  cplx e = eps_water_tkc(T_c, f);
  *re = e.re;
  *im = e.im;
}

void orc_lobatto(int num, double* mu, double* w) {
  std::vector<double> a, b;
  lobatto(num, a, b);
  for (int i = 0; i < num; i++) { mu[i] = a[i]; w[i] = b[i]; }
}

int orc_minvert(int n, const double* A, double* Ainv) { return minvert(n, A, Ainv); }

// Mie coefficients a_n, b_n (miecalc, src/mie_scat_utilities.f90:8-75) of a
// sphere of size parameter x and index m; returns the number of terms (at
// most cap), or -1.
int orc_miecalc(double x, double mr, double mi, int cap, double* a_re, double* a_im, double* b_re, double* b_im) {
  int nterms = 0;
  std::vector<cplx> a, b;
  if (miecalc(nterms, x, cmk(mr, mi), a, b)) return -1;
  for (int n = 0; n < nterms && n < cap; n++) {
    a_re[n] = a[n + 1].re;
    a_im[n] = a[n + 1].im;
    b_re[n] = b[n + 1].re;
    b_im[n] = b[n + 1].im;
  }
  return nterms;
}

// The start of a scattering layer (layer_start) for tests of the device's
// layer start: scat [4][n][n] (rows i2 + 2 j2, columns i1 + 2 j1), the
// optional T-matrix extinction matrix [2][2][N] and emission [2][N]; R and T
// [2][n][n] column-major, lin [2][n]; returns the number of doublings.
int orc_layer_start(int N, double zdiff, double gas, double planck0, double planck1, const double* scat, double ext_k,
                    double emis_k, const double* tm_ext, const double* tm_emis, double* R_out, double* T_out,
                    double* lin_out, double* linfactor) {
  const int n = 2 * N;
  std::vector<double> mu, w;
  lobatto(N, mu, w);
  std::vector<double> sc(scat, scat + (size_t)4 * n * n), lin;
  Mat R, T;
  int nd = 0;
  layer_start(N, mu, w, zdiff, gas, planck0, planck1, sc, ext_k, emis_k, tm_ext, tm_emis, R, T, lin, nd, *linfactor);
  std::copy(R.begin(), R.end(), R_out);
  std::copy(T.begin(), T.end(), T_out);
  std::copy(lin.begin(), lin.end(), lin_out);
  return nd;
}

// eps_mix((1,0), m, density) of src/eps_mix.f90 (the soft-spheroid mixing
// the T-matrix branch applies per bin, src/tmatrix.f90:171-175).
void orc_eps_mix_m(double re, double im, double dens, double* ore, double* oim) {
  cplx e = eps_mix_m(cmk(re, im), dens);
  *ore = e.re;
  *oim = e.im;
}

void orc_e_sat(double T, double* e) { *e = e_sat_gg_water(T); }

// Full passive path for one column (src/run_rt.f90 per frequency, with the
// column pre-processing of src/vars_atmosphere.f90:671).  Level arrays
// bottom-up [L+1], layer arrays [L], hydro arrays [L][H]; NaN = missing.
// tb: [noutlevels][2N][nfreq][2]; emissivity: [2][nfreq][N]; angles: [2N].
// Returns 0, or the reference error code (2) on a fatal condition.
int orc_run_column_fs(const orc_settings* st, const orc_species* sp, int nhydro, int L, const double* hgt_lev,
                      const double* temp_lev, const double* press_lev, const double* relhum_lev, const double* hgt,
                      const double* temp, const double* press, const double* relhum, const double* hydro_q,
                      const double* hydro_n, const double* hydro_reff, double groundtemp, int noutlevels,
                      const double* obs_height, char sfc_refl, int nfreq, const double* freqs, double* tb,
                      double* emissivity_out, double* angles_deg, orc_debug* dbg, const orc_fullspec* fs);

int orc_run_column(const orc_settings* st, const orc_species* sp, int nhydro, int L, const double* hgt_lev,
                   const double* temp_lev, const double* press_lev, const double* relhum_lev, const double* hgt,
                   const double* temp, const double* press, const double* relhum, const double* hydro_q,
                   const double* hydro_n, const double* hydro_reff, double groundtemp, int noutlevels,
                   const double* obs_height, char sfc_refl, int nfreq, const double* freqs, double* tb,
                   double* emissivity_out, double* angles_deg, orc_debug* dbg) {
  return orc_run_column_fs(st, sp, nhydro, L, hgt_lev, temp_lev, press_lev, relhum_lev, hgt, temp, press, relhum,
                           hydro_q, hydro_n, hydro_reff, groundtemp, noutlevels, obs_height, sfc_refl, nfreq, freqs,
                           tb, emissivity_out, angles_deg, dbg, nullptr);
}

int orc_run_column_tm(const orc_settings* st, const orc_species* sp, int nhydro, int L, const double* hgt_lev,
                      const double* temp_lev, const double* press_lev, const double* relhum_lev, const double* hgt,
                      const double* temp, const double* press, const double* relhum, const double* hydro_q,
                      const double* hydro_n, const double* hydro_reff, double groundtemp, int noutlevels,
                      const double* obs_height, char sfc_refl, int nfreq, const double* freqs, double* tb,
                      double* emissivity_out, double* angles_deg, orc_debug* dbg, const orc_fullspec* fs,
                      const int* scat_code, const double* canting);

// As orc_run_column; with `fs` the size distributions come from the given
// full spectra instead of hydro_q / hydro_n / hydro_reff.
int orc_run_column_fs(const orc_settings* st, const orc_species* sp, int nhydro, int L, const double* hgt_lev,
                      const double* temp_lev, const double* press_lev, const double* relhum_lev, const double* hgt,
                      const double* temp, const double* press, const double* relhum, const double* hydro_q,
                      const double* hydro_n, const double* hydro_reff, double groundtemp, int noutlevels,
                      const double* obs_height, char sfc_refl, int nfreq, const double* freqs, double* tb,
                      double* emissivity_out, double* angles_deg, orc_debug* dbg, const orc_fullspec* fs) {
  return orc_run_column_tm(st, sp, nhydro, L, hgt_lev, temp_lev, press_lev, relhum_lev, hgt, temp, press, relhum,
                           hydro_q, hydro_n, hydro_reff, groundtemp, noutlevels, obs_height, sfc_refl, nfreq, freqs,
                           tb, emissivity_out, angles_deg, dbg, fs, nullptr, nullptr);
}

// As orc_run_column_fs, with species whose scat_code[h] is 1 scattering as
// T-matrix spheroids (scat_name 'tmatrix', src/scatProperties.f90:289-367) of
// the species' aspect ratio and canting[h] (deg).  Their scattering matrix,
// extinction matrix and emission vector are added to the layer's after
// scatcnv (src/hydrometeor_extinction.f90:329-339); their extinction at the
// 16th quadrature angle joins kexttot (src/scatProperties.f90:367, :921).
// The reference leaves salb_hydro unset for them (:929-934); here it is 0,
// which only matters for layers that also hold Mie species.
int orc_run_column_tm(const orc_settings* st, const orc_species* sp, int nhydro, int L, const double* hgt_lev,
                      const double* temp_lev, const double* press_lev, const double* relhum_lev, const double* hgt,
                      const double* temp, const double* press, const double* relhum, const double* hydro_q,
                      const double* hydro_n, const double* hydro_reff, double groundtemp, int noutlevels,
                      const double* obs_height, char sfc_refl, int nfreq, const double* freqs, double* tb,
                      double* emissivity_out, double* angles_deg, orc_debug* dbg, const orc_fullspec* fs,
                      const int* scat_code, const double* canting) {
  const int N = st->nummu, n = 2 * N;
  if (scat_code && fs && !fs->as_ratio)
    for (int h = 0; h < nhydro; h++)
      if (scat_code[h] == 1) return 2;  // full spectra carry the aspect ratio per bin
  if (scat_code && N < 16)
    for (int h = 0; h < nhydro; h++)
      if (scat_code[h] == 1) return 2;  // kext_hydro reads extinct_matrix(1,1,16,1)
  Atmo a;
  a.L = L;
  a.hgt_lev.assign(hgt_lev, hgt_lev + L + 1);
  a.temp_lev.assign(temp_lev, temp_lev + L + 1);
  a.press_lev.assign(press_lev, press_lev + L + 1);
  a.relhum_lev.assign(relhum_lev, relhum_lev + L + 1);
  a.hgt.assign(hgt, hgt + L);
  a.temp.assign(temp, temp + L);
  a.press.assign(press, press + L);
  a.relhum.assign(relhum, relhum + L);
  a.groundtemp = groundtemp;
  fill_missing(a);

  std::vector<double> mu, qw;
  lobatto(N, mu, qw);
  if (angles_deg)
    for (int j = 0; j < N; j++) {
      angles_deg[j] = 180 - (180. * std::acos(mu[N - 1 - j]) / PI);
      angles_deg[N + j] = (180. * std::acos(mu[j]) / PI);
    }

  // output levels (src/run_rt.f90:166-184)
  std::vector<int> outlev(noutlevels);
  for (int io = 0; io < noutlevels; io++) {
    double ob = obs_height[io];
    if (ob >= a.hgt_lev[L]) outlev[io] = 1;
    else if (ob <= a.hgt_lev[0]) outlev[io] = L + 1;
    else {
      for (int nz = 1; nz <= L; nz++)
        if (a.hgt_lev[nz] >= ob) {
          if (std::fabs(a.hgt_lev[nz] - ob) <= std::fabs(a.hgt_lev[nz - 1] - ob)) outlev[io] = L - nz + 1;
          else outlev[io] = L - nz + 2;
          break;
        }
    }
  }

  // hydrometeor presence per layer is frequency independent
  std::vector<int> present(L, 0);

  // save_psd per-particle backscattering cross section of the last frequency
  // (src/scatProperties.f90:914-917: back_spec / num_density, NaN where a bin is empty)
  int fi_cur = 0;
  auto save_bscat = [&](int z, int h, const MieOut& mo, const std::vector<double>& ndens) {
    if (!dbg || !dbg->psd_bscat || fi_cur != nfreq - 1) return;
    const size_t po = ((size_t)z * nhydro + h) * dbg->psd_nbin;
    for (int i = 0; i < (int)ndens.size() && i < dbg->psd_nbin; i++) dbg->psd_bscat[po + i] = mo.back_spec[i] / ndens[i];
  };
  for (int fi = 0; fi < nfreq; fi++) {
    fi_cur = fi;
    const double freq = freqs[fi];
    const double wl = C_LIGHT / (freq * 1.e3);
    // gas (src/get_gasabs.f90)
    std::vector<double> kgas(L, 0.0);
    if (st->lgas_extinction)
      for (int z = 0; z < L; z++) {
        if (st->gas_mod == 1) kgas[z] = gas_l93(freq, a.press[z], a.vapor_pressure[z], a.temp[z]);
        else if (gas_r98(freq, a.temp[z], a.rho_vap[z], a.press[z], &kgas[z])) return 2;
      }
    // hydrometeors (src/hydrometeor_extinction.f90)
    std::vector<std::vector<double>> scat(L);
    std::vector<double> extk(L, 0.0), emk(L, 0.0), kext_h(L, 0.0), back_h(L, 0.0);
    // T-matrix species of each layer: scattering matrix (4 quadrants as scat),
    // extinction matrix extinct_matrix(i2, i1, j) [2][2][N], emission vector [2][N]
    std::vector<std::vector<double>> tm_scat(L), tm_ext(L), tm_emis(L);
    for (int z = 0; z < L; z++) {
      double kexttot = 0.0, salbedo = 0.0, backtot = 0.0;
      double legen_coef[3][MAXNLEG];
      std::memset(legen_coef, 0, sizeof(legen_coef));
      int nlegen_coef = 0;
      bool pres = false;
      double qsum = 0.0;
      for (int h = 0; h < nhydro; h++) qsum += hydro_q[z * nhydro + h];
      // calc_tmatrix of one species (src/scatProperties.f90:289-367): per-bin
      // aspect ratio and canting, negative or NaN read as 0 (:284-287)
      auto add_tmatrix = [&](const orc_species& s, const Bins& bn, const std::vector<double>& ndens, double refre,
                             double refim, std::vector<double> asl, std::vector<double> cl) -> int {
        const int nb = bn.nbin;
        for (int i = 0; i < nb; i++) {
          if (asl[i] < 0 || std::isnan(asl[i])) asl[i] = 0.0;
          if (cl[i] < 0 || std::isnan(cl[i])) cl[i] = 0.0;
        }
        std::vector<double> bk(nb), ts((size_t)8 * N * N), te(4 * N), tv(2 * N), sb(4);
        if (orc_tmatrix_species(N, freq * 1e9, refre, -refim, s.liq_ice, nb, bn.diam.data(), bn.delta_d.data(),
                                ndens.data(), bn.dens.data(), asl.data(), cl.data(), ts.data(), te.data(), tv.data(),
                                bk.data(), sb.data()))
          return 2;
        if (tm_scat[z].empty()) {
          tm_scat[z].assign((size_t)4 * n * n, 0.0);
          tm_ext[z].assign(4 * N, 0.0);
          tm_emis[z].assign(2 * N, 0.0);
        }
        // scatter_matrix(i2, ll, i1, jj, kk) -> quadrant L = kk and L = 5 - kk
        // (src/scatProperties.f90:316-317), rows (i2, ll), columns (i1, jj)
        for (int kk = 0; kk < 2; kk++)
          for (int jj = 0; jj < N; jj++)
            for (int i1 = 0; i1 < 2; i1++)
              for (int ll = 0; ll < N; ll++)
                for (int i2 = 0; i2 < 2; i2++) {
                  const double v = ts[i2 + 2 * (ll + N * (i1 + 2 * (jj + N * kk)))];
                  const size_t qi = (size_t)(i2 + 2 * ll) * n + (i1 + 2 * jj);
                  tm_scat[z][(size_t)kk * n * n + qi] += v;
                  tm_scat[z][(size_t)(3 - kk) * n * n + qi] += v;
                }
        for (int e = 0; e < 4 * N; e++) tm_ext[z][e] += te[e];
        for (int e = 0; e < 2 * N; e++) tm_emis[z][e] += tv[e];
        const double kext_hydro = te[0 + 2 * (0 + 2 * 15)];  // extinct_matrix(1,1,16,1) (:367)
        kexttot = kexttot + kext_hydro;
        backtot = backtot + 4.0 * PI * sb[0];  // "NN": 4 pi Sback(1,1) (:322-358)
        if (kexttot == 0.0) salbedo = 0.0;
        else salbedo = salbedo + (0.0 * kext_hydro);
        if (kexttot < 0.0 || std::isnan(kexttot)) return 2;
        return 0;
      };
      for (int h = 0; h < nhydro; h++) {
        const orc_species& s = sp[h];
        if (fs) {
          // src/hydrometeor_extinction.f90:122-151
          const int nb = fs->nbin;
          const size_t o = ((size_t)z * nhydro + h) * nb, ob = ((size_t)z * nhydro + h) * (nb + 1);
          double nsum = 0.0;
          for (int i = 0; i < nb; i++) nsum += fs->n[o + i];
          if (!(nsum > 0.0 || st->hydro_threshold <= 0)) continue;
          pres = true;
          if (s.dist == D_DISABLED) continue;  // scat_name 'disabled' (src/scatProperties.f90:203)
          Bins bn;
          bn.nbin = nb;
          bn.d_ds.assign(fs->d + o, fs->d + o + nb);
          bn.diam = bn.d_ds;
          bn.n_ds.assign(fs->n + o, fs->n + o + nb);
          bn.dens.assign(fs->rho + o, fs->rho + o + nb);
          bn.mass.assign(fs->mass + o, fs->mass + o + nb);
          bn.delta_d.resize(nb);
          for (int i = 0; i < nb; i++) bn.delta_d[i] = fs->d_bound[ob + i + 1] - fs->d_bound[ob + i];
          std::vector<double> ndens(nb);
          for (int i = 0; i < nb; i++) ndens[i] = bn.n_ds[i] / bn.delta_d[i];
          double refre, refim;
          if (s.liq_ice == 1) {
            if (ref_water_mod(st->liq_mod, a.temp[z] - F(273.15f), freq, refre, refim)) return 2;
          } else {
            ref_ice(a.temp[z], freq, refre, refim);
          }
          if (scat_code && scat_code[h] == 1) {
            // hydrofs_as_ratio / hydrofs_canting per bin (src/scatProperties.f90:257-265)
            std::vector<double> asl(fs->as_ratio + o, fs->as_ratio + o + nb);
            std::vector<double> cl = fs->canting ? std::vector<double>(fs->canting + o, fs->canting + o + nb)
                                                 : std::vector<double>(nb, 0.0);
            if (add_tmatrix(s, bn, ndens, refre, refim, asl, cl)) return 2;
            continue;
          }
          MieOut mo;
          if (calc_mie_spheres(*st, freq * 1e9, s.liq_ice, bn, ndens, refre, refim, mo)) return 2;
          save_bscat(z, h, mo, ndens);
          nlegen_coef = std::max(nlegen_coef, mo.nlegen);
          kexttot = kexttot + mo.kext;
          backtot = backtot + mo.back;
          if (kexttot == 0.0) salbedo = 0.0;
          else salbedo = salbedo + (mo.salb * mo.kext);
          if (nlegen_coef > 0)
            for (int jj = 0; jj < nlegen_coef; jj++)
              for (int k = 0; k < 3; k++) legen_coef[k][jj] = legen_coef[k][jj] + (mo.legen[k][jj] * mo.salb * mo.kext);
          if (kexttot < 0.0 || std::isnan(kexttot)) return 2;
          if (nlegen_coef > MAXNLEG - 1) return 2;
          continue;
        }
        if (s.dist == D_DISABLED) continue;
        double qall = (st->hydro_includehydroinrhoair && !std::isnan(qsum)) ? qsum : 0.0;
        double q_h = q2abs(hydro_q[z * nhydro + h], a.temp[z], a.press[z], a.q_hum[z], qall);
        double n_tot = q2abs(hydro_n[z * nhydro + h], a.temp[z], a.press[z], a.q_hum[z], qall);
        double r_eff = hydro_reff[z * nhydro + h];
        if (s.moment_in == 13 && (q_h < st->hydro_threshold || n_tot <= 1.)) continue;
        if ((q_h < st->hydro_threshold || std::isnan(q_h)) && (n_tot <= 0 || std::isnan(n_tot)) &&
            (r_eff <= 0 || std::isnan(r_eff)) && s.moment_in != 0)
          continue;
        pres = true;
        PSDIn in{s, q_h, n_tot, r_eff, a.temp[z], freq};
        Bins bn;
        if (run_psd(*st, in, bn) == 2) return 2;
        bool any = false;
        for (int i = 0; i < bn.nbin; i++) any |= (bn.n_ds[i] > 0);
        if (!any) continue;
        if (dbg && dbg->psd_d && fi == 0) {
          // src/hydrometeor_extinction.f90:303-309; area: src/drop_size_dist.f90:168-182
          const size_t po = ((size_t)z * nhydro + h) * dbg->psd_nbin;
          for (int i = 0; i < bn.nbin && i < dbg->psd_nbin; i++) {
            const double d = bn.d_ds[i];
            double area = -99.;
            if (s.alpha_as > 0. && s.beta_as > 0.) {
              area = s.alpha_as * std::pow(d, s.beta_as);
              if (s.liq_ice == -1 && st->hydro_limit_density_area && area > d * d) area = d * d;
            }
            dbg->psd_d[po + i] = d;
            dbg->psd_deltad[po + i] = bn.delta_d[i];
            dbg->psd_n[po + i] = bn.n_ds[i];
            dbg->psd_mass[po + i] = bn.mass[i];
            dbg->psd_area[po + i] = area;
          }
        }
        std::vector<double> ndens(bn.nbin);
        for (int i = 0; i < bn.nbin; i++) ndens[i] = bn.n_ds[i] / bn.delta_d[i];
        double refre, refim;
        if (s.liq_ice == 1) {  // 273.15 is default REAL (scatProperties.f90:227)
          if (ref_water_mod(st->liq_mod, a.temp[z] - F(273.15f), freq, refre, refim)) return 2;
        } else {
          ref_ice(a.temp[z], freq, refre, refim);
        }
        if (scat_code && scat_code[h] == 1) {
          // every bin with the species' aspect ratio and canting
          if (add_tmatrix(s, bn, ndens, refre, refim, std::vector<double>(bn.nbin, s.as_ratio),
                          std::vector<double>(bn.nbin, canting ? canting[h] : 0.0)))
            return 2;
          continue;
        }
        MieOut mo;
        if (calc_mie_spheres(*st, freq * 1e9, s.liq_ice, bn, ndens, refre, refim, mo)) return 2;
        save_bscat(z, h, mo, ndens);
        nlegen_coef = std::max(nlegen_coef, mo.nlegen);
        kexttot = kexttot + mo.kext;
        backtot = backtot + mo.back;  // rt_back (scatProperties.f90:922)
        if (kexttot == 0.0) salbedo = 0.0;
        else salbedo = salbedo + (mo.salb * mo.kext);
        if (nlegen_coef > 0)
          for (int jj = 0; jj < nlegen_coef; jj++)
            for (int k = 0; k < 3; k++) legen_coef[k][jj] = legen_coef[k][jj] + (mo.legen[k][jj] * mo.salb * mo.kext);
        if (kexttot < 0.0 || std::isnan(kexttot)) return 2;
        if (nlegen_coef > MAXNLEG - 1) return 2;
      }
      kext_h[z] = kexttot;
      back_h[z] = backtot;
      // finalize_rt3_scatProperties
      salbedo = salbedo / kexttot;
      for (int k = 0; k < 3; k++)
        for (int jj = 0; jj < MAXNLEG; jj++) legen_coef[k][jj] = legen_coef[k][jj] / (salbedo * kexttot);
      if (fi == 0) present[z] = pres;
      scat[z].assign((size_t)4 * n * n, 0.0);
      if (nlegen_coef > 0) scatcnv(N, nlegen_coef, legen_coef, kexttot, salbedo, scat[z], extk[z], emk[z]);
      // rt_* = (T-matrix species) + scatcnv (src/hydrometeor_extinction.f90:337-342)
      if (!tm_scat[z].empty())
        for (size_t e = 0; e < scat[z].size(); e++) scat[z][e] = tm_scat[z][e] + scat[z][e];
      if (!st->lhyd_scattering) std::fill(scat[z].begin(), scat[z].end(), 0.0);
      if (!st->lhyd_emission) {
        emk[z] = 0.0;
        std::fill(tm_emis[z].begin(), tm_emis[z].end(), 0.0);
      }
      if (dbg) {
        size_t o = (size_t)fi * L + z;
        if (dbg->kexttot) dbg->kexttot[o] = kexttot;
        if (dbg->salbedo) dbg->salbedo[o] = salbedo;
        if (dbg->nlegen) dbg->nlegen[o] = nlegen_coef;
        if (dbg->legen)
          for (int k = 0; k < 3; k++)
            for (int jj = 0; jj < MAXNLEG; jj++) dbg->legen[(o * 3 + k) * MAXNLEG + jj] = legen_coef[k][jj];
        if (dbg->scatter_matrix)
          std::copy(scat[z].begin(), scat[z].end(), dbg->scatter_matrix + o * 4 * n * n);
        if (dbg->ext) dbg->ext[o] = extk[z];
        if (dbg->emis) dbg->emis[o] = emk[z];
        if (dbg->kextatmo) dbg->kextatmo[o] = kgas[z];
      }
    }
    if (dbg && dbg->present && fi == 0)
      for (int z = 0; z < L; z++) dbg->present[z] = present[z];
    if (dbg && st->active) {
      std::vector<double> ze, ath, ata;
      radar_simple(*st, L, freq, a.hgt_lev, present, kext_h, back_h, kgas, ze, ath, ata);
      for (int z = 0; z < L; z++) {
        size_t o = (size_t)fi * L + z;
        if (dbg->back) dbg->back[o] = back_h[z];
        if (dbg->ze) dbg->ze[o] = ze[z];
        if (dbg->att_hydro) dbg->att_hydro[o] = ath[z];
        if (dbg->att_atmo) dbg->att_atmo[o] = ata[z];
      }
    }

    // rt4: flip to top-down (src/rt4.f90:274-305) and radtran4
    std::vector<Layer> lay(L + 1);
    for (int layer = 0; layer < L; layer++) {
      int z = L - 1 - layer;  // bottom-up index
      double h0 = a.hgt_lev[L - layer], h1 = a.hgt_lev[L - layer - 1];
      double t0 = a.temp_lev[L - layer], t1 = a.temp_lev[L - layer - 1];
      double zdiff = std::fabs(h0 - h1);
      double gas = std::max(kgas[z], 0.0);
      if (present[z]) {
        // CHECK_NORM4 (src/radscat4.f90:87-136)
        const double* Q = scat[z].data();
        double maxsum = 0.0;
        for (int j1 = 0; j1 < N; j1++)
          for (int l = 1; l <= 2; l++) {
            double sum = ((l == 1 || l == 2) ? emk[z] : 0.0) - extk[z];
            if (!tm_ext[z].empty())  // EMIS_VECTOR(1,J1,L) - EXTINCT_MATRIX(1,1,J1,L)
              sum = (tm_emis[z][0 + 2 * j1] + emk[z]) - (tm_ext[z][0 + 2 * (0 + 2 * j1)] + extk[z]);
            for (int j2 = 0; j2 < N; j2++) {
              size_t qi = (size_t)(0 + 2 * j2) * n + (0 + 2 * j1);
              sum = sum + 2.0 * 3.1415926535897932384 * qw[j2] *
                              (Q[(size_t)(l - 1) * n * n + qi] + Q[(size_t)(l + 1) * n * n + qi]);
            }
            maxsum = std::max(maxsum, std::fabs(sum));
          }
        if (maxsum > 5.0e-4) return 2;
      }
      double planck1 = planck(t1, wl), planck0 = planck(t0, wl);
      int nd = -1;
      if (!present[z]) nonscatter_layer(N, mu, zdiff * gas, planck0, planck1, lay[layer]);
      else
        scattering_layer(N, mu, qw, zdiff, gas, planck0, planck1, scat[z], extk[z], emk[z], lay[layer], nd,
                         tm_ext[z].empty() ? nullptr : tm_ext[z].data(),
                         tm_emis[z].empty() ? nullptr : tm_emis[z].data());
      if (dbg && dbg->num_doubles) dbg->num_doubles[(size_t)fi * L + z] = nd;
    }
    // surface (src/sfc_matrices.f90, default emissivity branch sfc_optics.f90:79-81)
    const double e = st->emissivity, rr = 1.0 - e;
    Layer& sf = lay[L];
    sf.R.assign((size_t)2 * n * n, 0.0);
    sf.T.assign((size_t)2 * n * n, 0.0);
    sf.S.assign(2 * n, 0.0);
    for (int r = 0; r < n; r++) { sf.T[r + (size_t)n * r] = 1.0; sf.T[n * n + r + (size_t)n * r] = 1.0; }
    double pg = planck(a.groundtemp, wl);
    std::vector<double> gnd(n, 0.0), sky(2 * n, 0.0);
    if (sfc_refl == 'S' || sfc_refl == 'F') {
      for (int j = 0; j < N; j++) {
        double r1 = (rr + rr) / 2.0, r2 = (rr - rr) / 2.0;
        int r0 = 0 + 2 * j, q1 = 1 + 2 * j;
        double* R2 = &sf.R[n * n];
        R2[r0 + (size_t)n * r0] = r1;
        R2[r0 + (size_t)n * q1] = r2;
        R2[q1 + (size_t)n * r0] = r2;
        R2[q1 + (size_t)n * q1] = r1;
        gnd[r0] = (1.0 - r1) * pg;
        gnd[q1] = -r2 * pg;
      }
    } else if (sfc_refl == 'L') {
      for (int j1 = 0; j1 < N; j1++)
        for (int j2 = 0; j2 < N; j2++)
          sf.R[n * n + (0 + 2 * j1) + (size_t)n * (0 + 2 * j2)] = 2.0 * rr * mu[j2] * qw[j2];
      for (int j = 0; j < N; j++) gnd[0 + 2 * j] = e * pg;
    } else {
      return 1;
    }
    if (emissivity_out)
      for (int i = 0; i < 2; i++)
        for (int j = 0; j < N; j++) emissivity_out[(i * nfreq + fi) * N + j] = e;
    double psky = planck(SKY_TEMP, wl);
    for (int j = 0; j < N; j++) { sky[0 + 2 * j] = (1.0 - 0.0) * psky; sky[n + 0 + 2 * j] = (1.0 - 0.0) * psky; }

    // output levels (src/radtran4.f90:375-422)
    for (int io = 0; io < noutlevels; io++) {
      int layer = std::min(std::max(outlev[io], 1), L + 2);
      Layer up, dn;
      up.R.assign((size_t)2 * n * n, 0.0);
      up.T.assign((size_t)2 * n * n, 0.0);
      up.S.assign(2 * n, 0.0);
      for (int r = 0; r < n; r++) { up.T[r + (size_t)n * r] = 1.0; up.T[n * n + r + (size_t)n * r] = 1.0; }
      dn = up;
      for (int l = 1; l <= layer - 1; l++) {
        if (l == 1) up = lay[0];
        else combine(n, Layer(up), lay[l - 1], up);
      }
      for (int l = layer; l <= L + 1; l++) {
        if (l == layer) dn = lay[l - 1];
        else combine(n, Layer(dn), lay[l - 1], dn);
      }
      std::vector<double> uprad(n), dnrad(n);
      internal_radiance(n, up, dn, sky.data(), gnd.data(), uprad.data(), dnrad.data());
      // collect_output + CONVERT_OUTPUT (VH, 'T')
      for (int j = 0; j < N; j++) {
        double u[2] = {uprad[0 + 2 * j], uprad[1 + 2 * j]}, d[2] = {dnrad[0 + 2 * j], dnrad[1 + 2 * j]};
        if (st->outpol_vh) {
          double iv = 0.5 * (u[0] + u[1]), ih = 0.5 * (u[0] - u[1]);
          u[0] = iv; u[1] = ih;
          iv = 0.5 * (d[0] + d[1]); ih = 0.5 * (d[0] - d[1]);
          d[0] = iv; d[1] = ih;
        }
        for (int i = 0; i < 2; i++) {
          double ru = u[i], rd = d[i];
          if (st->outpol_vh) { ru = 2.0 * ru; rd = 2.0 * rd; }
          double tu = rad_to_tb(ru, wl), td = rad_to_tb(rd, wl);
          tb[(((size_t)io * n + (N - 1 - j)) * nfreq + fi) * 2 + i] = tu;
          tb[(((size_t)io * n + (N + j)) * nfreq + fi) * 2 + i] = td;
        }
      }
    }
  }
  return 0;
}

}  // extern "C"
