// Column pre-processing, gas absorption, particle size distributions and
// the compaction of hydrometeor-bearing layers.
#pragma once
#include "common.cuh"
#include "work.cuh"

namespace pb {

// ---------------------------------------------------------------- atmosphere
// src/e_sat_gg_water.f90:1-21 (all constants default REAL)
__device__ double e_sat_gg_water(double T) {
  const double a = F(1013.246f), b = F(7.90298f), t0 = F(373.16f), c = F(5.02808f), d = F(1.3816e-7f),
               e = F(11.344f), g = F(8.1328e-3f), h = F(3.49149f);
  double ex = -(b * (t0 / T - 1)) + c * log10(t0 / T) - d * (pow(10.0, e * (1 - T / t0)) - 1) +
              g * (pow(10.0, -(h * (t0 / T - 1))) - 1);
  return a * pow(10.0, ex);
}

// One thread per column: src/vars_atmosphere.f90:671-901
// (fillMissing_atmosphere_vars) and the output-level search of
// src/run_rt.f90:166-184.
__global__ void k_atmo(Batch b, Work w) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= b.ncol) return;
  const int Lm = b.max_nlyrs, L = b.nlyrs[c];
  const double* ihl = b.hgt_lev + (size_t)c * (Lm + 1);
  const double* itl = b.temp_lev + (size_t)c * (Lm + 1);
  const double* ipl = b.press_lev + (size_t)c * (Lm + 1);
  const double* irl = b.relhum_lev + (size_t)c * (Lm + 1);
  const double* ih = b.hgt + (size_t)c * Lm;
  const double* it = b.temp + (size_t)c * Lm;
  const double* ip = b.press + (size_t)c * Lm;
  const double* ir = b.relhum + (size_t)c * Lm;
  double* hl = w.hgt_lev + (size_t)c * (Lm + 1);
  double* tl = w.temp_lev + (size_t)c * (Lm + 1);
  double* t = w.temp + (size_t)c * Lm;
  double* p = w.press + (size_t)c * Lm;
  double* rv = w.rho_vap + (size_t)c * Lm;
  double* qh = w.q_hum + (size_t)c * Lm;
  // A column whose quadrature is not 8, 16 or 32, not among the launched
  // ones, or wider than the output rows is solved by no kernel: report it
  // on every frequency of the column instead of leaving -9999 silently.
  const int nm = b.col_nummu(c);
  const int nbit = (nm == 8) ? 1 : (nm == 16) ? 2 : (nm == 32) ? 4 : 0;
  const bool bad_l = L < 2 || L > Lm;
  if (bad_l || !(nbit & b.nummu_mask) || nm > b.max_nummu) {
    w.col_status[c] |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE;
    const int nf = min(b.col_nfreq(c), b.max_nfreq);
    for (int f = 0; f < nf; f++) w.status[(size_t)c * b.max_nfreq + f] |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE;
    if (bad_l) return;
  }
  // layer heights first (only needs levels), then the level variables
  // Use local copies: h, r, plev (the level pressure and humidity are only
  // needed to fill layer values).
  double h_[1];
  (void)h_;
  auto H = [&](int z) -> double { double v = ih[z]; return isnan(v) ? 0.5 * (ihl[z] + ihl[z + 1]) : v; };
  // levels
  auto HL = [&](int z) -> double {
    double v = ihl[z];
    if (!isnan(v)) return v;
    if (z == 0) return H(0) - (H(1) - H(0)) * 0.5;
    if (z == L) return H(L - 1) + (H(L - 1) - H(L - 2)) * 0.5;
    return 0.5 * (H(z) + H(z - 1));
  };
  auto TL = [&](int z) -> double {
    double v = itl[z];
    if (!isnan(v)) return v;
    if (z == 0) return it[0] - (it[1] - it[0]) / (H(1) - H(0)) * (H(0) - HL(0));
    if (z == L) return it[L - 1] + (it[L - 1] - it[L - 2]) / (H(L - 1) - H(L - 2)) * (HL(L) - H(L - 1));
    return 0.5 * (it[z] + it[z - 1]);
  };
  auto RL = [&](int z) -> double {
    double v = irl[z];
    if (!isnan(v)) return v;
    if (z == 0) return ir[0] - (ir[1] - ir[0]) / (H(1) - H(0)) * (H(0) - HL(0));
    if (z == L) return ir[L - 1] + (ir[L - 1] - ir[L - 2]) / (H(L - 1) - H(L - 2)) * (HL(L) - H(L - 1));
    return 0.5 * (ir[z] + ir[z - 1]);
  };
  auto PL = [&](int z) -> double {
    double v = ipl[z];
    if (!isnan(v)) return v;
    if (z == 0) return exp(log(ip[0]) - (log(ip[1]) - log(ip[0])) / (H(1) - H(0)) * (H(0) - HL(0)));
    if (z == L)
      return exp(log(ip[L - 1]) + (log(ip[L - 1]) - log(ip[L - 2])) / (H(L - 1) - H(L - 2)) * (HL(L) - H(L - 1)));
    return exp(0.5 * (log(ip[z]) + log(ip[z - 1])));
  };
  for (int z = 0; z <= L; z++) {
    hl[z] = HL(z);
    tl[z] = TL(z);
  }
  for (int z = 0; z < L; z++) {
    double tz = it[z];
    if (isnan(tz)) tz = 0.5 * (tl[z] + tl[z + 1]);
    double rz = ir[z];
    if (isnan(rz)) rz = 0.5 * (RL(z) + RL(z + 1));
    double pz = ip[z];
    if (isnan(pz)) pz = exp(0.5 * (log(PL(z)) + log(PL(z + 1))));
    t[z] = tz;
    p[z] = pz;
    double vp = rz * e_sat_gg_water(tz);
    w.vap[(size_t)c * Lm + z] = vp;
    rv[z] = vp / (tz * R_V);
    qh[z] = R_V / R_D * vp / (pz - (1.0 - R_V / R_D) * vp);
  }
  double g = b.groundtemp[c];
  w.gtemp[c] = isnan(g) ? tl[0] : g;
  // output levels
  for (int io = 0; io < b.noutlevels; io++) {
    double ob = b.obs_height[(size_t)c * b.noutlevels + io];
    int lev = 1;
    if (ob >= hl[L]) lev = 1;
    else if (ob <= hl[0]) lev = L + 1;
    else {
      for (int nz = 1; nz <= L; nz++)
        if (hl[nz] >= ob) {
          lev = (fabs(hl[nz] - ob) <= fabs(hl[nz - 1] - ob)) ? L - nz + 1 : L - nz + 2;
          break;
        }
    }
    w.outlev[(size_t)c * b.noutlevels + io] = lev;
  }
}

// ---------------------------------------------------------------- gas (R98)
__constant__ float c_o2_w300[40], c_o2_y300[40], c_o2_v[40], c_o2_f[40], c_o2_s300[40], c_o2_be[40];
__constant__ float c_h2o_fl[15], c_h2o_s1[15], c_h2o_b2[15], c_h2o_w3[15], c_h2o_x[15], c_h2o_ws[15],
    c_h2o_xs[15];

// src/gasabs_module.f90:83-333 (absn2, o2abs, abh2o) and
// src/rosen98_gasabs.f90:2-153; returns Np/m (get_gasabs.f90:95).
__device__ int gas_r98(double f, double T, double rhowv, double pres, double* kext) {
  if (f <= 0.0 || f > 800.0 || T <= 100.0 || pres <= 0.0 || pres > 1.2e5) {
    *kext = 0.0;
    return PAMTRA_B200_FATAL | PAMTRA_B200_ST_GAS;
  }
  const double pmb = pres / 100.0, vapden = rhowv * 1000.0;
  // absn2
  double th = 300.0 / T;
  double absn2 = 6.4e-14 * pmb * pmb * f * f * pow(th, 3.55);
  // o2abs
  double th1 = th - 1.0;
  double bb = pow(th, F(0.8f));
  double preswv = vapden * T / 217.0;
  double presda = pmb - preswv;
  double den = 0.001 * (presda * bb + 1.1 * preswv * th);
  double dfnr = F(0.56f) * den;
  double sum = 1.6e-17 * f * f * dfnr / (th * (f * f + dfnr * dfnr));
  for (int k = 0; k < 40; k++) {
    double fk = F(c_o2_f[k]);
    double df = F(c_o2_w300[k]) * den;
    double y = 0.001 * pmb * bb * (F(c_o2_y300[k]) + F(c_o2_v[k]) * th1);
    double str = F(c_o2_s300[k]) * exp(-(F(c_o2_be[k]) * th1));
    double sf1 = (df + (f - fk) * y) / (p2(f - fk) + df * df);
    double sf2 = (df - (f + fk) * y) / (p2(f + fk) + df * df);
    sum = sum + str * (sf1 + sf2) * p2(f / fk);
  }
  double o2 = 0.5034e12 * sum * presda * p3(th) / PI;
  // abh2o
  double h2o = 0.0;
  if (vapden > 0.0) {
    double pvap = vapden * T / 217.0;
    double pda = pmb - pvap;
    double den2 = 3.335e16 * vapden;
    double ti = 300.0 / T;
    double ti2 = pow(ti, 2.5);
    double con = (5.43e-10 * 1.105 * pda * p3(ti) + 1.8e-8 * 0.79 * pvap * pow(ti, 7.5)) * pvap * f * f;
    double s2 = 0.0;
    for (int i = 0; i < 15; i++) {
      double fl = F(c_h2o_fl[i]);
      double width = F(c_h2o_w3[i]) * pda * pow(ti, F(c_h2o_x[i])) + F(c_h2o_ws[i]) * pvap * pow(ti, F(c_h2o_xs[i]));
      double wsq = width * width;
      double s = F(c_h2o_s1[i]) * ti2 * exp(F(c_h2o_b2[i]) * (1.0 - ti));
      double base = width / (562500.0 + wsq);
      double res = 0.0;
      double d1 = f - fl, d2 = f + fl;
      if (fabs(d1) < 750.0) res = res + width / (p2(d1) + wsq) - base;
      if (fabs(d2) < 750.0) res = res + width / (p2(d2) + wsq) - base;
      s2 = s2 + s * res * p2(f / fl);
    }
    h2o = 0.3183e-4 * den2 * s2 + con;
  }
  *kext = (absn2 + o2 + h2o) / 1.0e3;
  return 0;
}

// ---------------------------------------------------------------- gas (MPM93)
// Line catalogue of Liebe, Hufford and Cotton (1993), as the reference holds
// it in REAL(4) (src/mpm93.f90:131-222): oxygen {f0 GHz, a1..a6}, water
// vapour {f0 GHz, b1..b6}.
__constant__ float c_l93_o2[44][7] = {
    {50.474239f, 0.094f, 9.694f, 0.890f, 0.000f, 0.240f, 0.790f},
    {50.987747f, 0.246f, 8.694f, 0.910f, 0.000f, 0.220f, 0.780f},
    {51.503349f, 0.608f, 7.744f, 0.940f, 0.000f, 0.197f, 0.774f},
    {52.021412f, 1.414f, 6.844f, 0.970f, 0.000f, 0.166f, 0.764f},
    {52.542393f, 3.102f, 6.004f, 0.990f, 0.000f, 0.136f, 0.751f},
    {53.066906f, 6.410f, 5.224f, 1.020f, 0.000f, 0.131f, 0.714f},
    {53.595749f, 12.470f, 4.484f, 1.050f, 0.000f, 0.230f, 0.584f},
    {54.130001f, 22.800f, 3.814f, 1.070f, 0.000f, 0.335f, 0.431f},
    {54.671158f, 39.180f, 3.194f, 1.100f, 0.000f, 0.374f, 0.305f},
    {55.221367f, 63.160f, 2.624f, 1.130f, 0.000f, 0.258f, 0.339f},
    {55.783802f, 95.350f, 2.119f, 1.170f, 0.000f, -0.166f, 0.705f},
    {56.264774f, 54.890f, 0.015f, 1.730f, 0.000f, 0.390f, -0.113f},
    {56.363388f, 134.400f, 1.660f, 1.200f, 0.000f, -0.297f, 0.753f},
    {56.968204f, 176.300f, 1.260f, 1.240f, 0.000f, -0.416f, 0.742f},
    {57.612484f, 214.100f, 0.915f, 1.280f, 0.000f, -0.613f, 0.697f},
    {58.323875f, 238.600f, 0.626f, 1.330f, 0.000f, -0.205f, 0.051f},
    {58.446590f, 145.700f, 0.084f, 1.520f, 0.000f, 0.748f, -0.146f},
    {59.164207f, 240.400f, 0.391f, 1.390f, 0.000f, -0.722f, 0.266f},
    {59.590984f, 211.200f, 0.212f, 1.430f, 0.000f, 0.765f, -0.090f},
    {60.306061f, 212.400f, 0.212f, 1.450f, 0.000f, -0.705f, 0.081f},
    {60.434776f, 246.100f, 0.391f, 1.360f, 0.000f, 0.697f, -0.324f},
    {61.150558f, 250.400f, 0.626f, 1.310f, 0.000f, 0.104f, -0.067f},
    {61.800156f, 229.800f, 0.915f, 1.270f, 0.000f, 0.570f, -0.761f},
    {62.411217f, 193.300f, 1.260f, 1.230f, 0.000f, 0.360f, -0.777f},
    {62.486259f, 151.700f, 0.083f, 1.540f, 0.000f, -0.498f, 0.097f},
    {62.997978f, 150.300f, 1.665f, 1.200f, 0.000f, 0.239f, -0.768f},
    {63.568520f, 108.700f, 2.115f, 1.170f, 0.000f, 0.108f, -0.706f},
    {64.127769f, 73.350f, 2.620f, 1.130f, 0.000f, -0.311f, -0.332f},
    {64.678902f, 46.350f, 3.195f, 1.100f, 0.000f, -0.421f, -0.298f},
    {65.224068f, 27.480f, 3.815f, 1.070f, 0.000f, -0.375f, -0.423f},
    {65.764771f, 15.300f, 4.485f, 1.050f, 0.000f, -0.267f, -0.575f},
    {66.302094f, 8.009f, 5.225f, 1.020f, 0.000f, -0.168f, -0.700f},
    {66.836830f, 3.946f, 6.005f, 0.990f, 0.000f, -0.169f, -0.735f},
    {67.369598f, 1.832f, 6.845f, 0.970f, 0.000f, -0.200f, -0.744f},
    {67.900864f, 0.801f, 7.745f, 0.940f, 0.000f, -0.228f, -0.753f},
    {68.431007f, 0.330f, 8.695f, 0.920f, 0.000f, -0.240f, -0.760f},
    {68.960312f, 0.128f, 9.695f, 0.900f, 0.000f, -0.250f, -0.765f},
    {118.750343f, 94.500f, 0.009f, 1.630f, 0.000f, -0.036f, 0.009f},
    {368.498352f, 6.790f, 0.049f, 1.920f, 0.600f, 0.000f, 0.000f},
    {424.763123f, 63.800f, 0.044f, 1.930f, 0.600f, 0.000f, 0.000f},
    {487.249359f, 23.500f, 0.049f, 1.920f, 0.600f, 0.000f, 0.000f},
    {715.393127f, 9.960f, 0.145f, 1.810f, 0.600f, 0.000f, 0.000f},
    {773.839661f, 67.100f, 0.130f, 1.820f, 0.600f, 0.000f, 0.000f},
    {834.145325f, 18.000f, 0.147f, 1.810f, 0.600f, 0.000f, 0.000f},
};
__constant__ float c_l93_h2o[35][7] = {
    {22.235081f, 0.01130f, 2.143f, 2.811f, 4.80f, 0.69f, 1.00f},
    {67.803963f, 0.00012f, 8.735f, 2.858f, 4.93f, 0.69f, 0.82f},
    {119.995941f, 0.00008f, 8.356f, 2.948f, 4.78f, 0.70f, 0.79f},
    {183.310089f, 0.24200f, 0.668f, 3.050f, 5.30f, 0.64f, 0.85f},
    {321.225647f, 0.00483f, 6.181f, 2.303f, 4.69f, 0.67f, 0.54f},
    {325.152924f, 0.14990f, 1.540f, 2.783f, 4.85f, 0.68f, 0.74f},
    {336.222595f, 0.00011f, 9.829f, 2.693f, 4.74f, 0.69f, 0.61f},
    {380.197357f, 1.15200f, 1.048f, 2.873f, 5.38f, 0.54f, 0.89f},
    {390.134521f, 0.00046f, 7.350f, 2.152f, 4.81f, 0.63f, 0.55f},
    {437.346680f, 0.00650f, 5.050f, 1.845f, 4.23f, 0.60f, 0.48f},
    {439.150818f, 0.09218f, 3.596f, 2.100f, 4.29f, 0.63f, 0.52f},
    {443.018280f, 0.01976f, 5.050f, 1.860f, 4.23f, 0.60f, 0.50f},
    {448.001068f, 1.03200f, 1.405f, 2.632f, 4.84f, 0.66f, 0.67f},
    {470.888947f, 0.03297f, 3.599f, 2.152f, 4.57f, 0.66f, 0.65f},
    {474.689117f, 0.12620f, 2.381f, 2.355f, 4.65f, 0.65f, 0.64f},
    {488.491119f, 0.02520f, 2.853f, 2.602f, 5.04f, 0.69f, 0.72f},
    {503.568542f, 0.00390f, 6.733f, 1.612f, 3.98f, 0.61f, 0.43f},
    {504.482697f, 0.00130f, 6.733f, 1.612f, 4.01f, 0.61f, 0.45f},
    {547.676453f, 0.97010f, 0.114f, 2.600f, 4.50f, 0.70f, 1.00f},
    {552.020935f, 1.47700f, 0.114f, 2.600f, 4.50f, 0.70f, 1.00f},
    {556.935974f, 48.74000f, 0.159f, 3.210f, 4.11f, 0.69f, 1.00f},
    {620.700806f, 0.50120f, 2.200f, 2.438f, 4.68f, 0.71f, 0.68f},
    {645.866150f, 0.00713f, 8.580f, 1.800f, 4.00f, 0.60f, 0.50f},
    {658.005310f, 0.03022f, 7.820f, 3.210f, 4.14f, 0.69f, 1.00f},
    {752.033203f, 23.96000f, 0.396f, 3.060f, 4.09f, 0.68f, 0.84f},
    {841.053955f, 0.00140f, 8.180f, 1.590f, 5.76f, 0.33f, 0.45f},
    {859.962341f, 0.01472f, 7.989f, 3.060f, 4.09f, 0.68f, 0.84f},
    {899.306702f, 0.00605f, 7.917f, 2.985f, 4.53f, 0.68f, 0.90f},
    {902.616150f, 0.00426f, 8.432f, 2.865f, 5.10f, 0.70f, 0.95f},
    {906.207336f, 0.01876f, 5.111f, 2.408f, 4.70f, 0.70f, 0.53f},
    {916.171570f, 0.83400f, 1.442f, 2.670f, 4.78f, 0.70f, 0.78f},
    {923.118408f, 0.00869f, 10.220f, 2.900f, 5.00f, 0.70f, 0.80f},
    {970.315002f, 0.89720f, 1.920f, 2.550f, 4.94f, 0.64f, 0.67f},
    {987.926758f, 13.21000f, 0.258f, 2.985f, 4.55f, 0.68f, 0.90f},
    {1780.000000f, 2230.00000f, 0.952f, 17.620f, 30.50f, 2.00f, 5.00f},
};

struct cplxf {
  float re, im;
};
// Smith-style division in single precision, as gfortran emits it for
// COMPLEX(4) operands (-fcx-fortran-rules).
__device__ __forceinline__ cplxf cdivf(cplxf a, cplxf b) {
  float tr, ti, ratio, div;
  if (fabsf(b.re) < fabsf(b.im)) {
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

// Line shape term of src/mpm93.f90:269-270 / 300-301:
// f/f0 [CMPLX(1,-d)/CMPLX(f0-f,-g) - CMPLX(1,d)/CMPLX(f0+f,g)], where CMPLX
// without KIND makes each quotient single precision.
__device__ __forceinline__ cplx l93_shape(double f, double f0, double d, double g) {
  const cplxf q1 = cdivf({1.f, (float)(-d)}, {(float)(f0 - f), (float)(-g)});
  const cplxf q2 = cdivf({1.f, (float)d}, {(float)(f0 + f), (float)g});
  const double r = f / f0;
  return cmk(r * (double)(q1.re - q2.re), r * (double)(q1.im - q2.im));
}

// src/mpm93.f90 (gas_mod 'L93'): oxygen lines, dry-air continuum and water
// vapour pseudo-line continuum of Liebe's MPM93 with the cloud term at
// W = 0, as src/get_gasabs.f90:78-86 calls it (pressure and vapour pressure
// in Pa, T in K); returns Np/m.
__device__ double gas_l93(double freq, double press, double vap, double T) {
  const double Tc = T - 273.15;
  const double V = 300.0 / (Tc + 273.15);
  double Pb = 10.0 * (press / 1.e3);
  const double E = 10.0 * (vap / 1.e3);
  double P = Pb - E;
  if (P < 0) {
    P = 0.0;
    Pb = E;
  }
  const double V08 = pow(V, (double)0.8f), V3 = (V * V) * V, V35 = pow(V, 3.5);
  double zr = 0.0, zi = 0.0;
  for (int i = 0; i < 44; i++) {
    const float* a = c_l93_o2[i];
    const double f0 = a[0];
    const double S = (double)a[1] * P * V3 * exp((double)a[2] * (1.0 - V)) * 1.e-6;
    double g = (double)a[3] * (P * pow(V, 0.8 - (double)a[4]) + 1.1 * E * V) * 1.e-3;
    g = pow(g * g + (25.0 * 0.6e-4) * (25.0 * 0.6e-4), (double)0.5f);
    const double d = ((double)a[5] + (double)a[6] * V) * (P + E) * V08 * 1.e-3;
    const cplx zf = l93_shape(freq, f0, d, g);
    zr = zr + S * zf.re;
    zi = zi + S * zf.im;
  }
  double at1 = 0.182 * freq * zi;
  if (at1 < 0.) at1 = 0.0;
  // dry air continuum
  const double So = 6.14e-5 * P * (V * V);
  const double gamo = 0.56e-3 * (P + E) * V08;
  const cplx zfo = cdiv(cmk(-freq, 0.0), cmk((double)(float)freq, (double)(float)gamo));
  const double Sn = 1.40e-12 * (P * P) * V35;
  const double zfn = (double)(float)(freq / (1.93e-5 * pow(freq, (double)1.5f) + 1.0));
  const double at2 = 0.182 * freq * (So * zfo.im + Sn * zfn);
  // water vapour
  zr = 0.0;
  zi = 0.0;
  for (int i = 0; i < 35; i++) {
    const float* b = c_l93_h2o[i];
    const double f0 = b[0];
    const double S = (double)b[1] * E * V35 * exp((double)b[2] * (1.0 - V));
    double gh = (double)b[3] * (P * pow(V, (double)b[5]) + (double)b[4] * E * pow(V, (double)b[6])) * 1.e-3;
    const double fd = (double)1.46f * f0;
    const double gd2 = 1.e-12 / V * (fd * fd);
    gh = 0.535 * gh + pow(0.217 * (gh * gh) + gd2, (double)0.5f);
    const cplx zf = l93_shape(freq, f0, 0.0, gh);
    zr = zr + S * zf.re;
    zi = zi + S * zf.im;
  }
  const double at3 = 0.182 * freq * zi;
  return 0.23026 * (at1 + at2 + at3) / 1.e3;
}

// one thread per (column, frequency, layer)
__global__ void k_gas(Batch b, Work w, int lgas, int gas_mod) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq;
  if (idx >= (size_t)b.ncol * Fm * Lm) return;
  const int z = idx % Lm;
  const int f = (idx / Lm) % Fm;
  const int c = idx / ((size_t)Lm * Fm);
  double k = 0.0;
  if (z < b.nlyrs[c] && f < b.col_nfreq(c) && lgas) {
    const size_t lz = (size_t)c * Lm + z;
    if (gas_mod == PAMTRA_B200_GAS_L93) {
      k = gas_l93(b.freq(c, f), w.press[lz], w.vap[lz], w.temp[lz]);
    } else {
      int st = gas_r98(b.freq(c, f), w.temp[lz], w.rho_vap[lz], w.press[lz], &k);
      if (st) atomicOr(&w.status[(size_t)c * Fm + f], st);
    }
  }
  w.kgas[idx] = k;
}


// ---------------------------------------------------------------- PSD
__device__ __forceinline__ double q2abs(double spec, double t, double p, double qv, double qall) {
  return spec * p / (R_D * (1.0 + (R_V / R_D - 1.0) * qv - qall) * t);
}

struct DistPar {
  double n_0, lambda, gam, mu, n_t, sig, d_ln, d_mono;
};

// src/make_mass_size.f90 -> returns 0 ok / 2 fatal
__device__ int make_mass_size(const pamtra_b200_species& s, double& a_ms, double& b_ms) {
  a_ms = s.a_ms;
  b_ms = s.b_ms;
  const double rho = s.rho_ms, asr = s.as_ratio;
  const int li = s.liq_ice;
  if (b_ms > 3.5 || a_ms == 0.0 || rho == 0.0 || asr == 0.0) return 2;
  if (li == -1 && rho > 917.0) return 2;
  if (li == 1 && (a_ms > 0.0 || b_ms > 0.0 || rho > 0.0 || (asr != 1.0 && asr > 0.0))) {
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
  if (li == -1 && (asr < 0.0 || asr == 1.0)) { b_ms = 3.0; a_ms = PI / 6.0 * rho; return 0; }
  if (li == -1 && asr > 1.0) { b_ms = 3.0; a_ms = PI / 6.0 * rho * pow(1.0 / asr, 2.0); return 0; }
  if (li == -1 && asr > 0.0 && asr < 1.0) { b_ms = 3.0; a_ms = PI / 6.0 * rho * asr; return 0; }
  return 2;
}

// src/make_dist_param.f90 (exp, exp_field_t, exp_ryan, mgamma, mono, logn)
__device__ int make_dist_params(const pamtra_b200_species& s, double q_h, double n_tot, double r_eff, double layer_t,
                                double a_ms, double b_ms, DistPar& dp) {
  const double NaN = __longlong_as_double(0x7ff8000000000000ULL);
  dp.n_0 = -99; dp.lambda = -99; dp.gam = NaN; dp.mu = NaN; dp.n_t = -99; dp.sig = -99; dp.d_ln = NaN; dp.d_mono = -99;
  const int mi = s.moment_in;
  const double p_1 = s.p_1, p_2 = s.p_2, p_3 = s.p_3, p_4 = s.p_4, d_1 = s.d_1;
  if (mi == 3 && q_h <= 0.) return 2;
  if (mi == 1 && n_tot <= 0.) return 2;
  if (mi == 2 && r_eff <= 0.) return 2;
  if (mi == 13 && (q_h <= 0. || n_tot <= 0.)) return 2;
  if (mi == 23 && (q_h <= 0. || r_eff <= 0.)) return 2;
  if (mi == 12 && (n_tot <= 0. || r_eff <= 0.)) return 2;
  const int dist = s.dist;
  if (dist == PAMTRA_B200_DIST_MONO) {
    dp.lambda = 0; dp.mu = 0; dp.gam = 0;
    if (d_1 != -99. && p_1 == -99.) {
      dp.d_mono = d_1;
      if (mi == 3) dp.n_0 = q_h / (DELTA_D_MONO * a_ms * pow(d_1, b_ms));
      if (mi == 1) dp.n_0 = n_tot / DELTA_D_MONO;
    }
    if (p_1 != -99. && d_1 == -99.) {
      dp.n_0 = p_1 / DELTA_D_MONO;
      if (mi == 3) dp.d_mono = pow(q_h / (p_1 * a_ms), 1.0 / b_ms);
      if (mi == 2) dp.d_mono = r_eff * 2.0;
    }
    if (mi == 23) {
      dp.d_mono = r_eff * 2.0;
      dp.n_0 = q_h / (DELTA_D_MONO * a_ms * pow(dp.d_mono, b_ms));
    }
    return (dp.n_0 <= 0.0 || dp.d_mono <= 0.0) ? 2 : 0;
  }
  if (dist == PAMTRA_B200_DIST_EXP || dist == PAMTRA_B200_DIST_EXP_FIELD_T || dist == PAMTRA_B200_DIST_EXP_RYAN) {
    dp.gam = 1.0;
    dp.mu = 0.0;
    const double gb = tgamma(b_ms + 1.0);
    if (dist == PAMTRA_B200_DIST_EXP) {
      if (p_1 != -99. && p_2 != -99. && mi == 0) { dp.lambda = p_1; dp.n_0 = p_2; }
      if (p_1 != -99. && p_2 != -99. && mi == 3) {
        dp.lambda = pow(p_1 * a_ms * gb / q_h, 1.0 / (b_ms + 1 - p_2));
        dp.n_0 = p_1 * pow(dp.lambda, p_2);
      }
      if (p_1 != -99. && p_2 == -99. && p_3 == -99.) {
        if (mi == 3) dp.lambda = pow(p_1 * a_ms * gb / q_h, 1.0 / b_ms);
        if (mi == 2) dp.lambda = 3.0 / r_eff;
        dp.n_0 = p_1 * dp.lambda;
      }
      if (p_1 == -99. && p_2 != -99. && p_3 == -99.) {
        dp.lambda = 3.0 / p_2;
        if (mi == 3) dp.n_0 = (q_h * pow(dp.lambda, b_ms + 1.0)) / (a_ms * gb);
        if (mi == 1) dp.n_0 = n_tot * dp.lambda;
      }
      if (p_1 == -99. && p_2 == -99. && p_3 != -99.) {
        dp.n_0 = p_3;
        if (mi == 3) dp.lambda = pow(dp.n_0 * a_ms * gb / q_h, 1.0 / (b_ms + 1.0));
        if (mi == 1) dp.lambda = dp.n_0 / n_tot;
        if (mi == 2) dp.lambda = 3.0 / r_eff;
      }
      if (p_1 == -99. && p_2 == -99.) {
        if (mi == 13) { dp.lambda = pow(n_tot * a_ms * gb / q_h, 1.0 / b_ms); dp.n_0 = n_tot * dp.lambda; }
        if (mi == 23) { dp.lambda = 3.0 / r_eff; dp.n_0 = (q_h * pow(dp.lambda, b_ms + 1)) / (a_ms * gb); }
        if (mi == 12) { dp.lambda = 3.0 / r_eff; dp.n_0 = n_tot * dp.lambda; }
      }
    }
    if (dist == PAMTRA_B200_DIST_EXP_RYAN) {
      dp.lambda = 1220.0 * pow(10.0, -0.0245 * (273.15 - layer_t));
      if (mi == 3) dp.n_0 = (q_h * pow(dp.lambda, b_ms + 1)) / (a_ms * gb);
      if (mi == 1) dp.n_0 = n_tot * dp.lambda;
    }
    if (dist == PAMTRA_B200_DIST_EXP_FIELD_T) {
      dp.n_0 = 7.628e6 * exp(0.107 * (273.15 - layer_t));
      if (mi == 3) dp.lambda = pow(a_ms * dp.n_0 * gb / q_h, 1.0 / (b_ms + 1.0));
      if (mi == 2) dp.lambda = 3.0 / r_eff;
    }
    return (dp.gam != 1.0 || dp.mu != 0.0 || dp.n_0 <= 0.0 || dp.lambda <= 0.0) ? 2 : 0;
  }
  if (dist == PAMTRA_B200_DIST_LOGN) {
    if (p_1 != -99. && p_3 != -99.) {
      dp.n_t = p_1;
      dp.sig = p_3;
      if (mi == 3) dp.d_ln = (1.0 / b_ms) * (log(q_h / (a_ms * dp.n_t)) - (0.5 * pow(b_ms * dp.sig, 2.0)));
      if (mi == 2) dp.d_ln = log(2.0 * r_eff) - 2.5 * pow(dp.sig, 2.0);
    }
    if (p_1 != -99. && p_2 != -99. && p_3 == -99. && mi == 3) {
      dp.n_t = p_1;
      double w1 = q_h / (a_ms * dp.n_t * pow(2.0 * p_2, 2.0));
      double w2 = 2.0 / (b_ms * (b_ms - 5.0));
      dp.sig = sqrt(log(w1) * w2);
      dp.d_ln = log(2.0 * p_2) - 2.5 * pow(dp.sig, 2.0);
    }
    if (p_1 == -99. && p_2 != -99. && p_3 != -99.) {
      dp.sig = p_3;
      dp.d_ln = log(2.0 * p_2) - 2.5 * pow(dp.sig, 2.0);
      if (mi == 3) dp.n_t = q_h / a_ms * exp(-1.0 * ((b_ms * dp.d_ln) + (0.5 * pow(b_ms * dp.sig, 2.0))));
      if (mi == 1) dp.n_t = n_tot;
    }
    return (dp.n_t <= 0.0 || isnan(dp.d_ln) || dp.sig <= 0.0) ? 2 : 0;
  }
  if (dist == PAMTRA_B200_DIST_MGAMMA) {
    if (p_3 == -99. || p_4 == -99.) return 2;
    const double mu = p_3, gam = p_4;
    dp.mu = mu;
    dp.gam = gam;
    if (p_1 != -99. && p_2 == -99.) {
      if (mi == 3) {
        double w2 = tgamma((mu + b_ms + 1.0) / gam), w3 = tgamma((mu + 1.0) / gam);
        dp.lambda = pow(a_ms / q_h * p_1 * w2 / w3, gam / b_ms);
        dp.n_0 = gam * p_1 / w3 * pow(dp.lambda, (mu + 1.0) / gam);
      }
      if (mi == 2) {
        double w1 = tgamma((mu + 4.0) / gam), w2 = tgamma((mu + 3.0) / gam) * r_eff * 2.0;
        dp.lambda = pow(w1 / w2, gam);
        w1 = (mu + 1.0) / gam;
        dp.n_0 = p_1 * gam * pow(dp.lambda, w1) / tgamma(w1);
      }
    }
    if (p_1 == -99. && p_2 != -99.) {
      if (mi == 3) {
        double w1 = tgamma((mu + 4.0) / gam), w2 = tgamma((mu + 3.0) / gam) * p_2 * 2.0;
        dp.lambda = pow(w1 / w2, gam);
        w1 = q_h * gam / a_ms;
        w2 = (mu + b_ms + 1.0) / gam;
        dp.n_0 = w1 * pow(dp.lambda, w2) / tgamma(w2);
      }
      if (mi == 1) {
        double w1 = tgamma((mu + 4.0) / gam), w2 = tgamma((mu + 3.0) / gam) * p_2 * 2.0;
        dp.lambda = pow(w1 / w2, gam);
        w1 = (mu + 1.0) / gam;
        dp.n_0 = n_tot * gam * pow(dp.lambda, w1) / tgamma(w1);
      }
    }
    if (p_1 == -99. && p_2 == -99.) {
      if (mi == 13) {
        double w2 = tgamma((mu + b_ms + 1.0) / gam), w3 = tgamma((mu + 1.0) / gam);
        dp.lambda = pow(a_ms / q_h * n_tot * w2 / w3, gam / b_ms);
        dp.n_0 = gam * n_tot / w3 * pow(dp.lambda, (mu + 1.0) / gam);
      }
      if (mi == 23) {
        double w1 = tgamma((mu + 4.0) / gam), w2 = tgamma((mu + 3.0) / gam) * r_eff * 2.0;
        dp.lambda = pow(w1 / w2, gam);
        w1 = q_h * gam / a_ms;
        w2 = (mu + b_ms + 1.0) / gam;
        dp.n_0 = w1 * pow(dp.lambda, w2) / tgamma(w2);
      }
      if (mi == 12) {
        double w1 = tgamma((mu + 4.0) / gam), w2 = tgamma((mu + 3.0) / gam) * r_eff * 2.0;
        dp.lambda = pow(w1 / w2, gam);
        w1 = (mu + 1.0) / gam;
        dp.n_0 = n_tot * gam * pow(dp.lambda, w1) / tgamma(w1);
      }
    }
    return (dp.lambda <= 0.0 || dp.n_0 <= 0.0 || isnan(mu) || isnan(gam)) ? 2 : 0;
  }
  return 2;
}

__device__ __forceinline__ double fdist(int dist, const DistPar& dp, double d) {
  if (dist == PAMTRA_B200_DIST_LOGN)
    return dp.n_t / (d * dp.sig * sqrt(2.0 * PI)) * exp(-(p2(log(d) - dp.d_ln)) / (2.0 * p2(dp.sig)));
  return dp.n_0 * pow(d, dp.mu) * exp(-dp.lambda * pow(d, dp.gam));
}

// Bin-boundary grid of src/make_dist.f90:104-259: a linear grid of nlin+1
// points and a log grid of nlog+1 points merged in ascending order (ties
// take the log point first), generated on the fly.
struct MergedGrid {
  double d1, w_lin, w_log, log_d1;
  int nlin, nlog, il, ig;
  __device__ void init(double d1w, double d2w, int nw) {
    nlin = (int)(nw / 2.0);
    nlog = (int)(nw / 2.0);
    if (nlin + nlog == nw) nlin = nlin - 1;
    d1 = d1w;
    w_lin = (d2w - d1w) / (nlin + 1);
    log_d1 = log(d1w);
    w_log = (log(d2w) - log_d1) / (nlog + 1);
    il = 1;
    ig = 1;
  }
  __device__ double next() {
    const double big = F(1.e30f);
    double vl = (il <= nlin + 1) ? d1 + w_lin * il : big;
    double vg = (ig <= nlog + 1) ? exp(w_log * (ig - 1) + log_d1) : big;
    if (vg <= vl) { ig++; return vg; }
    il++;
    return vl;
  }
};

// One thread per (column, layer, species) slot: presence test of
// src/hydrometeor_extinction.f90:246-283, then run_drop_size_dist
// (src/drop_size_dist.f90:107-218): make_mass_size, make_dist_params,
// make_dist (adaptive grid, trapezoid bins, mass rescaling), particle mass and
// make_soft_spheroid for ice.
__global__ void k_psd(Batch b, Work w, pamtra_b200_settings st) {
  const size_t s_idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int Lm = b.max_nlyrs, H = b.nhydro;
  if (s_idx >= (size_t)b.ncol * Lm * H) return;
  const int h = s_idx % H;
  const int z = (s_idx / H) % Lm;
  const int c = s_idx / ((size_t)H * Lm);
  w.slot_st[s_idx] = 0;
  w.slot_nb[s_idx] = 0;
  if (z >= b.nlyrs[c]) return;
  const pamtra_b200_species s = b.species_of(c, h);
  if (s.dist == PAMTRA_B200_DIST_DISABLED) return;
  const size_t lz = (size_t)c * Lm + z;
  const double T = w.temp[lz], P = w.press[lz], qv = w.q_hum[lz];
  double qsum = 0.0;
  for (int k = 0; k < H; k++) qsum += b.hydro_q[lz * H + k];
  const double qall = (st.hydro_includehydroinrhoair && !isnan(qsum)) ? qsum : 0.0;
  const double q_h = q2abs(b.hydro_q[lz * H + h], T, P, qv, qall);
  const double n_tot = q2abs(b.hydro_n[lz * H + h], T, P, qv, qall);
  const double r_eff = b.hydro_reff[lz * H + h];
  if (s.moment_in == 13 && (q_h < st.hydro_threshold || n_tot <= 1.)) return;
  if ((q_h < st.hydro_threshold || isnan(q_h)) && (n_tot <= 0 || isnan(n_tot)) && (r_eff <= 0 || isnan(r_eff)) &&
      s.moment_in != 0)
    return;
  // layer carries hydrometeors from here on
  w.slot_st[s_idx] = 1;
  double a_ms, b_ms;
  DistPar dp;
  int nbin = (s.dist == PAMTRA_B200_DIST_MONO) ? 2 : s.nbin;
  if (nbin < 1 || nbin > b.max_nbin || make_mass_size(s, a_ms, b_ms) || make_dist_params(s, q_h, n_tot, r_eff, T, a_ms, b_ms, dp)) {
    w.slot_st[s_idx] = 3;  // fatal
    return;
  }
  const size_t base = s_idx * (size_t)b.max_nbin;
  double* d_ds = w.b_d + base;     // holds bin centres, later diameter2scat
  double* del = w.b_dd + base;
  double* nds = w.b_nd + base;
  double* rho = w.b_rho + base;
  double* mass = w.b_mass + base;
  // boundaries and f at boundaries are staged in d_ds/nds (nbin+1 entries need
  // one extra slot: the last boundary goes to del[nbin-1] staging below)
  double fb_prev = 0.0, db_prev = 0.0;
  if (s.dist == PAMTRA_B200_DIST_MONO) {
    double db[3] = {dp.d_mono - DELTA_D_MONO * .5, dp.d_mono, dp.d_mono + DELTA_D_MONO * .5};
    double fb[3];
    for (int i = 0; i < 3; i++) fb[i] = fdist(s.dist, dp, db[i]);
    for (int i = 0; i < 2; i++) {
      d_ds[i] = (db[i] + db[i + 1]) * .5;
      del[i] = db[i + 1] - db[i];
      nds[i] = fb[i];
      mass[i] = fb[i + 1];  // staging: f at upper boundary
    }
  } else {
    const bool adaptive = st.hydro_adaptive_grid != 0;
    const double min_d = (double)(float)1.0e-7, max_d = (double)(float)2.0e-2;  // REAL(4) (make_dist.f90:70-72)
    double d1w, d2w;
    if (!adaptive) {
      d1w = s.d_1 + 1.e-8;
      d2w = s.d_2;
    } else {
      // first pass: 500 bins over [min_d, max_d], locate where f crosses 0.1
      const double thres = 0.1;
      MergedGrid g;
      g.init(min_d, max_d, 500);
      const int nw = 500;
      double dprev = g.next(), fprev = fdist(s.dist, dp, dprev);
      double d1n = -1.0, d2n = -1.0;
      bool d1done = false;
      int last_cross = -1;  // largest i with f(i)>=thr && f(i+1)<thr
      double d_at_last_cross = 0.0, d_second = 0.0;
      double ftop = 0.0, dtop = 0.0;
      for (int i = 1; i <= nw; i++) {  // pairs (i, i+1), 1-based
        double dcur = g.next(), fcur = fdist(s.dist, dp, dcur);
        if (i == 1) d_second = dcur;
        if (fprev >= thres && fcur < thres) { last_cross = i; d_at_last_cross = dcur; }
        if (!d1done) {
          d1n = dprev;
          if (fprev >= fcur) { d1n = min_d; d1done = true; }
          else if (fprev < thres && fcur >= thres) d1done = true;
        }
        dprev = dcur;
        fprev = fcur;
        if (i == nw) { ftop = fcur; dtop = dcur; }
      }
      if (ftop >= thres) d2n = dtop;
      else if (last_cross >= 0) d2n = d_at_last_cross;
      else d2n = d_second;
      if (d1n < -1.e-30 || d2n < -1.e-30 || d1n > d2n) {
        w.slot_st[s_idx] = 3;
        return;
      }
      d1w = d1n;
      d2w = d2n;
    }
    MergedGrid g;
    g.init(d1w, d2w, nbin);
    db_prev = g.next();
    fb_prev = fdist(s.dist, dp, db_prev);
    for (int i = 0; i < nbin; i++) {
      double db = g.next(), fb = fdist(s.dist, dp, db);
      d_ds[i] = (db_prev + db) * .5;
      del[i] = db - db_prev;
      nds[i] = fb_prev;  // staging: f at lower boundary
      mass[i] = fb;      // staging: f at upper boundary
      db_prev = db;
      fb_prev = fb;
    }
  }
  // mass_tot and rescaling (make_dist.f90:264-279)
  double mass_tot = 0.0;
  for (int i = 0; i < nbin; i++) mass_tot = mass_tot + a_ms * (nds[i] + mass[i]) / 2.0 * del[i] * pow(d_ds[i], b_ms);
  const int mi = s.moment_in;
  const bool resc = st.conserve_mass_rescale_dsd && (mi == 3 || mi == 23 || mi == 13);
  double n_sum = 0.0;
  for (int i = 0; i < nbin; i++) {
    double fl = nds[i], fu = mass[i];
    if (resc) { fl = fl * q_h / mass_tot; fu = fu * q_h / mass_tot; }
    double n = (fl + fu) / 2.0 * del[i];
    nds[i] = n;
    n_sum += n;
  }
  bool any = false;
  for (int i = 0; i < nbin; i++) {
    if (nds[i] < n_sum / nbin * 1e-60) nds[i] = 0.0;
    any |= nds[i] > 0;
    mass[i] = a_ms * pow(d_ds[i], b_ms);
  }
  w.slot_nb[s_idx] = nbin;
  if (!any) return;  // hydrometeor_extinction.f90:294-298: layer present, species skipped
  if (w.psd_d) {
    // save_psd (hydrometeor_extinction.f90:303-309; area of drop_size_dist.f90:168-182)
    const size_t po = s_idx * (size_t)w.psd_nbin;
    for (int i = 0; i < nbin && i < w.psd_nbin; i++) {
      const double d = d_ds[i];
      double area = -99.;
      if (s.alpha_as > 0. && s.beta_as > 0.) {
        area = s.alpha_as * pow(d, s.beta_as);
        if (s.liq_ice == -1 && st.hydro_limit_density_area && area > d * d) area = d * d;
      }
      w.psd_d[po + i] = d;
      w.psd_dd[po + i] = del[i];
      w.psd_n[po + i] = nds[i];
      w.psd_mass[po + i] = mass[i];
      w.psd_area[po + i] = area;
    }
  }
  // scattering density / diameter (drop_size_dist.f90:198-208, make_soft_spheroid.f90)
  if (s.liq_ice == 1) {
    for (int i = 0; i < nbin; i++) rho[i] = RHO_WATER;
  } else {
    const double rho_ms = s.rho_ms, asr = s.as_ratio, mind = st.hydro_softsphere_min_density;
    if (rho_ms == 0.) { w.slot_st[s_idx] = 3; return; }
    for (int i = 0; i < nbin; i++) {
      double r = 0.0, dd = 0.0, m = mass[i], d = d_ds[i];
      if (rho_ms > 0.) {
        r = rho_ms;
        if (asr < 0.) dd = pow((6.0 * m) / (PI * rho_ms), 1.0 / 3.0);
        else if (asr > 0. && asr <= 1.) dd = pow((6.0 * m) / (PI * rho_ms * asr), 1.0 / 3.0);
        else if (asr > 1.) dd = pow((6.0 * m * pow(asr, 2.0)) / (PI * rho_ms), 1.0 / 3.0);
      } else {
        dd = d;
        if (asr <= 1.) {
          if (asr == -99.) r = (6.0 * m) / (PI * pow(d, 3.0));
          if (asr == -10.) r = 917.0;
          if (asr == -20. || asr == -30.) r = -1.0;  // frequency dependent: resolved per frequency
          if (asr > 0.) r = (6.0 * m) / (PI * pow(d, 3.0) * asr);
          if (r != -1.0 && r < mind) r = mind;
          if (asr == -10.) dd = pow((6.0 * m) / (PI * r), 1.0 / 3.0);
        } else {
          r = (6.0 * m * pow(asr, 2.0)) / (PI * pow(d, 3.0));
        }
      }
      if (r != -1.0 && st.hydro_limit_density_area) {
        if (r > RHO_ICE) r = RHO_ICE;
        else if (r < mind) r = mind;
      }
      if ((r != -1.0 && r <= 0.) || dd <= 0.) { w.slot_st[s_idx] = 3; return; }
      rho[i] = r;
      d_ds[i] = dd;  // d_ds now holds diameter2scat
    }
  }
  w.slot_st[s_idx] = 2;
}

// Size distributions given as full spectra (src/hydrometeor_extinction.f90:122-151):
// bins, densities and masses are taken as given, the bin widths from the bin
// bounds; a slot takes part when its number concentrations sum above zero, or
// for every slot when hydro_threshold <= 0.  One thread per (column, layer,
// species) slot, as k_psd.
__global__ void k_fullspec(Batch b, Work w, pamtra_b200_settings st) {
  const size_t s_idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int Lm = b.max_nlyrs, H = b.nhydro;
  if (s_idx >= (size_t)b.ncol * Lm * H) return;
  const int z = (s_idx / H) % Lm;
  const int c = s_idx / ((size_t)H * Lm);
  w.slot_st[s_idx] = 0;
  w.slot_nb[s_idx] = 0;
  if (z >= b.nlyrs[c]) return;
  const int nb = b.fs_nbin;
  const double* n = b.fs_n + s_idx * nb;
  double nsum = 0.0;
  for (int i = 0; i < nb; i++) nsum += n[i];
  if (!(nsum > 0.0 || st.hydro_threshold <= 0)) return;
  w.slot_st[s_idx] = 1;
  if (b.species_of(c, s_idx % H).dist == PAMTRA_B200_DIST_DISABLED) return;  // scat_name 'disabled'
  const double* d = b.fs_d + s_idx * nb;
  const double* db = b.fs_d_bound + s_idx * (nb + 1);
  const double* rho = b.fs_rho + s_idx * nb;
  const double* mass = b.fs_mass + s_idx * nb;
  const size_t base = s_idx * (size_t)b.max_nbin;
  for (int i = 0; i < nb; i++) {
    w.b_d[base + i] = d[i];
    w.b_dd[base + i] = db[i + 1] - db[i];
    w.b_nd[base + i] = n[i];
    w.b_rho[base + i] = rho[i];
    w.b_mass[base + i] = mass[i];
  }
  w.slot_nb[s_idx] = nb;
  w.slot_st[s_idx] = 2;
}

// Compaction of hydrometeor-bearing layers: pres_idx[c][z] = compact index
// (column-major order, deterministic) or -1; plist[p] = c*Lm + z.  One block.
__global__ void k_compact(Batch b, Work w) {
  const int Lm = b.max_nlyrs, H = b.nhydro;
  const int ncol = b.ncol;
  const int t = threadIdx.x, T = blockDim.x;
  __shared__ int part[1024];
  // contiguous column ranges per thread
  const int per = (ncol + T - 1) / T;
  const int c0 = min(ncol, t * per), c1 = min(ncol, c0 + per);
  int cnt = 0;
  for (int c = c0; c < c1; c++)
    for (int z = 0; z < b.nlyrs[c] && z < Lm; z++) {
      bool pres = false;
      for (int h = 0; h < H; h++) {
        int st = w.slot_st[((size_t)c * Lm + z) * H + h];
        if (st == 3) atomicOr(&w.col_status[c], PAMTRA_B200_FATAL | PAMTRA_B200_ST_PSD);
        pres |= st >= 1;
      }
      cnt += pres;
    }
  part[t] = cnt;
  __syncthreads();
  if (t == 0) {
    int acc = 0;
    for (int i = 0; i < T; i++) { int v = part[i]; part[i] = acc; acc += v; }
    w.counters[0] = acc;
  }
  __syncthreads();
  int idx = part[t];
  for (int c = c0; c < c1; c++)
    for (int z = 0; z < Lm; z++) {
      int out = -1;
      if (z < b.nlyrs[c]) {
        bool pres = false;
        for (int h = 0; h < H; h++) pres |= w.slot_st[((size_t)c * Lm + z) * H + h] >= 1;
        if (pres) {
          if (idx < w.pmax) { out = idx; w.plist[idx] = c * Lm + z; }
          else atomicOr(&w.col_status[c], PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE);
          idx++;
        }
      }
      w.pres_idx[(size_t)c * Lm + z] = out;
    }
}

}  // namespace pb
