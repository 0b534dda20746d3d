// C-ABI implementation: context, scratch arena, launch sequence.
//
// One batch = columns x frequencies.  Launch sequence on the caller's stream:
//   k_atmo      column pre-processing + output levels        (thread/column)
//   k_gas       Rosenkranz-98 gas absorption                 (thread/layer-frequency)
//   k_psd       size distributions                           (thread/layer-species)
//   k_compact   list of hydrometeor-bearing layers           (one block)
//   k_mie       Mie + species sums -> Legendre coefficients  (warp/layer-frequency, persistent)
//   k_layer<N>  scatcnv + doubling -> layer R, T, S          (CTA/layer-frequency, persistent)
//   k_adding<N> adding + radiance + TB                       (CTA/column-frequency, persistent)
// All work lists live on the device, so the sequence has no host
// synchronisation and can be captured in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "mie.cuh"
#include "prep.cuh"
#include "rt.cuh"
#include "tc.cuh"
#include "layer_tc.cuh"
#include "layer_tc64.cuh"
#include "add_tc.cuh"
#include "tmatrix.cuh"
#include "work.cuh"

using namespace pb;

namespace {

// Rosenkranz-98 line tables (src/gasabs_module.f90:106-211, 214-333); the
// reference declares them as default REAL literals.
const float H_O2_W300[40] = {1.63f, 1.646f, 1.468f, 1.449f, 1.382f, 1.360f, 1.319f, 1.297f, 1.266f, 1.248f,
                             1.221f, 1.207f, 1.181f, 1.171f, 1.144f, 1.139f, 1.110f, 1.108f, 1.079f, 1.078f,
                             1.05f,  1.05f,  1.02f,  1.02f,  1.0f,   1.0f,   0.97f,  0.97f,  0.94f,  0.94f,
                             0.92f,  0.92f,  0.89f,  0.89f,  1.92f,  1.92f,  1.92f,  1.81f,  1.81f,  1.81f};
const float H_O2_Y300[40] = {-0.0233f, 0.2408f,  -0.3486f, 0.5227f,  -0.5430f, 0.5877f,  -0.3970f, 0.3237f,
                             -0.1348f, 0.0311f,  0.0725f,  -0.1663f, 0.2832f,  -0.3629f, 0.3970f,  -0.4599f,
                             0.4695f,  -0.5199f, 0.5187f,  -0.5597f, 0.5903f,  -0.6246f, 0.6656f,  -0.6942f,
                             0.7086f,  -0.7325f, 0.7348f,  -0.7546f, 0.7702f,  -0.7864f, 0.8083f,  -0.8210f,
                             0.8439f,  -0.8529f, 0.f,      0.f,      0.f,      0.f,      0.f,      0.f};
const float H_O2_V[40] = {0.0079f,  -0.0978f, 0.0844f,  -0.1273f, 0.0699f,  -0.0776f, 0.2309f,  -0.2825f,
                          0.0436f,  -0.0584f, 0.6056f,  -0.6619f, 0.6451f,  -0.6759f, 0.6547f,  -0.6675f,
                          0.6135f,  -0.6139f, 0.2952f,  -0.2895f, 0.2654f,  -0.2590f, 0.3750f,  -0.3680f,
                          0.5085f,  -0.5002f, 0.6206f,  -0.6091f, 0.6526f,  -0.6393f, 0.6640f,  -0.6475f,
                          0.6729f,  -0.6545f, 0.f,      0.f,      0.f,      0.f,      0.f,      0.f};
const float H_O2_F[40] = {118.7503f, 56.2648f, 62.4863f, 58.4466f, 60.3061f, 59.5910f, 59.1642f, 60.4348f,
                          58.3239f,  61.1506f, 57.6125f, 61.8002f, 56.9682f, 62.4112f, 56.3634f, 62.9980f,
                          55.7838f,  63.5685f, 55.2214f, 64.1278f, 54.6712f, 64.6789f, 54.1300f, 65.2241f,
                          53.5957f,  65.7648f, 53.0669f, 66.3021f, 52.5424f, 66.8368f, 52.0214f, 67.3696f,
                          51.5034f,  67.9009f, 368.4984f, 424.7631f, 487.2494f, 715.3932f, 773.8397f, 834.1453f};
const float H_O2_S300[40] = {0.2936E-14f, 0.8079E-15f, 0.2480E-14f, 0.2228E-14f, 0.3351E-14f, 0.3292E-14f,
                             0.3721E-14f, 0.3891E-14f, 0.3640E-14f, 0.4005E-14f, 0.3227E-14f, 0.3715E-14f,
                             0.2627E-14f, 0.3156E-14f, 0.1982E-14f, 0.2477E-14f, 0.1391E-14f, 0.1808E-14f,
                             0.9124E-15f, 0.1230E-14f, 0.5603E-15f, 0.7842E-15f, 0.3228E-15f, 0.4689E-15f,
                             0.1748E-15f, 0.2632E-15f, 0.8898E-16f, 0.1389E-15f, 0.4264E-16f, 0.6899E-16f,
                             0.1924E-16f, 0.3229E-16f, 0.8191E-17f, 0.1423E-16f, 0.6460E-15f, 0.7047E-14f,
                             0.3011E-14f, 0.1826E-14f, 0.1152E-13f, 0.3971E-14f};
const float H_O2_BE[40] = {0.009f, 0.015f, 0.083f, 0.084f, 0.212f, 0.212f, 0.391f, 0.391f, 0.626f, 0.626f,
                           0.915f, 0.915f, 1.26f,  1.26f,  1.66f,  1.665f, 2.119f, 2.115f, 2.624f, 2.625f,
                           3.194f, 3.194f, 3.814f, 3.814f, 4.484f, 4.484f, 5.224f, 5.224f, 6.004f, 6.004f,
                           6.844f, 6.844f, 7.744f, 7.744f, 0.048f, 0.044f, 0.049f, 0.145f, 0.141f, 0.145f};
const float H_H2O_FL[15] = {22.2351f, 183.3101f, 321.2256f, 325.1529f, 380.1974f, 439.1508f, 443.0183f, 448.0011f,
                            470.8890f, 474.6891f, 488.4911f, 556.9360f, 620.7008f, 752.0332f, 916.1712f};
const float H_H2O_S1[15] = {0.1310E-13f, 0.2273E-11f, 0.8036E-13f, 0.2694E-11f, 0.2438E-10f,
                            0.2179E-11f, 0.4624E-12f, 0.2562E-10f, 0.8369E-12f, 0.3263E-11f,
                            0.6659E-12f, 0.1531E-08f, 0.1707E-10f, 0.1011E-08f, 0.4227E-10f};
const float H_H2O_B2[15] = {2.144f, .668f, 6.179f, 1.541f, 1.048f, 3.595f, 5.048f, 1.405f,
                            3.597f, 2.379f, 2.852f, .159f,  2.391f, .396f,  1.441f};
const float H_H2O_W3[15] = {0.002656f, 0.00281f, 0.0023f,  0.00278f, 0.00287f, 0.0021f,  0.00186f, 0.00263f,
                            0.00215f,  0.00236f, 0.0026f,  0.00321f, 0.00244f, 0.00306f, 0.00267f};
const float H_H2O_X[15] = {0.69f, 0.64f, 0.67f, 0.68f, 0.54f, 0.63f, 0.60f, 0.66f,
                           0.66f, 0.65f, 0.69f, 0.69f, 0.71f, 0.68f, 0.70f};
const float H_H2O_WS[15] = {0.0127488f, 0.01491f, 0.0108f,  0.0135f,  0.01541f, 0.0090f,  0.00788f, 0.01275f,
                            0.00983f,   0.01095f, 0.01313f, 0.01320f, 0.01140f, 0.01253f, 0.01275f};
const float H_H2O_XS[15] = {0.61f, 0.85f, 0.54f, 0.74f, 0.89f, 0.52f, 0.50f, 0.67f,
                            0.65f, 0.64f, 0.72f, 1.0f,  0.68f, 0.84f, 0.78f};

constexpr int GQ_MAX = 256;

// Gauss-Legendre nodes/weights for every n = 1..GQ_MAX (src/scat_utilities.f90:1-44),
// packed at offset n*(n-1)/2.  Block per n, thread per node pair.
__global__ void k_gauss_table(double* gx, double* gw) {
  const int n = blockIdx.x + 1;
  const int jj = threadIdx.x + 1;
  if (jj > (n + 1) / 2) return;
  double* xa = gx + (size_t)n * (n - 1) / 2;
  double* wt = gw + (size_t)n * (n - 1) / 2;
  double x = cos(PI * (jj - 0.25) / (n + 0.5));
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
  } while (fabs(x - xp) > 3.0e-13 && i < 10);
  xa[jj - 1] = -x;
  xa[n - jj] = x;
  double ww = 2.0 / ((1.0 - x * x) * dpl * dpl);
  wt[jj - 1] = ww;
  wt[n - jj] = ww;
}

// Lobatto nodes/weights for N = 8, 16, 32 (src/rt_utilities.f90:165-203).
__global__ void k_lobatto_table(double* mu, double* w) {
  const int which = blockIdx.x;  // 0: 8, 1: 16, 2: 32
  const int num = 8 << which;
  const int off = lob_off(num);
  const int jj = threadIdx.x + 1;
  if (jj > num) return;
  if (jj == num) {
    mu[off + num - 1] = 1.0;
    w[off + num - 1] = 2.0 / ((2 * num) * (2 * num - 1));
    return;
  }
  const int n = 2 * num, n1 = n - 1;
  const double ci = 0.50;
  double x = sin(F(3.141592654f) * (jj - ci) / (n - .5));
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
  } while (fabs(x - xp) > 3.0e-14 && i < 10);
  mu[off + jj - 1] = x;
  w[off + jj - 1] = 2.0 / (n * n1 * pl * pl);
}

__global__ void k_fill_d(double* p, double v, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// angles in degrees (src/run_rt.f90:196-197) for N = max_nummu
__global__ void k_angles(double* out, const double* lob_mu, int N) {
  int jj = threadIdx.x;
  if (jj >= N) return;
  const double* mu = lob_mu + lob_off(N);
  out[jj] = 180 - (180. * acos(mu[N - 1 - jj]) / PI);
  out[N + jj] = (180. * acos(mu[jj]) / PI);
}

// save_ssp-style per-(column, frequency, layer) outputs
__global__ void k_ssp_out(Batch b, Work w, pamtra_b200_outputs out) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq;
  if (idx >= (size_t)b.ncol * Fm * Lm) return;
  const int z = idx % Lm, f = (idx / Lm) % Fm, c = idx / ((size_t)Lm * Fm);
  const int p = (z < b.nlyrs[c]) ? w.pres_idx[(size_t)c * Lm + z] : -1;
  const size_t item = (size_t)p * Fm + f;
  if (out.kexttot) out.kexttot[idx] = (p >= 0) ? w.m_kext[item] : 0.0;
  if (out.salbedo) out.salbedo[idx] = (p >= 0) ? w.m_salb[item] : 0.0;
  if (out.num_doubles) out.num_doubles[idx] = (p >= 0) ? w.lay_nd[item] : -1;
}

// Simple radar per (column, frequency): src/radar_simulator.f90:123-176
// (radar_mode 'simple', one polarisation, no noise) over the layers in the
// reference's loop order (top-down when the attenuation is integrated from
// the top, src/hydrometeor_extinction.f90:96-106), with the gas attenuation
// of src/run_rt.f90:119-121.  Layers without hydrometeors keep Ze = -9999
// and zero hydrometeor attenuation.
__global__ void k_radar(Batch b, Work w, pamtra_b200_settings st, pamtra_b200_outputs out) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq;
  if (u >= b.ncol * Fm) return;
  const int c = u / Fm, f = u % Fm;
  const size_t o = ((size_t)c * Fm + f) * Lm;
  const int L = (f < b.col_nfreq(c)) ? b.nlyrs[c] : 0;
  for (int z = 0; z < Lm; z++) {
    if (out.ze) out.ze[o + z] = -9999.0;
    if (out.att_hydro) out.att_hydro[o + z] = 0.0;
    if (out.att_atmo) out.att_atmo[o + z] = 0.0;
  }
  if (L == 0) return;
  const double* hl = w.hgt_lev + (size_t)c * (Lm + 1);
  const double wavelength = C_LIGHT / (b.freq(c, f) * 1.e9);  // m
  const double K2 = st.radar_k2;
  const bool down = st.radar_attenuation == PAMTRA_B200_ATT_TOP_DOWN;
  const double pi2 = PI * PI, w2 = wavelength * wavelength;
  const double pi5 = (pi2 * pi2) * PI, w4 = w2 * w2;  // pi**5, wavelength**4
  double acc_h = 0.0, acc_a = 0.0;  // hydrometeor / gas attenuation of the layers already passed (dB)
  for (int k = 0; k < L; k++) {
    const int z = down ? L - 1 - k : k;
    const double dh = hl[z + 1] - hl[z];
    const double att_atmo = 10.0 * log10(exp(w.kgas[((size_t)c * Fm + f) * Lm + z] * dh));
    if (out.att_atmo) out.att_atmo[o + z] = att_atmo;
    const int p = w.pres_idx[(size_t)c * Lm + z];
    double att_hydro = 0.0;
    if (p >= 0) {
      const size_t item = (size_t)p * Fm + f;
      att_hydro = 10.0 * log10(exp(w.m_kext[item] * dh));
      double ze_back = 1.e18 * (1.0 / (K2 * pi5)) * w.m_back[item] * w4;
      double pia = 0.0;
      if (st.radar_attenuation != PAMTRA_B200_ATT_DISABLED) {
        if (k > 0) pia = 2.0 * (acc_h + acc_a);
        pia = pia + att_hydro + att_atmo;
      }
      pia = pow(10.0, 0.1 * pia);
      ze_back = ze_back / pia;
      if (out.att_hydro) out.att_hydro[o + z] = att_hydro;
      if (out.ze) out.ze[o + z] = (ze_back == 0.0) ? -9999.0 : 10.0 * log10(ze_back);
    }
    acc_h = acc_h + att_hydro;
    acc_a = acc_a + att_atmo;
  }
}

__global__ void k_status_out(Work w, int32_t* out, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = w.status[i];
}

struct Plan {
  size_t total;
  size_t o_hgt_lev, o_temp_lev, o_temp, o_press, o_rho_vap, o_q_hum, o_vap, o_gtemp, o_outlev, o_kgas;
  size_t o_slot_st, o_slot_nb, o_bd, o_bdd, o_bnd, o_brho, o_bmass;
  size_t o_pres_idx, o_plist, o_counters, o_mkext, o_msalb, o_mback, o_mrefr, o_mnleg, o_mlegen, o_lay, o_laynd, o_status,
      o_colst;
  size_t o_species, o_addscr, o_mieslab, o_addstk;
  int mie_nslab;  // k_mie warps the slabs are sized for
  bool f32_coef;
  bool tc_add;  // split-precision adding for NUMMU 16 (FP32 layer records, stacks)
  int add_grid;  // CTAs of k_adding<32> the scratch is sized for
  int pmax;
  int max_nbin;
  int maxN;
  size_t lay_stride;
};

size_t lay_stride_for(int N) {
  return (lay_stride_n(N) + 1) & ~(size_t)1;  // keep 16-byte alignment of each item
}

Plan make_plan(const pamtra_b200_columns* c, int default_nummu, int sms, int mie_slabs, bool f32_coef = false,
               bool tc_add = false) {
  Plan p{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = (off + 255) & ~(size_t)255;
    off = o + bytes;
    return o;
  };
  const size_t C = c->ncol, Lm = c->max_nlyrs, H = c->nhydro, Fm = c->max_nfreq;
  int mb = 1;
  const size_t nsp = c->species_stride ? C * H : H;
  if (c->fs_d) mb = std::max(mb, c->fs_nbin);
  else
    for (size_t i = 0; i < nsp; i++) mb = std::max(mb, c->species[i].dist == PAMTRA_B200_DIST_MONO ? 2 : c->species[i].nbin);
  p.max_nbin = mb;
  int mask = c->nummu_mask ? c->nummu_mask : (default_nummu == 8 ? 1 : default_nummu == 16 ? 2 : 4);
  p.maxN = (mask & 4) ? 32 : (mask & 2) ? 16 : 8;
  p.pmax = c->max_present > 0 ? c->max_present : (int)(C * Lm);
  p.lay_stride = lay_stride_for(p.maxN);
  const size_t S = C * Lm * H;
  p.o_hgt_lev = take(C * (Lm + 1) * 8);
  p.o_temp_lev = take(C * (Lm + 1) * 8);
  p.o_temp = take(C * Lm * 8);
  p.o_press = take(C * Lm * 8);
  p.o_rho_vap = take(C * Lm * 8);
  p.o_q_hum = take(C * Lm * 8);
  p.o_vap = take(C * Lm * 8);
  p.o_gtemp = take(C * 8);
  p.o_outlev = take(C * std::max(1, c->noutlevels) * 4);
  p.o_kgas = take(C * Fm * Lm * 8);
  p.o_slot_st = take(std::max<size_t>(S, 1));
  p.o_slot_nb = take(std::max<size_t>(S, 1) * 4);
  p.o_bd = take(std::max<size_t>(S, 1) * mb * 8);
  p.o_bdd = take(std::max<size_t>(S, 1) * mb * 8);
  p.o_bnd = take(std::max<size_t>(S, 1) * mb * 8);
  p.o_brho = take(std::max<size_t>(S, 1) * mb * 8);
  p.o_bmass = take(std::max<size_t>(S, 1) * mb * 8);
  p.o_pres_idx = take(C * Lm * 4);
  p.o_plist = take((size_t)std::max(1, p.pmax) * 4);
  p.o_counters = take(16 * 4);
  const size_t items = (size_t)std::max(1, p.pmax) * Fm;
  p.o_mkext = take(items * 8);
  p.o_msalb = take(items * 8);
  p.o_mback = take(items * 8);
  p.o_mrefr = take(items * 4 * 8);
  p.o_mnleg = take(items * 4);
  p.f32_coef = f32_coef;  // Legendre coefficients stored in FP32 (split-precision form)
  p.o_mlegen = take(items * 3 * MAXNLEG * (f32_coef ? 4 : 8));
  p.o_lay = take(items * p.lay_stride * 8);
  p.o_laynd = take(items * 4);
  p.o_status = take(C * Fm * 4);
  p.o_colst = take(C * 4);
  p.o_species = take(std::max<size_t>(nsp, 1) * sizeof(pamtra_b200_species));
  p.add_grid = (mask & 4) ? std::max(1, sms) : 0;
  p.o_addscr = take((size_t)p.add_grid * (10 - AddSmem<32>::NS) * RTCfg<32>::MAT * 8);
  // one slab per k_mie warp; more warps than (layer, frequency) items would idle
  p.mie_nslab = c->nhydro > 0 ? (int)std::min<size_t>((size_t)mie_slabs, items) : 0;
  p.o_mieslab = take((size_t)p.mie_nslab * MIE_SLAB_STRIDE * 8);
  p.tc_add = tc_add && (mask & 2);
  p.o_addstk = take(p.tc_add ? C * Fm * STK_FLOATS * 4 : 0);
  p.total = take(0) + 256;
  return p;
}

int occupancy_blocks(const void* func, int threads, size_t smem, int sms) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, func, threads, smem) != cudaSuccess || nb < 1) nb = 1;
  return nb * sms;
}

// Persistent grid: `cps` CTAs per SM when set (capped at the resident
// maximum), else the resident maximum.
int persistent_grid(const void* func, int threads, size_t smem, int sms, int cps) {
  const int full = occupancy_blocks(func, threads, smem, sms);
  return cps > 0 ? std::min(full, cps * sms) : full;
}

}  // namespace

namespace {
// ---------------------------------------------------------------- single stages
__global__ void k_gas_elem(const double* f, const double* T, const double* rv, const double* p, double* k,
                                  int32_t* st, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int s = gas_r98(f[i], T[i], rv[i], p[i], &k[i]);
  if (st) st[i] = s;
}

template <int n>
__global__ void k_minvert(const double* a, double* ainv, int32_t* status, int count) {
  constexpr int LD = Team<n>::LD, T = Team<n>::T;
  extern __shared__ double smem_raw[];
  double* M = smem_raw;
  InvScratch<n>& S = *reinterpret_cast<InvScratch<n>*>(smem_raw + n * LD);
  const int t = threadIdx.x;
  for (int m = blockIdx.x; m < count; m += gridDim.x) {
    const double* src = a + (size_t)m * n * n;
    for (int e = t; e < n * n; e += T) M[(e / n) * LD + e % n] = src[e];
    __syncthreads();
    int s = ginv<n>(M, S);
    double* dst = ainv + (size_t)m * n * n;
    for (int e = t; e < n * n; e += T) dst[e] = M[(e / n) * LD + e % n];
    if (status && t == 0) status[m] = s ? (PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT) : 0;
    __syncthreads();
  }
}

// C = A * B for `count` column-major 32 x 32 matrices as 3xTF32 tcgen05
// products (FP32 accumulation in tensor memory).  One CTA of 128 threads per
// matrix pair: thread m writes row m of A into the A tile, warp 1 transposes
// the rows of B it loaded so that tile row n is column n of B, and TMEM lane
// m holds row m of C.
// Rows 32..127 of the A tile stay zero.
__global__ void __launch_bounds__(128) k_mmult_3xtf32(const double* a, const double* b, double* c, int count,
                                                      int* err) {
  extern __shared__ __align__(128) float tsm[];
  float* a_hi = tsm;
  float* a_lo = tsm + 128 * 32;
  float* b_hi = tsm + 2 * 128 * 32;
  float* b_lo = b_hi + 32 * 32;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  if (warp == 0) tc::tmem_alloc(&tslot, 32);
  if (t == 0) tc::mbar_init(&mbar, 1);
  for (int i = t; i < 2 * 128 * 32; i += 128) tsm[i] = 0.f;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tslot;
  uint32_t parity = 0;
  bool ok = true;
  for (int m = blockIdx.x; m < count && ok; m += gridDim.x) {
    const double* am = a + (size_t)m * 1024;
    const double* bm = b + (size_t)m * 1024;
    if (t < 32) {
      float v[32];
#pragma unroll
      for (int k = 0; k < 32; k++) v[k] = (float)am[k * 32 + t];  // row t of A
      tc::put_row(a_hi, a_lo, t, v);
    } else if (t < 64) {
      float v[32];
#pragma unroll
      for (int k = 0; k < 32; k++) v[k] = (float)bm[k * 32 + (t - 32)];  // row t-32 of B, transposed below
      tc::put_rows_from_cols(b_hi, b_lo, v);  // tile row n = column n of B
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (t == 0) tc::mma3(tbase, a_hi, a_lo, b_hi, b_lo, &mbar);
    ok = tc::mbar_wait(&mbar, parity);
    parity ^= 1;
    tc::fence_after_sync();
    if (ok && warp == 0) {
      float d[32];
      tc::tmem_ld32(tbase, d);
      double* cm = c + (size_t)m * 1024;
#pragma unroll
      for (int n = 0; n < 32; n++) cm[n * 32 + lane] = d[n];
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
  if (!ok) {
    if (t == 0) atomicOr(err, 1);
    tc::mbar_wait(&mbar, parity ^ 1);  // let a late MMA finish before the memory is released
  }
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 32);
}

}  // namespace

struct pamtra_b200_ctx {
  int device = 0;
  int sm_count = 0;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  double* gq_x = nullptr;
  double* gq_w = nullptr;
  double* lob_mu = nullptr;
  double* lob_w = nullptr;
  // species tables: pinned staging ring and the table last left in the arena
  static constexpr int NSP_RING = 3;
  struct SpStage {
    pamtra_b200_species* h = nullptr;
    size_t cap = 0;
    cudaEvent_t ev = nullptr;
    int used = 0;
  } sp_ring[NSP_RING];
  int sp_next = 0;
  std::vector<unsigned char> sp_last;
  const char* sp_last_arena = nullptr;
  size_t sp_last_off = 0;
  // scatcnv weight tables per NUMMU (allocated when first needed) and their
  // need / ready flags [2][3][SCAT_NPI]
  double* wtab[3] = {nullptr, nullptr, nullptr};
  int* wt_flags = nullptr;
  int last_launches = 0;
  char* tm_buf = nullptr;  // T-matrix branch: inputs, per-bin results and the CTAs' scratch slots
  size_t tm_bytes = 0;
  char* stage = nullptr;  // device staging for run_host
  size_t stage_bytes = 0;
  // launch shapes (pamtra_b200_set_launch; 0 = occupancy default)
  int mie_warps = MIE_WARPS;  // warps per k_mie CTA (2, 4 or 8)
  int mie_cps = 0;            // k_mie CTAs per SM
  int layer_cps = 0;          // k_layer / k_layer_tc CTAs per SM
  int adding_cps = 0;         // k_adding CTAs per SM
  int mie_group = MIE_GROUP;  // bins per k_mie work item (4 or 8)
  uint32_t spin_limit = tc::MBAR_SPIN_LIMIT;  // polls per wait on a tensor-core MMA
  const int* last_counters = nullptr;          // work counters of the last run (in the arena)
  // optional per-stage timing (events recorded on the run's stream)
  int timing = 0;
  cudaEvent_t ev[16] = {};
  int nev = 0;
  int ev_stage[16] = {};
};

enum Stage { STG_PREP = 0, STG_PSD, STG_MIE, STG_LAYER, STG_ADDING, STG_COUNT };

static void mark(pamtra_b200_ctx* ctx, cudaStream_t s, int stage) {
  if (!ctx->timing || ctx->nev >= 16) return;
  if (!ctx->ev[ctx->nev]) cudaEventCreate(&ctx->ev[ctx->nev]);
  cudaEventRecord(ctx->ev[ctx->nev], s);
  ctx->ev_stage[ctx->nev] = stage;
  ctx->nev++;
}

// c_n of mieangle in REAL(4) arithmetic (host float division is IEEE, as on
// the device) and 1/n
static int upload_mie_constants() {
  static_assert(MAXNLEG > NT_MAX, "1/n table covers the Mie terms");
  double c[NT_MAX + 1], r[MAXNLEG];
  c[0] = 0.0;
  r[0] = 0.0;
  for (int n = 1; n <= NT_MAX; n++) c[n] = (double)((float)(2 * n + 1) / (float)(n * (n + 1)));
  for (int n = 1; n < MAXNLEG; n++) r[n] = 1.0 / n;
  return (cudaMemcpyToSymbol(c_mie_c, c, sizeof(c)) != cudaSuccess ||
          cudaMemcpyToSymbol(c_mie_inv, r, sizeof(r)) != cudaSuccess) ? 1 : 0;
}

static int set_smem_attrs() {
  static std::once_flag once;
  static int rc = 0;
  std::call_once(once, [] {
    auto set = [](const void* f, size_t bytes) {
      if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) rc = 1;
    };
    set((const void*)k_mie<4>, MIE_MAX_WARPS * sizeof(MieSmem));
    set((const void*)k_mie<8>, MIE_MAX_WARPS * sizeof(MieSmem));
    set((const void*)k_layer<8>, sizeof(LayerSmem<8>));
    set((const void*)k_layer<16>, sizeof(LayerSmem<16>));
    set((const void*)k_layer<32>, sizeof(LayerSmem<32>));
    set((const void*)k_layer_tc<16>, layer_tc_smem<16>());
    set((const void*)k_layer_tc64, layer_tc64_smem());
    set((const void*)k_adding<8>, sizeof(AddSmem<8>));
    set((const void*)k_adding<16>, sizeof(AddSmem<16>));
    set((const void*)k_adding<32>, sizeof(AddSmem<32>));
    set((const void*)k_adding<8, true>, sizeof(AddSmem<8>));
    set((const void*)k_adding<16, true>, sizeof(AddSmem<16>));
    set((const void*)k_adding<32, true>, sizeof(AddSmem<32>));
    set((const void*)k_minvert<64>, Team<64>::MAT * 8 + sizeof(InvScratch<64>));
    set((const void*)k_adding_tc<16>, add_tc_smem());
    set((const void*)k_adding_finish<16>, sizeof(AddSmem<16>));
  });
  return rc;
}

extern "C" {

int32_t pamtra_b200_create(int32_t device, pamtra_b200_ctx** out) {
  if (!out) return PAMTRA_B200_FATAL;
  if (cudaSetDevice(device) != cudaSuccess) return PAMTRA_B200_FATAL;
  pamtra_b200_ctx* ctx = new pamtra_b200_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  if (set_smem_attrs()) { delete ctx; return PAMTRA_B200_FATAL; }
  const size_t gq_n = (size_t)GQ_MAX * (GQ_MAX + 1) / 2;
  if (cudaMalloc(&ctx->gq_x, gq_n * 8) || cudaMalloc(&ctx->gq_w, gq_n * 8) || cudaMalloc(&ctx->lob_mu, 56 * 8) ||
      cudaMalloc(&ctx->lob_w, 56 * 8)) {
    delete ctx;
    return PAMTRA_B200_FATAL;
  }
  k_gauss_table<<<GQ_MAX, 128>>>(ctx->gq_x, ctx->gq_w);
  {
    double la[MAXNLEG], lb[MAXNLEG];
    la[0] = 0.0;
    lb[0] = 0.0;
    for (int l = 1; l < MAXNLEG; l++) {
      la[l] = (2.0 * l - 1.0) / l;
      lb[l] = (l - 1.0) / l;
    }
    cudaMemcpyToSymbol(c_leg_a, la, sizeof(la));
    cudaMemcpyToSymbol(c_leg_b, lb, sizeof(lb));
  }
  upload_mie_constants();
  k_lobatto_table<<<3, 32>>>(ctx->lob_mu, ctx->lob_w);
  cudaMemcpyToSymbol(c_o2_w300, H_O2_W300, sizeof(H_O2_W300));
  cudaMemcpyToSymbol(c_o2_y300, H_O2_Y300, sizeof(H_O2_Y300));
  cudaMemcpyToSymbol(c_o2_v, H_O2_V, sizeof(H_O2_V));
  cudaMemcpyToSymbol(c_o2_f, H_O2_F, sizeof(H_O2_F));
  cudaMemcpyToSymbol(c_o2_s300, H_O2_S300, sizeof(H_O2_S300));
  cudaMemcpyToSymbol(c_o2_be, H_O2_BE, sizeof(H_O2_BE));
  cudaMemcpyToSymbol(c_h2o_fl, H_H2O_FL, sizeof(H_H2O_FL));
  cudaMemcpyToSymbol(c_h2o_s1, H_H2O_S1, sizeof(H_H2O_S1));
  cudaMemcpyToSymbol(c_h2o_b2, H_H2O_B2, sizeof(H_H2O_B2));
  cudaMemcpyToSymbol(c_h2o_w3, H_H2O_W3, sizeof(H_H2O_W3));
  cudaMemcpyToSymbol(c_h2o_x, H_H2O_X, sizeof(H_H2O_X));
  cudaMemcpyToSymbol(c_h2o_ws, H_H2O_WS, sizeof(H_H2O_WS));
  cudaMemcpyToSymbol(c_h2o_xs, H_H2O_XS, sizeof(H_H2O_XS));
  if (cudaDeviceSynchronize() != cudaSuccess) {
    delete ctx;
    return PAMTRA_B200_FATAL;
  }
  *out = ctx;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_destroy(pamtra_b200_ctx* ctx) {
  if (!ctx) return PAMTRA_B200_OK;
  cudaSetDevice(ctx->device);
  cudaFree(ctx->arena);
  cudaFree(ctx->gq_x);
  cudaFree(ctx->gq_w);
  cudaFree(ctx->lob_mu);
  cudaFree(ctx->lob_w);
  cudaFree(ctx->stage);
  cudaFree(ctx->tm_buf);
  for (double* p : ctx->wtab) cudaFree(p);
  cudaFree(ctx->wt_flags);
  for (auto& sg : ctx->sp_ring) {
    if (sg.ev) cudaEventSynchronize(sg.ev), cudaEventDestroy(sg.ev);
    if (sg.h) cudaFreeHost(sg.h);
  }
  for (int i = 0; i < 16; i++)
    if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
  delete ctx;
  return PAMTRA_B200_OK;
}

size_t pamtra_b200_workspace_bytes(const pamtra_b200_columns* cols, int32_t precision) {
  if (!cols || !cols->species) return 0;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const bool split = precision == PAMTRA_B200_PREC_3XTF32 || precision == PAMTRA_B200_PREC_3XTF32_FP64ADD;
  return make_plan(cols, 16, sms, sms * MIE_SLAB_WARPS_PER_SM, split, precision == PAMTRA_B200_PREC_3XTF32).total;
}

int32_t pamtra_b200_reserve(pamtra_b200_ctx* ctx, size_t bytes) {
  if (!ctx) return PAMTRA_B200_FATAL;
  if (bytes <= ctx->arena_bytes) return PAMTRA_B200_OK;
  cudaSetDevice(ctx->device);
  cudaFree(ctx->arena);
  ctx->arena = nullptr;
  ctx->arena_bytes = 0;
  ctx->sp_last_arena = nullptr;  // the arena contents are gone
  if (cudaMalloc(&ctx->arena, bytes) != cudaSuccess) return PAMTRA_B200_FATAL;
  ctx->arena_bytes = bytes;
  return PAMTRA_B200_OK;
}

// ---------------------------------------------------------------- CUDA graphs
struct pamtra_b200_graph {
  pamtra_b200_ctx* ctx = nullptr;
  const char* arena = nullptr;  // the arena the captured launches address
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
};

int32_t pamtra_b200_graph_capture(pamtra_b200_ctx* ctx, const pamtra_b200_settings* st,
                                  const pamtra_b200_columns* cols, const pamtra_b200_outputs* out, int32_t precision,
                                  void* stream_, pamtra_b200_graph** gout) {
  if (!ctx || !gout) return PAMTRA_B200_FATAL;
  *gout = nullptr;
  cudaSetDevice(ctx->device);
  cudaStream_t stream = (cudaStream_t)stream_;
  // one direct run sizes the arena, fills the tables and leaves the species
  // table resident, so the captured sequence has no host-side waits
  const int timing = ctx->timing;
  ctx->timing = 0;
  int32_t rc = pamtra_b200_run(ctx, st, cols, out, precision, stream);
  if (rc == PAMTRA_B200_OK && cudaStreamSynchronize(stream) != cudaSuccess) rc = PAMTRA_B200_FATAL;
  cudaStream_t cs = nullptr;
  if (rc == PAMTRA_B200_OK && cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) rc = PAMTRA_B200_FATAL;
  pamtra_b200_graph* g = nullptr;
  if (rc == PAMTRA_B200_OK) {
    g = new pamtra_b200_graph();
    g->ctx = ctx;
    g->arena = ctx->arena;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = PAMTRA_B200_FATAL;
    if (rc == PAMTRA_B200_OK) {
      const int32_t rr = pamtra_b200_run(ctx, st, cols, out, precision, cs);
      const cudaError_t ce = cudaStreamEndCapture(cs, &g->graph);
      if (rr != PAMTRA_B200_OK || ce != cudaSuccess || ctx->arena != g->arena) rc = PAMTRA_B200_FATAL;
      g->launches = ctx->last_launches;
    }
    if (rc == PAMTRA_B200_OK && cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess) rc = PAMTRA_B200_FATAL;
  }
  if (cs) cudaStreamDestroy(cs);
  ctx->timing = timing;
  cudaGetLastError();
  if (rc != PAMTRA_B200_OK) {
    if (g) {
      if (g->exec) cudaGraphExecDestroy(g->exec);
      if (g->graph) cudaGraphDestroy(g->graph);
      delete g;
    }
    return rc;
  }
  *gout = g;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_graph_launch(pamtra_b200_graph* g, void* stream) {
  if (!g || !g->exec) return PAMTRA_B200_FATAL;
  if (g->ctx->arena != g->arena) return PAMTRA_B200_FATAL;  // the arena was regrown after the capture
  cudaSetDevice(g->ctx->device);
  g->ctx->last_launches = g->launches;
  return cudaGraphLaunch(g->exec, (cudaStream_t)stream) == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

int32_t pamtra_b200_graph_destroy(pamtra_b200_graph* g) {
  if (!g) return PAMTRA_B200_OK;
  cudaSetDevice(g->ctx->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_last_launch_count(const pamtra_b200_ctx* ctx) { return ctx ? ctx->last_launches : 0; }

int32_t pamtra_b200_abi_sizes(size_t* out, int32_t n) {
  const size_t sz[6] = {sizeof(pamtra_b200_settings), sizeof(pamtra_b200_species), sizeof(pamtra_b200_columns),
                        sizeof(pamtra_b200_outputs), sizeof(pamtra_b200_tmatrix_in), sizeof(pamtra_b200_tmatrix_out)};
  for (int i = 0; i < n && i < 6; i++) out[i] = sz[i];
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_set_launch(pamtra_b200_ctx* ctx, const int32_t* params, int32_t n) {
  if (!ctx || (n > 0 && !params) || n < 0 || n > PAMTRA_B200_NLAUNCH) return PAMTRA_B200_FATAL;
  int v[PAMTRA_B200_NLAUNCH] = {MIE_WARPS, 0, 0, 0, 0};
  for (int i = 0; i < n; i++) v[i] = params[i];
  if (!(v[0] == 0 || v[0] == 2 || v[0] == 4 || v[0] == 8)) return PAMTRA_B200_FATAL;
  for (int i = 1; i < 4; i++)
    if (v[i] < 0 || v[i] > 32) return PAMTRA_B200_FATAL;
  if (!(v[4] == 0 || v[4] == 4 || v[4] == 8)) return PAMTRA_B200_FATAL;
  ctx->mie_warps = v[0] ? v[0] : MIE_WARPS;
  ctx->mie_cps = v[1];
  ctx->layer_cps = v[2];
  ctx->adding_cps = v[3];
  ctx->mie_group = v[4] ? v[4] : MIE_GROUP;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_get_launch(const pamtra_b200_ctx* ctx, int32_t* params, int32_t n) {
  if (!ctx || !params || n < 0) return PAMTRA_B200_FATAL;
  const int v[PAMTRA_B200_NLAUNCH] = {ctx->mie_warps, ctx->mie_cps, ctx->layer_cps, ctx->adding_cps,
                                     ctx->mie_group};
  for (int i = 0; i < n && i < PAMTRA_B200_NLAUNCH; i++) params[i] = v[i];
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_layer_products(pamtra_b200_ctx* ctx, uint64_t* out, void* stream) {
  if (!ctx || !out) return PAMTRA_B200_FATAL;
  *out = 0;
  if (!ctx->last_counters || ctx->last_counters < (const int*)ctx->arena ||
      ctx->last_counters >= (const int*)(ctx->arena + ctx->arena_bytes))
    return PAMTRA_B200_FATAL;
  cudaSetDevice(ctx->device);
  unsigned long long v = 0;
  if (cudaMemcpyAsync(&v, ctx->last_counters + COUNTER_PRODUCTS, sizeof(v), cudaMemcpyDeviceToHost,
                      (cudaStream_t)stream) != cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return PAMTRA_B200_FATAL;
  *out = v;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_set_wait_limit(pamtra_b200_ctx* ctx, uint32_t polls) {
  if (!ctx) return PAMTRA_B200_FATAL;
  ctx->spin_limit = polls;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_set_timing(pamtra_b200_ctx* ctx, int32_t enable) {
  if (!ctx) return PAMTRA_B200_FATAL;
  ctx->timing = enable ? 1 : 0;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_stage_ms(pamtra_b200_ctx* ctx, float* ms, int32_t n) {
  if (!ctx || !ms) return PAMTRA_B200_FATAL;
  for (int i = 0; i < n; i++) ms[i] = 0.f;
  if (ctx->nev < 2) return PAMTRA_B200_OK;
  if (cudaEventSynchronize(ctx->ev[ctx->nev - 1]) != cudaSuccess) return PAMTRA_B200_FATAL;
  for (int i = 1; i < ctx->nev; i++) {
    float t = 0.f;
    cudaEventElapsedTime(&t, ctx->ev[i - 1], ctx->ev[i]);
    int st = ctx->ev_stage[i];
    if (st >= 0 && st < n) ms[st] += t;
  }
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_run(pamtra_b200_ctx* ctx, const pamtra_b200_settings* st, const pamtra_b200_columns* cols,
                        const pamtra_b200_outputs* out, int32_t precision, void* stream_) {
  if (!ctx || !st || !cols || !out || !out->tb) return PAMTRA_B200_FATAL;
  if (precision != PAMTRA_B200_PREC_FP64 && precision != PAMTRA_B200_PREC_3XTF32 &&
      precision != PAMTRA_B200_PREC_FP64_BATCHED && precision != PAMTRA_B200_PREC_3XTF32_FP64ADD)
    return PAMTRA_B200_FATAL;
  const bool one_inv = precision != PAMTRA_B200_PREC_FP64;  // one inverse per adding combine
  // split precision: 3xTF32 doubling (and, for PREC_3XTF32, adding of NUMMU 16)
  const bool split = precision == PAMTRA_B200_PREC_3XTF32 || precision == PAMTRA_B200_PREC_3XTF32_FP64ADD;
  if (cols->ncol < 1 || cols->max_nlyrs < 2 || cols->max_nfreq < 1 || cols->noutlevels < 1 || cols->nhydro < 0)
    return PAMTRA_B200_FATAL;
  if (cols->nhydro > 0 && !cols->species) return PAMTRA_B200_FATAL;
  if (!(st->nummu == 8 || st->nummu == 16 || st->nummu == 32)) return PAMTRA_B200_FATAL;
  if (st->liq_mod < PAMTRA_B200_LIQ_TKC || st->liq_mod > PAMTRA_B200_LIQ_STO ||
      (st->gas_mod != PAMTRA_B200_GAS_R98 && st->gas_mod != PAMTRA_B200_GAS_L93))
    return PAMTRA_B200_FATAL;
  if (cols->fs_d && (cols->fs_nbin < 1 || !cols->fs_d_bound || !cols->fs_n || !cols->fs_rho || !cols->fs_mass))
    return PAMTRA_B200_FATAL;
  if (out->psd_d && (out->psd_nbin < 1 || !out->psd_deltad || !out->psd_n || !out->psd_mass || !out->psd_area ||
                     !out->psd_bscat))
    return PAMTRA_B200_FATAL;
  cudaStream_t stream = (cudaStream_t)stream_;
  cudaSetDevice(ctx->device);
  pamtra_b200_species dummy{};
  pamtra_b200_columns cc = *cols;
  if (cc.nhydro == 0) { cc.species = &dummy; cc.species_stride = 0; }
  Plan pl = make_plan(&cc, st->nummu, ctx->sm_count, ctx->sm_count * MIE_SLAB_WARPS_PER_SM, split,
                      precision == PAMTRA_B200_PREC_3XTF32);
  if (pl.max_nbin > MAXBIN) return PAMTRA_B200_FATAL;
  if (pl.total > ctx->arena_bytes) {
    cudaStreamSynchronize(stream);
    if (pamtra_b200_reserve(ctx, pl.total + pl.total / 8)) return PAMTRA_B200_FATAL;
  }
  const int mask = cc.nummu_mask ? cc.nummu_mask : (st->nummu == 8 ? 1 : st->nummu == 16 ? 2 : 4);
  if (pl.maxN > cc.max_nummu) return PAMTRA_B200_FATAL;
  char* A = ctx->arena;
  // species table -> device.  The table the previous run left in the arena is
  // reused when it is byte-identical and at the same place (no host wait, so
  // steady-state runs can be captured in a CUDA graph); otherwise it goes
  // through a ring of pinned staging buffers, waiting only for a buffer whose
  // previous copy is still queued.
  const size_t nsp = cc.species_stride ? (size_t)cc.ncol * cc.nhydro : (size_t)std::max(cc.nhydro, 1);
  const size_t spb = nsp * sizeof(pamtra_b200_species);
  pamtra_b200_species* d_species = (pamtra_b200_species*)(A + pl.o_species);
  const bool cached = ctx->sp_last_arena == A && ctx->sp_last_off == pl.o_species && ctx->sp_last.size() == spb &&
                      std::memcmp(ctx->sp_last.data(), cc.species, spb) == 0;
  if (!cached) {
    pamtra_b200_ctx::SpStage& sg = ctx->sp_ring[ctx->sp_next];
    ctx->sp_next = (ctx->sp_next + 1) % pamtra_b200_ctx::NSP_RING;
    if (sg.used && cudaEventSynchronize(sg.ev) != cudaSuccess) return PAMTRA_B200_FATAL;
    if (spb > sg.cap) {
      if (sg.h) cudaFreeHost(sg.h);
      sg.h = nullptr;
      sg.cap = 0;
      if (cudaMallocHost(&sg.h, spb) != cudaSuccess) return PAMTRA_B200_FATAL;
      sg.cap = spb;
    }
    if (!sg.ev && cudaEventCreateWithFlags(&sg.ev, cudaEventDisableTiming) != cudaSuccess) return PAMTRA_B200_FATAL;
    std::memcpy(sg.h, cc.species, spb);
    cudaMemcpyAsync(d_species, sg.h, spb, cudaMemcpyHostToDevice, stream);
    cudaEventRecord(sg.ev, stream);
    sg.used = 1;
    ctx->sp_last.assign((const unsigned char*)cc.species, (const unsigned char*)cc.species + spb);
    ctx->sp_last_arena = A;
    ctx->sp_last_off = pl.o_species;
  }

  Batch b{};
  b.ncol = cc.ncol; b.max_nlyrs = cc.max_nlyrs; b.nhydro = cc.nhydro; b.max_nfreq = cc.max_nfreq;
  b.noutlevels = cc.noutlevels; b.max_nummu = cc.max_nummu; b.max_nbin = pl.max_nbin;
  b.species_stride = cc.species_stride; b.default_nummu = st->nummu; b.species = d_species;
  b.nummu_mask = mask;
  b.nlyrs = cc.nlyrs; b.nummu = cc.nummu; b.nfreq = cc.nfreq; b.freqs = cc.freqs; b.freq_per_col = cc.nfreq != nullptr;
  b.hgt_lev = cc.hgt_lev; b.temp_lev = cc.temp_lev; b.press_lev = cc.press_lev; b.relhum_lev = cc.relhum_lev;
  b.hgt = cc.hgt; b.temp = cc.temp; b.press = cc.press; b.relhum = cc.relhum;
  b.hydro_q = cc.hydro_q; b.hydro_n = cc.hydro_n; b.hydro_reff = cc.hydro_reff;
  b.groundtemp = cc.groundtemp; b.obs_height = cc.obs_height; b.sfc_refl = cc.sfc_refl;
  b.fs_nbin = cc.fs_nbin; b.fs_d = cc.fs_d; b.fs_d_bound = cc.fs_d_bound; b.fs_n = cc.fs_n; b.fs_rho = cc.fs_rho;
  b.fs_mass = cc.fs_mass;

  Work w{};
  w.hgt_lev = (double*)(A + pl.o_hgt_lev); w.temp_lev = (double*)(A + pl.o_temp_lev);
  w.temp = (double*)(A + pl.o_temp); w.press = (double*)(A + pl.o_press);
  w.rho_vap = (double*)(A + pl.o_rho_vap); w.q_hum = (double*)(A + pl.o_q_hum); w.vap = (double*)(A + pl.o_vap);
  w.gtemp = (double*)(A + pl.o_gtemp); w.outlev = (int*)(A + pl.o_outlev); w.kgas = (double*)(A + pl.o_kgas);
  w.slot_st = (int8_t*)(A + pl.o_slot_st); w.slot_nb = (int*)(A + pl.o_slot_nb);
  w.b_d = (double*)(A + pl.o_bd); w.b_dd = (double*)(A + pl.o_bdd); w.b_nd = (double*)(A + pl.o_bnd);
  w.b_rho = (double*)(A + pl.o_brho); w.b_mass = (double*)(A + pl.o_bmass);
  w.psd_d = out->psd_d; w.psd_dd = out->psd_deltad; w.psd_n = out->psd_n; w.psd_mass = out->psd_mass;
  w.psd_area = out->psd_area; w.psd_bscat = out->psd_bscat; w.psd_nbin = out->psd_nbin;
  w.pres_idx = (int*)(A + pl.o_pres_idx); w.plist = (int*)(A + pl.o_plist); w.pmax = pl.pmax;
  w.counters = (int*)(A + pl.o_counters);
  w.m_kext = (double*)(A + pl.o_mkext); w.m_salb = (double*)(A + pl.o_msalb); w.m_nleg = (int*)(A + pl.o_mnleg);
  w.m_back = (double*)(A + pl.o_mback); w.m_refr = (double*)(A + pl.o_mrefr);
  w.m_legen = pl.f32_coef ? nullptr : (double*)(A + pl.o_mlegen);
  w.m_legen32 = pl.f32_coef ? (float*)(A + pl.o_mlegen) : nullptr;
  w.lay = (double*)(A + pl.o_lay); w.lay_stride = pl.lay_stride; w.lay_nd = (int*)(A + pl.o_laynd);
  w.lay32 = pl.tc_add ? 1 : 0;
  w.add_stk = pl.tc_add ? (float*)(A + pl.o_addstk) : nullptr;
  w.status = (int*)(A + pl.o_status); w.col_status = (int*)(A + pl.o_colst);
  w.add_scr = (double*)(A + pl.o_addscr);
  w.mie_slab = (double*)(A + pl.o_mieslab); w.mie_nslab = pl.mie_nslab;
  w.spin_limit = ctx->spin_limit;
  ctx->last_counters = w.counters;
  // scatcnv weight tables (context-resident; a table that cannot be allocated
  // leaves the direct azimuth sums in place)
  if (cc.nhydro > 0) {
    if (!ctx->wt_flags && cudaMalloc(&ctx->wt_flags, 2 * 3 * SCAT_NPI * sizeof(int)) == cudaSuccess)
      cudaMemsetAsync(ctx->wt_flags, 0, 2 * 3 * SCAT_NPI * sizeof(int), stream);
    const int Ns[3] = {8, 16, 32};
    for (int i = 0; i < 3; i++)
      if (ctx->wt_flags && (mask & (1 << i)) && !ctx->wtab[i] &&
          cudaMalloc(&ctx->wtab[i], scat_weight_doubles(Ns[i]) * sizeof(double)) != cudaSuccess) {
        ctx->wtab[i] = nullptr;
        cudaGetLastError();
      }
  }
  for (int i = 0; i < 3; i++) w.wtab[i] = ctx->wt_flags ? ctx->wtab[i] : nullptr;
  w.wt_need = ctx->wt_flags;
  w.wt_ready = ctx->wt_flags ? ctx->wt_flags + 3 * SCAT_NPI : nullptr;
  w.gq_x = ctx->gq_x; w.gq_w = ctx->gq_w; w.gq_max = GQ_MAX; w.lob_mu = ctx->lob_mu; w.lob_w = ctx->lob_w;

  int launches = 0;
  ctx->nev = 0;
  const size_t C = cc.ncol, Lm = cc.max_nlyrs, Fm = cc.max_nfreq, H = cc.nhydro;
  mark(ctx, stream, -1);
  cudaMemsetAsync(w.counters, 0, 16 * 4, stream);
  cudaMemsetAsync(w.status, 0, C * Fm * 4, stream);
  cudaMemsetAsync(w.col_status, 0, C * 4, stream);
  const size_t ntb = C * cc.noutlevels * 2 * cc.max_nummu * Fm * 2;
  k_fill_d<<<(unsigned)((ntb + 255) / 256), 256, 0, stream>>>(out->tb, -9999.0, ntb); launches++;
  if (w.psd_d && H > 0) {
    const size_t npsd = C * Lm * H * (size_t)w.psd_nbin;
    for (double* a : {w.psd_d, w.psd_dd, w.psd_n, w.psd_mass, w.psd_area, w.psd_bscat}) {
      k_fill_d<<<(unsigned)((npsd + 255) / 256), 256, 0, stream>>>(a, -9999.0, npsd);
      launches++;
    }
  }
  k_atmo<<<(unsigned)((C + 127) / 128), 128, 0, stream>>>(b, w); launches++;
  const size_t ngas = C * Fm * Lm;
  k_gas<<<(unsigned)((ngas + 255) / 256), 256, 0, stream>>>(b, w, st->lgas_extinction, st->gas_mod); launches++;
  mark(ctx, stream, STG_PREP);
  if (H > 0) {
    const size_t ns = C * Lm * H;
    if (cc.fs_d) k_fullspec<<<(unsigned)((ns + 127) / 128), 128, 0, stream>>>(b, w, *st);
    else k_psd<<<(unsigned)((ns + 127) / 128), 128, 0, stream>>>(b, w, *st);
    launches++;
  } else {
    cudaMemsetAsync(w.slot_st, 0, 1, stream);
  }
  k_compact<<<1, 1024, 0, stream>>>(b, w); launches++;
  mark(ctx, stream, STG_PSD);
  const int sms = ctx->sm_count;
  if (H > 0) {
    const int mw = ctx->mie_warps;
    const size_t sm_mie = mw * sizeof(MieSmem);
    const void* kmie = ctx->mie_group == 8 ? (const void*)k_mie<8> : (const void*)k_mie<4>;
    int g = std::min(persistent_grid(kmie, 32 * mw, sm_mie, sms, ctx->mie_cps), std::max(1, pl.mie_nslab / mw));
    const size_t nref = (size_t)std::max(1, pl.pmax) * Fm;
    k_refr<<<(unsigned)((nref + 127) / 128), 128, 0, stream>>>(b, w, *st); launches++;
    if (ctx->mie_group == 8) k_mie<8><<<g, 32 * mw, sm_mie, stream>>>(b, w, *st);
    else k_mie<4><<<g, 32 * mw, sm_mie, stream>>>(b, w, *st);
    launches++;
    if (w.wtab[0] && (mask & 1)) {
      k_scat_weights<8><<<SCAT_NPI * ((2 * 8 * 8 + 127) / 128), 128, 0, stream>>>(ctx->wtab[0], w.wt_need, w.wt_ready, ctx->lob_mu);
      launches++;
    }
    if (w.wtab[1] && (mask & 2)) {
      k_scat_weights<16><<<SCAT_NPI * ((2 * 16 * 16 + 127) / 128), 128, 0, stream>>>(ctx->wtab[1], w.wt_need, w.wt_ready, ctx->lob_mu);
      launches++;
    }
    if (w.wtab[2] && (mask & 4)) {
      k_scat_weights<32><<<SCAT_NPI * ((2 * 32 * 32 + 127) / 128), 128, 0, stream>>>(ctx->wtab[2], w.wt_need, w.wt_ready, ctx->lob_mu);
      launches++;
    }
  }
  mark(ctx, stream, STG_MIE);
  double* ssp = out->scatter_matrix;
  if (mask & 1) {
    int g = persistent_grid((const void*)k_layer<8>, RTCfg<8>::T, sizeof(LayerSmem<8>), sms, ctx->layer_cps);
    if (H > 0) { k_layer<8><<<g, RTCfg<8>::T, sizeof(LayerSmem<8>), stream>>>(b, w, *st, ssp); launches++; }
    mark(ctx, stream, STG_LAYER);
    g = persistent_grid((const void*)k_adding<8>, RTCfg<8>::T, sizeof(AddSmem<8>), sms, ctx->adding_cps);
    if (one_inv) k_adding<8, true><<<g, RTCfg<8>::T, sizeof(AddSmem<8>), stream>>>(b, w, *st, *out);
    else k_adding<8><<<g, RTCfg<8>::T, sizeof(AddSmem<8>), stream>>>(b, w, *st, *out);
    launches++;
    mark(ctx, stream, STG_ADDING);
  }
  if (mask & 2) {
    if (H > 0 && split) {
      // three CTAs (three item pairs) per SM by shared memory, registers and
      // tensor memory (3 x 128 columns); the persistent CTAs take pairs of
      // items from a counter
      const size_t smb = layer_tc_smem<16>();
      const int g = (ctx->layer_cps > 0 ? std::min(ctx->layer_cps, 3) : 3) * sms;
      k_layer_tc<16><<<g, 128, smb, stream>>>(b, w, *st, ssp); launches++;
    } else if (H > 0) {
      int g = persistent_grid((const void*)k_layer<16>, RTCfg<16>::T, sizeof(LayerSmem<16>), sms, ctx->layer_cps);
      k_layer<16><<<g, RTCfg<16>::T, sizeof(LayerSmem<16>), stream>>>(b, w, *st, ssp); launches++;
    }
    mark(ctx, stream, STG_LAYER);
    if (pl.tc_add) {
      // two CTAs (two unit pairs) per SM by shared memory and tensor memory
      // (2 x 256 columns); the FP64 surface and radiance part follows
      k_adding_tc<16><<<2 * sms, 128, add_tc_smem(), stream>>>(b, w, *st);
      const int gf = persistent_grid((const void*)k_adding_finish<16>, RTCfg<16>::T, sizeof(AddSmem<16>), sms, 0);
      k_adding_finish<16><<<gf, RTCfg<16>::T, sizeof(AddSmem<16>), stream>>>(b, w, *st, *out);
      launches += 2;
    } else {
      const int g = persistent_grid((const void*)k_adding<16>, RTCfg<16>::T, sizeof(AddSmem<16>), sms, ctx->adding_cps);
      if (one_inv) k_adding<16, true><<<g, RTCfg<16>::T, sizeof(AddSmem<16>), stream>>>(b, w, *st, *out);
      else k_adding<16><<<g, RTCfg<16>::T, sizeof(AddSmem<16>), stream>>>(b, w, *st, *out);
      launches++;
    }
    mark(ctx, stream, STG_ADDING);
  }
  if (mask & 4) {
    int g = persistent_grid((const void*)k_layer<32>, RTCfg<32>::T, sizeof(LayerSmem<32>), sms, ctx->layer_cps);
    if (H > 0 && split) {
      // one item per CTA, one CTA per SM (165 KB shared memory, 256 TMEM columns)
      k_layer_tc64<<<sms, 256, layer_tc64_smem(), stream>>>(b, w, *st, ssp); launches++;
    } else if (H > 0) {
      k_layer<32><<<g, RTCfg<32>::T, sizeof(LayerSmem<32>), stream>>>(b, w, *st, ssp); launches++;
    }
    mark(ctx, stream, STG_LAYER);
    g = std::min(persistent_grid((const void*)k_adding<32>, RTCfg<32>::T, sizeof(AddSmem<32>), sms, ctx->adding_cps),
                 pl.add_grid);
    if (one_inv) k_adding<32, true><<<g, RTCfg<32>::T, sizeof(AddSmem<32>), stream>>>(b, w, *st, *out);
    else k_adding<32><<<g, RTCfg<32>::T, sizeof(AddSmem<32>), stream>>>(b, w, *st, *out);
    launches++;
    mark(ctx, stream, STG_ADDING);
  }
  if (out->angles_deg) { k_angles<<<1, 32, 0, stream>>>(out->angles_deg, ctx->lob_mu, cc.max_nummu); launches++; }
  if (out->kexttot || out->salbedo || out->num_doubles) {
    k_ssp_out<<<(unsigned)((ngas + 255) / 256), 256, 0, stream>>>(b, w, *out); launches++;
  }
  if (out->kextatmo) cudaMemcpyAsync(out->kextatmo, w.kgas, ngas * 8, cudaMemcpyDeviceToDevice, stream);
  if (st->active && (out->ze || out->att_hydro || out->att_atmo)) {
    k_radar<<<(unsigned)((C * Fm + 127) / 128), 128, 0, stream>>>(b, w, *st, *out); launches++;
  }
  if (out->status) {
    k_status_out<<<(unsigned)((C * Fm + 255) / 256), 256, 0, stream>>>(w, out->status, (int)(C * Fm)); launches++;
  }
  mark(ctx, stream, STG_PREP);
  ctx->last_launches = launches;
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

int32_t pamtra_b200_run_host(pamtra_b200_ctx* ctx, const pamtra_b200_settings* st, const pamtra_b200_columns* hc,
                             const pamtra_b200_outputs* ho, int32_t precision, void* stream_) {
  if (!ctx || !st || !hc || !ho || !ho->tb) return PAMTRA_B200_FATAL;
  if (hc->fs_d && (hc->fs_nbin < 1 || !hc->fs_d_bound || !hc->fs_n || !hc->fs_rho || !hc->fs_mass))
    return PAMTRA_B200_FATAL;
  if (ho->psd_d && (ho->psd_nbin < 1 || !ho->psd_deltad || !ho->psd_n || !ho->psd_mass || !ho->psd_area ||
                    !ho->psd_bscat))
    return PAMTRA_B200_FATAL;
  cudaStream_t stream = (cudaStream_t)stream_;
  cudaSetDevice(ctx->device);
  const size_t C = hc->ncol, Lm = hc->max_nlyrs, Fm = hc->max_nfreq, H = hc->nhydro, NO = hc->noutlevels;
  const size_t NA = 2 * (size_t)hc->max_nummu;
  struct Seg { const void* h; size_t bytes; size_t off; };
  std::vector<Seg> in;
  size_t off = 0;
  auto add = [&](const void* h, size_t bytes) -> size_t {
    size_t o = (off + 255) & ~(size_t)255;
    off = o + bytes;
    if (h) in.push_back({h, bytes, o});
    return o;
  };
  const size_t nfq = hc->nfreq ? C * Fm : Fm;
  size_t o_nly = add(hc->nlyrs, C * 4), o_nmu = add(hc->nummu, hc->nummu ? C * 4 : 0);
  size_t o_nfr = add(hc->nfreq, hc->nfreq ? C * 4 : 0), o_frq = add(hc->freqs, nfq * 8);
  size_t o_hl = add(hc->hgt_lev, C * (Lm + 1) * 8), o_tl = add(hc->temp_lev, C * (Lm + 1) * 8);
  size_t o_pl = add(hc->press_lev, C * (Lm + 1) * 8), o_rl = add(hc->relhum_lev, C * (Lm + 1) * 8);
  size_t o_h = add(hc->hgt, C * Lm * 8), o_t = add(hc->temp, C * Lm * 8), o_p = add(hc->press, C * Lm * 8);
  size_t o_r = add(hc->relhum, C * Lm * 8);
  size_t o_q = add(hc->hydro_q, C * Lm * H * 8), o_n = add(hc->hydro_n, C * Lm * H * 8);
  size_t o_re = add(hc->hydro_reff, C * Lm * H * 8);
  size_t o_g = add(hc->groundtemp, C * 8), o_ob = add(hc->obs_height, C * NO * 8), o_sr = add(hc->sfc_refl, C);
  const size_t FB = hc->fs_d ? C * Lm * H * (size_t)hc->fs_nbin : 0;
  size_t o_fd = add(hc->fs_d, FB * 8), o_fdb = add(hc->fs_d ? hc->fs_d_bound : nullptr, (FB + C * Lm * H) * 8);
  size_t o_fn = add(hc->fs_d ? hc->fs_n : nullptr, FB * 8), o_fr = add(hc->fs_d ? hc->fs_rho : nullptr, FB * 8);
  size_t o_fm = add(hc->fs_d ? hc->fs_mass : nullptr, FB * 8);
  size_t o_tb = add(nullptr, C * NO * NA * Fm * 2 * 8);
  size_t o_em = add(nullptr, ho->emissivity ? C * 2 * Fm * hc->max_nummu * 8 : 0);
  size_t o_an = add(nullptr, ho->angles_deg ? NA * 8 : 0);
  size_t o_st = add(nullptr, ho->status ? C * Fm * 4 : 0);
  size_t o_ka = add(nullptr, ho->kextatmo ? C * Fm * Lm * 8 : 0);
  size_t o_kt = add(nullptr, ho->kexttot ? C * Fm * Lm * 8 : 0);
  size_t o_sa = add(nullptr, ho->salbedo ? C * Fm * Lm * 8 : 0);
  size_t o_sc = add(nullptr, ho->scatter_matrix ? C * Fm * Lm * 4 * NA * NA * 8 : 0);
  size_t o_nd = add(nullptr, ho->num_doubles ? C * Fm * Lm * 4 : 0);
  size_t o_ze = add(nullptr, ho->ze ? C * Fm * Lm * 8 : 0);
  size_t o_ah = add(nullptr, ho->att_hydro ? C * Fm * Lm * 8 : 0);
  size_t o_aa = add(nullptr, ho->att_atmo ? C * Fm * Lm * 8 : 0);
  const size_t NP = ho->psd_d ? C * Lm * H * (size_t)ho->psd_nbin : 0;
  size_t o_psd[6];
  for (int i = 0; i < 6; i++) o_psd[i] = add(nullptr, NP * 8);
  if (off > ctx->stage_bytes) {
    cudaStreamSynchronize(stream);
    cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    if (cudaMalloc(&ctx->stage, off + off / 8) != cudaSuccess) return PAMTRA_B200_FATAL;
    ctx->stage_bytes = off + off / 8;
  }
  char* D = ctx->stage;
  for (auto& s : in) cudaMemcpyAsync(D + s.off, s.h, s.bytes, cudaMemcpyHostToDevice, stream);
  pamtra_b200_columns dc = *hc;
  auto dp = [&](const void* h, size_t o) -> const void* { return h ? (const void*)(D + o) : nullptr; };
  dc.nlyrs = (const int32_t*)dp(hc->nlyrs, o_nly);
  dc.nummu = (const int32_t*)dp(hc->nummu, o_nmu);
  dc.nfreq = (const int32_t*)dp(hc->nfreq, o_nfr);
  dc.freqs = (const double*)dp(hc->freqs, o_frq);
  dc.hgt_lev = (const double*)dp(hc->hgt_lev, o_hl);
  dc.temp_lev = (const double*)dp(hc->temp_lev, o_tl);
  dc.press_lev = (const double*)dp(hc->press_lev, o_pl);
  dc.relhum_lev = (const double*)dp(hc->relhum_lev, o_rl);
  dc.hgt = (const double*)dp(hc->hgt, o_h);
  dc.temp = (const double*)dp(hc->temp, o_t);
  dc.press = (const double*)dp(hc->press, o_p);
  dc.relhum = (const double*)dp(hc->relhum, o_r);
  dc.hydro_q = (const double*)dp(hc->hydro_q, o_q);
  dc.hydro_n = (const double*)dp(hc->hydro_n, o_n);
  dc.hydro_reff = (const double*)dp(hc->hydro_reff, o_re);
  dc.groundtemp = (const double*)dp(hc->groundtemp, o_g);
  dc.obs_height = (const double*)dp(hc->obs_height, o_ob);
  dc.sfc_refl = (const int8_t*)dp(hc->sfc_refl, o_sr);
  if (hc->fs_d) {
    dc.fs_d = (const double*)(D + o_fd);
    dc.fs_d_bound = (const double*)(D + o_fdb);
    dc.fs_n = (const double*)(D + o_fn);
    dc.fs_rho = (const double*)(D + o_fr);
    dc.fs_mass = (const double*)(D + o_fm);
  }
  pamtra_b200_outputs dout{};
  dout.tb = (double*)(D + o_tb);
  dout.emissivity = ho->emissivity ? (double*)(D + o_em) : nullptr;
  dout.angles_deg = ho->angles_deg ? (double*)(D + o_an) : nullptr;
  dout.status = ho->status ? (int32_t*)(D + o_st) : nullptr;
  dout.kextatmo = ho->kextatmo ? (double*)(D + o_ka) : nullptr;
  dout.kexttot = ho->kexttot ? (double*)(D + o_kt) : nullptr;
  dout.salbedo = ho->salbedo ? (double*)(D + o_sa) : nullptr;
  dout.scatter_matrix = ho->scatter_matrix ? (double*)(D + o_sc) : nullptr;
  dout.num_doubles = ho->num_doubles ? (int32_t*)(D + o_nd) : nullptr;
  dout.ze = ho->ze ? (double*)(D + o_ze) : nullptr;
  dout.att_hydro = ho->att_hydro ? (double*)(D + o_ah) : nullptr;
  dout.att_atmo = ho->att_atmo ? (double*)(D + o_aa) : nullptr;
  if (ho->psd_d) {
    dout.psd_nbin = ho->psd_nbin;
    dout.psd_d = (double*)(D + o_psd[0]);
    dout.psd_deltad = (double*)(D + o_psd[1]);
    dout.psd_n = (double*)(D + o_psd[2]);
    dout.psd_mass = (double*)(D + o_psd[3]);
    dout.psd_area = (double*)(D + o_psd[4]);
    dout.psd_bscat = (double*)(D + o_psd[5]);
  }
  if (dout.scatter_matrix) cudaMemsetAsync(dout.scatter_matrix, 0, C * Fm * Lm * 4 * NA * NA * 8, stream);
  int32_t rc = pamtra_b200_run(ctx, st, &dc, &dout, precision, stream);
  if (rc != PAMTRA_B200_OK) return rc;
  cudaMemcpyAsync(ho->tb, dout.tb, C * NO * NA * Fm * 2 * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->emissivity) cudaMemcpyAsync(ho->emissivity, dout.emissivity, C * 2 * Fm * hc->max_nummu * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->angles_deg) cudaMemcpyAsync(ho->angles_deg, dout.angles_deg, NA * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->status) cudaMemcpyAsync(ho->status, dout.status, C * Fm * 4, cudaMemcpyDeviceToHost, stream);
  if (ho->kextatmo) cudaMemcpyAsync(ho->kextatmo, dout.kextatmo, C * Fm * Lm * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->kexttot) cudaMemcpyAsync(ho->kexttot, dout.kexttot, C * Fm * Lm * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->salbedo) cudaMemcpyAsync(ho->salbedo, dout.salbedo, C * Fm * Lm * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->scatter_matrix)
    cudaMemcpyAsync(ho->scatter_matrix, dout.scatter_matrix, C * Fm * Lm * 4 * NA * NA * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->num_doubles) cudaMemcpyAsync(ho->num_doubles, dout.num_doubles, C * Fm * Lm * 4, cudaMemcpyDeviceToHost, stream);
  if (ho->ze) cudaMemcpyAsync(ho->ze, dout.ze, C * Fm * Lm * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->att_hydro) cudaMemcpyAsync(ho->att_hydro, dout.att_hydro, C * Fm * Lm * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->att_atmo) cudaMemcpyAsync(ho->att_atmo, dout.att_atmo, C * Fm * Lm * 8, cudaMemcpyDeviceToHost, stream);
  if (ho->psd_d) {
    cudaMemcpyAsync(ho->psd_d, dout.psd_d, NP * 8, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(ho->psd_deltad, dout.psd_deltad, NP * 8, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(ho->psd_n, dout.psd_n, NP * 8, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(ho->psd_mass, dout.psd_mass, NP * 8, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(ho->psd_area, dout.psd_area, NP * 8, cudaMemcpyDeviceToHost, stream);
    cudaMemcpyAsync(ho->psd_bscat, dout.psd_bscat, NP * 8, cudaMemcpyDeviceToHost, stream);
  }
  if (cudaStreamSynchronize(stream) != cudaSuccess) return PAMTRA_B200_FATAL;
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_gas_r98(const double* freq, const double* temp, const double* rho_vap, const double* press,
                            double* kext, int32_t* status, int32_t n, void* stream) {
  if (n <= 0) return PAMTRA_B200_OK;
  k_gas_elem<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(freq, temp, rho_vap, press, kext, status, n);
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

__global__ void k_tkc_elem(const double* tc, const double* f, double* re, double* im, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  cplx e = eps_water_tkc(tc[i], f[i]);
  re[i] = e.re;
  im[i] = e.im;
}

int32_t pamtra_b200_eps_water_tkc(const double* t_c, const double* freq, double* eps_re, double* eps_im, int32_t n,
                                  void* stream) {
  if (n <= 0) return PAMTRA_B200_OK;
  k_tkc_elem<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(t_c, freq, eps_re, eps_im, n);
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

__global__ void k_eps_water_elem(int liq_mod, const double* s, const double* tc, const double* f, double* re,
                                 double* im, int32_t* st, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int bad = 0;
  cplx e;
  switch (liq_mod) {
    case PAMTRA_B200_LIQ_ELL: e = eps_water_ellison(s[i], tc[i], f[i]); break;
    case PAMTRA_B200_LIQ_LIE: e = eps_water_liebe(tc[i], f[i]); break;
    case PAMTRA_B200_LIQ_RAY: e = eps_water_ray(tc[i], f[i], &bad); break;
    case PAMTRA_B200_LIQ_STO: e = eps_water_stogryn(s[i], tc[i], f[i]); break;
    default: e = eps_water_tkc(tc[i], f[i]); break;
  }
  re[i] = e.re;
  im[i] = e.im;
  if (st) st[i] = bad ? (PAMTRA_B200_FATAL | PAMTRA_B200_ST_RANGE) : 0;
}

int32_t pamtra_b200_get_eps_water(int32_t liq_mod, const double* s, const double* t_c, const double* freq,
                                  double* eps_re, double* eps_im, int32_t* status, int32_t n, void* stream) {
  if (n <= 0) return PAMTRA_B200_OK;
  if (liq_mod < PAMTRA_B200_LIQ_TKC || liq_mod > PAMTRA_B200_LIQ_STO || !s) return PAMTRA_B200_FATAL;
  k_eps_water_elem<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(liq_mod, s, t_c, freq, eps_re, eps_im, status,
                                                                     n);
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

__global__ void k_l93_elem(const double* f, const double* p, const double* e, const double* T, double* k, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  k[i] = gas_l93(f[i], p[i], e[i], T[i]);
}

int32_t pamtra_b200_gas_l93(const double* freq, const double* press, const double* vap, const double* temp,
                            double* kext, int32_t n, void* stream) {
  if (n <= 0) return PAMTRA_B200_OK;
  k_l93_elem<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(freq, press, vap, temp, kext, n);
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

// ---------------------------------------------------------------- T-matrix branch
int32_t pamtra_b200_tmatrix(pamtra_b200_ctx* ctx, const pamtra_b200_tmatrix_in* in, pamtra_b200_tmatrix_out* out,
                            void* stream_) {
  if (!ctx || !in || !out) return PAMTRA_B200_FATAL;
  const int ni = in->n_items, nb = in->nbins, nummu = in->nummu;
  if (ni <= 0 || nb <= 0) return PAMTRA_B200_OK;
  if (nummu != 8 && nummu != 16 && nummu != 32) return PAMTRA_B200_FATAL;
  if ((size_t)ni * nb > (size_t)INT32_MAX / 4) return PAMTRA_B200_FATAL;
  cudaSetDevice(ctx->device);
  cudaStream_t stream = (cudaStream_t)stream_;
  const size_t n = (size_t)ni * nb;
  const size_t NS = (size_t)2 * nummu * 2 * nummu * 2, NE = 4 * (size_t)nummu, NM = 2 * (size_t)nummu;
  // two 256-thread CTAs per SM (128 registers per thread), persistent
  const int grid = (int)std::min<size_t>(n, (size_t)2 * ctx->sm_count);
  // device layout (8-byte units, each array 256-byte aligned)
  size_t off = 0;
  auto take = [&](size_t elems8) { const size_t o = off; off += (elems8 + 31) / 32 * 32; return o; };
  const bool host = !in->on_device;
  const size_t o_freq = take(ni), o_rre = take(ni), o_rim = take(ni), o_phase = take((ni + 1) / 2);
  const size_t o_dmax = take(n), o_dd = take(n), o_nd = take(n), o_rho = take(n), o_asr = take(n), o_cant = take(n);
  const size_t o_mrr = take(n), o_mri = take(n), o_axi = take(n), o_nde = take(n), o_pst = take((n + 1) / 2),
               o_pnm = take((n + 1) / 2);
  const size_t o_pscat = take(n * NS), o_pext = take(n * NE), o_pemis = take(n * NM), o_psb = take(n * 4);
  const size_t o_scat = take((size_t)ni * NS), o_ext = take((size_t)ni * NE), o_emis = take((size_t)ni * NM),
               o_sb = take((size_t)ni * 4), o_back = take(n), o_st = take(((size_t)ni + 1) / 2), o_cnt = take(1);
  const size_t o_slot = take((size_t)grid * TM_SLOT_DOUBLES);
  const size_t bytes = off * 8;
  if (bytes > ctx->tm_bytes) {
    cudaStreamSynchronize(stream);
    cudaFree(ctx->tm_buf);
    ctx->tm_buf = nullptr;
    ctx->tm_bytes = 0;
    if (cudaMalloc(&ctx->tm_buf, bytes) != cudaSuccess) return PAMTRA_B200_FATAL;
    ctx->tm_bytes = bytes;
  }
  char* B = ctx->tm_buf;
  auto D = [&](size_t o) { return reinterpret_cast<double*>(B + o * 8); };
  auto I = [&](size_t o) { return reinterpret_cast<int*>(B + o * 8); };
  const double *freq = in->freq, *rre = in->ref_re, *rim = in->ref_im, *dmax = in->dmax, *dd = in->del_d,
               *nd = in->ndens, *rho = in->density, *asr = in->as_ratio, *cant = in->canting;
  const int* phase = in->phase;
  if (host) {
    auto up = [&](size_t o, const void* src, size_t b) { cudaMemcpyAsync(B + o * 8, src, b, cudaMemcpyHostToDevice, stream); };
    up(o_freq, freq, ni * 8); up(o_rre, rre, ni * 8); up(o_rim, rim, ni * 8); up(o_phase, phase, ni * 4);
    up(o_dmax, dmax, n * 8); up(o_dd, dd, n * 8); up(o_nd, nd, n * 8); up(o_rho, rho, n * 8);
    up(o_asr, asr, n * 8); up(o_cant, cant, n * 8);
    freq = D(o_freq); rre = D(o_rre); rim = D(o_rim); phase = I(o_phase);
    dmax = D(o_dmax); dd = D(o_dd); nd = D(o_nd); rho = D(o_rho); asr = D(o_asr); cant = D(o_cant);
  }
  k_tmat_prep<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(ni, nb, freq, rre, rim, phase, dmax, dd, nd, rho, asr, cant,
                                                                D(o_mrr), D(o_mri), D(o_axi), D(o_nde), I(o_pst));
  cudaMemsetAsync(I(o_cnt), 0, 4, stream);
  TmArgs A;
  A.n_items = ni; A.nbins = nb; A.nummu = nummu;
  A.freq = freq; A.mrr = D(o_mrr); A.mri = D(o_mri); A.axi = D(o_axi); A.asr = asr; A.beta = cant; A.ndens = D(o_nde);
  A.mu = ctx->lob_mu + lob_off(nummu); A.wq = ctx->lob_w + lob_off(nummu);
  A.scat = D(o_pscat); A.ext = D(o_pext); A.emis = D(o_pemis); A.sback = D(o_psb);
  A.nmax = (!host && out->nmax) ? out->nmax : I(o_pnm);
  A.status = I(o_pst); A.scratch = D(o_slot); A.counter = I(o_cnt);
  k_tmatrix<<<grid, TM_THREADS, 0, stream>>>(A);
  double *scat = out->scatter_matrix, *ext = out->extinct_matrix, *emis = out->emis_vector, *sb = out->sback,
         *back = out->back_spec;
  int* st = out->status;
  if (host) {
    scat = D(o_scat); ext = D(o_ext); emis = D(o_emis); sb = D(o_sb); back = D(o_back); st = I(o_st);
  }
  k_tmat_sum<<<ni, 256, 0, stream>>>(ni, nb, nummu, D(o_nde), dd, D(o_pscat), D(o_pext), D(o_pemis), D(o_psb), I(o_pst),
                                     scat, ext, emis, sb, back, st);
  ctx->last_launches = 3;
  if (cudaGetLastError() != cudaSuccess) return PAMTRA_B200_FATAL;
  if (host) {
    auto dn = [&](void* dst, size_t o, size_t b) { cudaMemcpyAsync(dst, B + o * 8, b, cudaMemcpyDeviceToHost, stream); };
    dn(out->scatter_matrix, o_scat, (size_t)ni * NS * 8);
    dn(out->extinct_matrix, o_ext, (size_t)ni * NE * 8);
    dn(out->emis_vector, o_emis, (size_t)ni * NM * 8);
    dn(out->sback, o_sb, (size_t)ni * 4 * 8);
    dn(out->back_spec, o_back, n * 8);
    dn(out->status, o_st, (size_t)ni * 4);
    if (out->nmax) dn(out->nmax, o_pnm, n * 4);
    if (cudaStreamSynchronize(stream) != cudaSuccess) return PAMTRA_B200_FATAL;
  }
  return PAMTRA_B200_OK;
}

int32_t pamtra_b200_minvert_batched(const double* a, double* ainv, int32_t* status, int32_t n, int32_t count,
                                    void* stream) {
  if (count <= 0) return PAMTRA_B200_OK;
  cudaStream_t s = (cudaStream_t)stream;
  const int g = std::min(count, 65535);
  if (n == 16)
    k_minvert<16><<<g, Team<16>::T, Team<16>::MAT * 8 + sizeof(InvScratch<16>), s>>>(a, ainv, status, count);
  else if (n == 32)
    k_minvert<32><<<g, Team<32>::T, Team<32>::MAT * 8 + sizeof(InvScratch<32>), s>>>(a, ainv, status, count);
  else if (n == 64)
    k_minvert<64><<<g, Team<64>::T, Team<64>::MAT * 8 + sizeof(InvScratch<64>), s>>>(a, ainv, status, count);
  else return PAMTRA_B200_FATAL;
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

int32_t pamtra_b200_mmult_3xtf32_batched(const double* a, const double* b, double* c, int32_t n, int32_t count,
                                         int32_t* err, void* stream) {
  if (count <= 0) return PAMTRA_B200_OK;
  if (n != 32 || !a || !b || !c || !err) return PAMTRA_B200_FATAL;
  const int g = std::min(count, 65535);
  k_mmult_3xtf32<<<g, 128, (2 * 128 * 32 + 2 * 32 * 32) * sizeof(float), (cudaStream_t)stream>>>(a, b, c, count, err);
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}

}  // extern "C"

// ---------------------------------------------------------------- allocation-free single column
// Scratch of pamtra_b200_run_noalloc: a fixed, file-scope device array, so the
// entry point never calls an allocator.  Every GPU that loads this library
// holds it until the process exits.  Its capacity bounds the column sizes the
// entry point accepts (see PAMTRA_B200_NOALLOC_* in the header).
constexpr size_t NOALLOC_SCRATCH_BYTES = (size_t)PAMTRA_B200_NOALLOC_SCRATCH_MIB << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
// quadrature tables of the allocation-free path (filled at per-device set-up)
constexpr int NOALLOC_GQ = 256;
// k_mie warps of the allocation-free path (each takes a coefficient slab of the scratch)
constexpr int NOALLOC_MIE_SLABS = 16;
static __device__ __align__(256) double g_noalloc_tables[2 * (NOALLOC_GQ * (NOALLOC_GQ + 1) / 2) + 2 * 56];

namespace {
struct NoallocDevice {
  int ready = 0;
  char* scratch = nullptr;  // device address of g_noalloc_scratch
  double* tables = nullptr; // device address of g_noalloc_tables
};
NoallocDevice g_noalloc_dev[64];
std::mutex g_noalloc_mu;
}  // namespace

extern "C" int32_t pamtra_b200_run_noalloc(const pamtra_b200_settings* st, const pamtra_b200_columns* cols,
                                           const pamtra_b200_outputs* out, void* stream_) {
  if (!st || !cols || !out || !out->tb) return PAMTRA_B200_FATAL;
  cudaStream_t stream = (cudaStream_t)stream_;
  // size limits of the static scratch
  if (cols->ncol != 1 || cols->max_nlyrs < 2 || cols->max_nlyrs > PAMTRA_B200_NOALLOC_MAX_NLYRS ||
      cols->max_nfreq < 1 || cols->max_nfreq > PAMTRA_B200_NOALLOC_MAX_NFREQ || cols->nhydro < 0 ||
      cols->nhydro > PAMTRA_B200_NOALLOC_MAX_NHYDRO || cols->noutlevels < 1 || cols->noutlevels > 2 ||
      !(cols->max_nummu == 8 || cols->max_nummu == 16) || !(st->nummu == 8 || st->nummu == 16) ||
      (cols->nhydro > 0 && !cols->species) || cols->fs_d || out->psd_d || st->liq_mod < PAMTRA_B200_LIQ_TKC ||
      st->liq_mod > PAMTRA_B200_LIQ_STO || (st->gas_mod != PAMTRA_B200_GAS_R98 && st->gas_mod != PAMTRA_B200_GAS_L93))
    return PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return PAMTRA_B200_FATAL;
  NoallocDevice& D = g_noalloc_dev[dev];
  {
    // once per device, with that device current: resolve the device addresses
    // of the static arrays and fill the tables
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!D.ready) {
      void* sp = nullptr;
      void* tp = nullptr;
      if (cudaGetSymbolAddress(&sp, g_noalloc_scratch) != cudaSuccess) return PAMTRA_B200_FATAL;
      if (cudaGetSymbolAddress(&tp, g_noalloc_tables) != cudaSuccess) return PAMTRA_B200_FATAL;
      if (set_smem_attrs()) return PAMTRA_B200_FATAL;
      double* tab = (double*)tp;
      const size_t gqn = (size_t)NOALLOC_GQ * (NOALLOC_GQ + 1) / 2;
      k_gauss_table<<<NOALLOC_GQ, 128, 0, stream>>>(tab, tab + gqn);
      k_lobatto_table<<<3, 32, 0, stream>>>(tab + 2 * gqn, tab + 2 * gqn + 56);
      double la[MAXNLEG], lb[MAXNLEG];
      la[0] = 0.0;
      lb[0] = 0.0;
      for (int l = 1; l < MAXNLEG; l++) {
        la[l] = (2.0 * l - 1.0) / l;
        lb[l] = (l - 1.0) / l;
      }
      if (upload_mie_constants() || cudaMemcpyToSymbol(c_leg_a, la, sizeof(la)) || cudaMemcpyToSymbol(c_leg_b, lb, sizeof(lb)) ||
          cudaMemcpyToSymbol(c_o2_w300, H_O2_W300, sizeof(H_O2_W300)) ||
          cudaMemcpyToSymbol(c_o2_y300, H_O2_Y300, sizeof(H_O2_Y300)) ||
          cudaMemcpyToSymbol(c_o2_v, H_O2_V, sizeof(H_O2_V)) || cudaMemcpyToSymbol(c_o2_f, H_O2_F, sizeof(H_O2_F)) ||
          cudaMemcpyToSymbol(c_o2_s300, H_O2_S300, sizeof(H_O2_S300)) ||
          cudaMemcpyToSymbol(c_o2_be, H_O2_BE, sizeof(H_O2_BE)) ||
          cudaMemcpyToSymbol(c_h2o_fl, H_H2O_FL, sizeof(H_H2O_FL)) ||
          cudaMemcpyToSymbol(c_h2o_s1, H_H2O_S1, sizeof(H_H2O_S1)) ||
          cudaMemcpyToSymbol(c_h2o_b2, H_H2O_B2, sizeof(H_H2O_B2)) ||
          cudaMemcpyToSymbol(c_h2o_w3, H_H2O_W3, sizeof(H_H2O_W3)) ||
          cudaMemcpyToSymbol(c_h2o_x, H_H2O_X, sizeof(H_H2O_X)) ||
          cudaMemcpyToSymbol(c_h2o_ws, H_H2O_WS, sizeof(H_H2O_WS)) ||
          cudaMemcpyToSymbol(c_h2o_xs, H_H2O_XS, sizeof(H_H2O_XS)))
        return PAMTRA_B200_FATAL;
      if (cudaStreamSynchronize(stream) != cudaSuccess) return PAMTRA_B200_FATAL;
      D.scratch = (char*)sp;
      D.tables = tab;
      D.ready = 1;
    }
  }
  // scratch layout (same plan as the arena of pamtra_b200_run); bins are
  // sized for PAMTRA_B200_NOALLOC_MAX_NBIN
  pamtra_b200_columns cc = *cols;
  pamtra_b200_species plan_sp[PAMTRA_B200_NOALLOC_MAX_NHYDRO] = {};  // one entry per species slot make_plan reads
  for (auto& s : plan_sp) s.nbin = PAMTRA_B200_NOALLOC_MAX_NBIN;
  cc.species = plan_sp;
  cc.species_stride = 0;
  const int nh = cc.nhydro;
  cc.nhydro = nh > 0 ? nh : 0;
  Plan pl = make_plan(&cc, st->nummu, 0, NOALLOC_MIE_SLABS);
  // the widest quadrature launched must fit the caller's output rows (2 * max_nummu angles)
  if (pl.total > NOALLOC_SCRATCH_BYTES || pl.maxN > 16 || pl.maxN > cc.max_nummu)
    return PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE;
  const int mask = cc.nummu_mask ? cc.nummu_mask : (st->nummu == 8 ? 1 : 2);
  if (mask & ~3) return PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE;
  char* A = D.scratch;
  const size_t gqn = (size_t)NOALLOC_GQ * (NOALLOC_GQ + 1) / 2;
  Batch b{};
  b.ncol = 1; b.max_nlyrs = cc.max_nlyrs; b.nhydro = nh; b.max_nfreq = cc.max_nfreq;
  b.noutlevels = cc.noutlevels; b.max_nummu = cc.max_nummu; b.max_nbin = pl.max_nbin;
  b.species_stride = 0; b.default_nummu = st->nummu; b.species = cols->species;  // device pointer here
  b.nummu_mask = mask;
  b.nlyrs = cc.nlyrs; b.nummu = cc.nummu; b.nfreq = cc.nfreq; b.freqs = cc.freqs; b.freq_per_col = cc.nfreq != nullptr;
  b.hgt_lev = cc.hgt_lev; b.temp_lev = cc.temp_lev; b.press_lev = cc.press_lev; b.relhum_lev = cc.relhum_lev;
  b.hgt = cc.hgt; b.temp = cc.temp; b.press = cc.press; b.relhum = cc.relhum;
  b.hydro_q = cc.hydro_q; b.hydro_n = cc.hydro_n; b.hydro_reff = cc.hydro_reff;
  b.groundtemp = cc.groundtemp; b.obs_height = cc.obs_height; b.sfc_refl = cc.sfc_refl;
  Work w{};
  w.hgt_lev = (double*)(A + pl.o_hgt_lev); w.temp_lev = (double*)(A + pl.o_temp_lev);
  w.temp = (double*)(A + pl.o_temp); w.press = (double*)(A + pl.o_press);
  w.rho_vap = (double*)(A + pl.o_rho_vap); w.q_hum = (double*)(A + pl.o_q_hum); w.vap = (double*)(A + pl.o_vap);
  w.gtemp = (double*)(A + pl.o_gtemp); w.outlev = (int*)(A + pl.o_outlev); w.kgas = (double*)(A + pl.o_kgas);
  w.slot_st = (int8_t*)(A + pl.o_slot_st); w.slot_nb = (int*)(A + pl.o_slot_nb);
  w.b_d = (double*)(A + pl.o_bd); w.b_dd = (double*)(A + pl.o_bdd); w.b_nd = (double*)(A + pl.o_bnd);
  w.b_rho = (double*)(A + pl.o_brho); w.b_mass = (double*)(A + pl.o_bmass);
  w.pres_idx = (int*)(A + pl.o_pres_idx); w.plist = (int*)(A + pl.o_plist); w.pmax = pl.pmax;
  w.counters = (int*)(A + pl.o_counters);
  w.m_kext = (double*)(A + pl.o_mkext); w.m_salb = (double*)(A + pl.o_msalb); w.m_nleg = (int*)(A + pl.o_mnleg);
  w.m_back = (double*)(A + pl.o_mback); w.m_refr = (double*)(A + pl.o_mrefr);
  w.m_legen = pl.f32_coef ? nullptr : (double*)(A + pl.o_mlegen);
  w.m_legen32 = pl.f32_coef ? (float*)(A + pl.o_mlegen) : nullptr;
  w.lay = (double*)(A + pl.o_lay); w.lay_stride = pl.lay_stride; w.lay_nd = (int*)(A + pl.o_laynd);
  w.status = (int*)(A + pl.o_status); w.col_status = (int*)(A + pl.o_colst);
  w.spin_limit = tc::MBAR_SPIN_LIMIT;
  w.mie_slab = (double*)(A + pl.o_mieslab); w.mie_nslab = pl.mie_nslab;
  w.gq_x = D.tables; w.gq_w = D.tables + gqn; w.gq_max = NOALLOC_GQ;
  w.lob_mu = D.tables + 2 * gqn; w.lob_w = D.tables + 2 * gqn + 56;
  const size_t Lm = cc.max_nlyrs, Fm = cc.max_nfreq;
  // the scratch keeps the previous call's contents: clear what must start at zero
  cudaMemsetAsync(w.counters, 0, 16 * 4, stream);
  cudaMemsetAsync(w.status, 0, Fm * 4, stream);
  cudaMemsetAsync(w.col_status, 0, 4, stream);
  const size_t ntb = (size_t)cc.noutlevels * 2 * cc.max_nummu * Fm * 2;
  k_fill_d<<<(unsigned)((ntb + 255) / 256), 256, 0, stream>>>(out->tb, -9999.0, ntb);
  k_atmo<<<1, 128, 0, stream>>>(b, w);
  k_gas<<<(unsigned)((Fm * Lm + 255) / 256), 256, 0, stream>>>(b, w, st->lgas_extinction, st->gas_mod);
  if (nh > 0) k_psd<<<(unsigned)((Lm * nh + 127) / 128), 128, 0, stream>>>(b, w, *st);
  k_compact<<<1, 1024, 0, stream>>>(b, w);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (nh > 0) {
    const size_t sm_mie = MIE_WARPS * sizeof(MieSmem);
    k_refr<<<(unsigned)(((size_t)std::max(1, pl.pmax) * Fm + 127) / 128), 128, 0, stream>>>(b, w, *st);
    k_mie<MIE_GROUP><<<NOALLOC_MIE_SLABS / MIE_WARPS, 32 * MIE_WARPS, sm_mie, stream>>>(b, w, *st);
  }
  if (mask & 1) {
    if (nh > 0) k_layer<8><<<sms, RTCfg<8>::T, sizeof(LayerSmem<8>), stream>>>(b, w, *st, out->scatter_matrix);
    k_adding<8><<<sms, RTCfg<8>::T, sizeof(AddSmem<8>), stream>>>(b, w, *st, *out);
  }
  if (mask & 2) {
    if (nh > 0) k_layer<16><<<sms, RTCfg<16>::T, sizeof(LayerSmem<16>), stream>>>(b, w, *st, out->scatter_matrix);
    k_adding<16><<<sms, RTCfg<16>::T, sizeof(AddSmem<16>), stream>>>(b, w, *st, *out);
  }
  if (out->angles_deg) k_angles<<<1, 32, 0, stream>>>(out->angles_deg, w.lob_mu, cc.max_nummu);
  if (out->kexttot || out->salbedo || out->num_doubles)
    k_ssp_out<<<(unsigned)((Fm * Lm + 255) / 256), 256, 0, stream>>>(b, w, *out);
  if (out->kextatmo) cudaMemcpyAsync(out->kextatmo, w.kgas, Fm * Lm * 8, cudaMemcpyDeviceToDevice, stream);
  if (st->active && (out->ze || out->att_hydro || out->att_atmo)) k_radar<<<1, 128, 0, stream>>>(b, w, *st, *out);
  if (out->status) k_status_out<<<1, 256, 0, stream>>>(w, out->status, (int)Fm);
  return cudaGetLastError() == cudaSuccess ? PAMTRA_B200_OK : PAMTRA_B200_FATAL;
}
