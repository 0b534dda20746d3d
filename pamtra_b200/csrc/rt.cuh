// RT4 on the GPU.
//   k_layer<N>: per (present layer, frequency) item -- scatcnv (Legendre
//     series -> quadrature phase matrices), check_norm4, INITIALIZE4 /
//     INITIAL_SOURCE4 and DOUBLING_INTEGRATION4; writes the layer's R, T and
//     S+/S- to the scratch arena.
//   k_adding<N>: per (column, frequency) unit -- adding of all layers top
//     down (COMBINE_LAYERS4 specialised by structure), surface, internal
//     radiance at the output levels and conversion to brightness temperature.
// Both are persistent kernels: one CTA ("team", see common.cuh) per item,
// items taken from a device-side counter.
#pragma once
#include "common.cuh"
#include "work.cuh"

namespace pb {

constexpr double TWO_PI = 2.0 * 3.1415926535897932384;
constexpr double LN2_F32 = 0.693147182464599609375;  // log(2.) in REAL(4) (radtran4.f90:325)
constexpr int KMAX = 104;                             // azimuth points: numpts/2+1 for nlegen <= 199

// Legendre upward-recurrence coefficients P_l = a_l x P_{l-1} - b_l P_{l-2},
// a_l = (2l-1)/l, b_l = (l-1)/l (filled at context creation).
__constant__ double c_leg_a[MAXNLEG], c_leg_b[MAXNLEG];

// src/rt_utilities.f90:69-90 PLANCK_FUNCTION, UNITS='r'
__device__ __forceinline__ double planck(double T, double wl) {
  return (T > 0.0) ? 1.1911e8 / p5(wl) / (exp(1.4388e4 / (wl * T)) - 1) : 0.0;
}

// src/rt_utilities.f90:687-735 CONVERT_OUTPUT (UNITS='T', FLUXCODE=0)
__device__ __forceinline__ double rad_to_tb(double rad, double wl) {
  if (rad > 0.0) return 1.4388e4 / (wl * log(1.0 + 1.1911e8 / (rad * p5(wl))));
  if (rad == 0.0) return 0.0;
  return -1.4388e4 / (wl * log(1.0 + 1.1911e8 / (-rad * p5(wl))));
}

template <int N>
struct RTCfg {
  static constexpr int n = 2 * N;
  static constexpr int T = Team<n>::T;
  static constexpr int LD = Team<n>::LD;
  static constexpr int MAT = Team<n>::MAT;
};

__host__ __device__ __forceinline__ size_t lay_stride_n(int N) {
  const int n = 2 * N;
  return 2 * (size_t)n * (n + 4) + 2 * n;
}

// ============================================================== layer kernel
template <int N>
struct LayerSmem {
  static constexpr int n = RTCfg<N>::n, MAT = RTCfg<N>::MAT;
  // matrices: R, T, G, W (and Y = R T as a fifth for N != 16).  For N = 16
  // four matrices keep the block under 45.6 KB, so five CTAs fit per SM; the
  // doubling then forms Y in G's buffer once G is consumed.  During scatcnv
  // G (and W for N = 8) hold the coefficients, the last matrix the azimuth table.
  static constexpr int NM = (N == 16) ? 4 : 5;
  double m[NM][MAT];
  double lin[2 * n], cst[2 * n];
  double lin2[2 * n], cst2[2 * n];  // the other half of the doubled source buffers
  double v[4][n], u[4][n];
  double mu[N], wq[N], nrm[N];
  InvScratch<n> inv;
  int item, stat;
  // set-up buffers (layer_setup): R, T, coefficients, azimuth table
  __device__ __forceinline__ double* mat(int i) { return m[i < NM ? i : NM - 1]; }
};

// Azimuth weights of scatcnv (src/scatcnv.f90:103-192 with SUM_LEGENDRE,
// ROTATE_PHASE_MATRIX, MATRIX_SYMMETRY and FOURIER_BASIS order 0 of
// src/rt_utilities.f90:242-493).  For NSTOKES = 2 the m = 0 phase-matrix
// entries of one (mu1, mu2) pair are linear in the Legendre coefficients
// c0, c1, c2 of an item:
//   P11 = sum_l c0_l A_l,  P12 = sum_l c1_l B_l,  P21 = sum_l c1_l C_l,
//   P22 = sum_l (c0_l D_l + c2_l E_l),
// where A..E are the azimuth sums over k = 0..numpts/2 (weight 1 at the two
// ends, 2 inside, / numpts) of P_l(cos Theta_k) times 1, cos 2i1, cos 2i2,
// cos 2i1 cos 2i2 and -sin 2i1 sin 2i2.  The tables depend only on NUMMU and
// numpts, so one kernel fills every numpts a batch has met (wt_need) that is
// not filled yet (wt_ready); one thread per (numpts, mu1, mu2).
template <int N>
__global__ void __launch_bounds__(128) k_scat_weights(double* __restrict__ tab, const int* __restrict__ need,
                                                      const int* __restrict__ ready, const double* lob_mu) {
  constexpr int C2 = 2 * N * N;
  constexpr int NB = (C2 + 127) / 128;
  const int pi = blockIdx.x / NB;
  const int combo = (blockIdx.x % NB) * 128 + threadIdx.x;
  const int ni = nmu_index(N);
  if (pi >= SCAT_NPI || combo >= C2 || !need[ni * SCAT_NPI + pi] || ready[ni * SCAT_NPI + pi]) return;
  const int numpts = 2 * pi + 4, K = numpts / 2 + 1, nl = numpts - 3;
  const int q = combo / (N * N), j1 = (combo / N) % N, j2 = combo % N;
  const double mu1 = (q == 0) ? lob_mu[lob_off(N) + j1] : -lob_mu[lob_off(N) + j1];
  const double mu2 = lob_mu[lob_off(N) + j2];
  const double st1 = sqrt(1. - mu1 * mu1), st2 = sqrt(1. - mu2 * mu2);
  const double sqm = sqrt((1. - mu1 * mu1) * (1. - mu2 * mu2));
  double* T = tab + scat_weight_offset(N, pi) + combo;
  for (int e = 0; e < nl * 5; e++) T[(size_t)e * C2] = 0.0;
  for (int k = 0; k < K; k++) {
    const double delphi = (TWO_PI * k) / numpts;
    const double cosphi = cos(delphi), sinphi = sin(delphi);
    const double cs = mu1 * mu2 + sqm * cosphi;
    const double ss = sqrt(fmax(0.0, 1. - cs * cs));
    double sin1, sin2, cos1, cos2;
    if (ss == 0.0) {
      sin1 = 0; sin2 = 0; cos1 = 1; cos2 = -1;
    } else {
      const double r = 1.0 / ss;
      sin1 = st2 * sinphi * r;
      sin2 = st1 * sinphi * r;
      cos1 = (st1 * mu2 - st2 * mu1 * cosphi) * r;
      cos2 = (st2 * mu1 - st1 * mu2 * cosphi) * r;
    }
    const double sin21 = 2.0 * sin1 * cos1, cos21 = 1.0 - 2.0 * (sin1 * sin1);
    const double sin22 = 2.0 * sin2 * cos2, cos22 = 1.0 - 2.0 * (sin2 * sin2);
    const double wk = (k > 0 && k < K - 1) ? 2.0 : 1.0;
    const double f[5] = {wk, wk * cos21, wk * cos22, wk * (cos21 * cos22), -wk * (sin21 * sin22)};
    double pl1 = 1.0, pl2 = 0.0;
    for (int l = 0; l < nl; l++) {
      double pl = 1.0;
      if (l > 0) {
        pl = fma(c_leg_a[l] * cs, pl1, -c_leg_b[l] * pl2);
        pl2 = pl1;
        pl1 = pl;
      }
      double* Tl = T + (size_t)l * 5 * C2;
#pragma unroll
      for (int e = 0; e < 5; e++) Tl[(size_t)e * C2] = fma(pl, f[e], Tl[(size_t)e * C2]);
    }
  }
  const double inv = 1.0 / numpts;
  for (int e = 0; e < nl * 5; e++) T[(size_t)e * C2] *= inv;
}

// Mark the numpts tables of N filled by k_scat_weights (run by one block of
// the kernel that follows it on the stream).
template <int N>
__device__ __forceinline__ void scat_weights_mark_ready(const Work& w) {
  const int ni = nmu_index(N);
  if (blockIdx.x == 0 && w.wt_need)
    for (int i = threadIdx.x; i < SCAT_NPI; i += blockDim.x)
      if (w.wt_need[ni * SCAT_NPI + i]) w.wt_ready[ni * SCAT_NPI + i] = 1;
}

// Per-item state of the layer stage after the thin-layer initialisation.
struct LayerItem {
  int c, z, fi, nd, status;
  double linfac;
};

// scatcnv, CHECK_NORM4, number of doublings, INITIALIZE4 and
// INITIAL_SOURCE4 of one (present layer, frequency) item: leaves the
// thin-layer R (S.m[0]) and T (S.m[1]) and the sources S.lin / S.cst in
// shared memory.  Returns false when the item is not for this N.
template <int N, class SM, int T = RTCfg<N>::T>
__device__ __forceinline__ bool layer_setup(const Batch& b, const Work& w, const pamtra_b200_settings& st,
                                            double* __restrict__ ssp_scat, SM& S, int item,
                                            LayerItem& it) {
  constexpr int n = RTCfg<N>::n, LD = RTCfg<N>::LD, MAT = RTCfg<N>::MAT;
  const int t = threadIdx.x;
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq;
    const int p = item / Fm, fi = item % Fm;
    const int cz = w.plist[p];
    const int c = cz / Lm, z = cz % Lm;
    if (fi >= b.col_nfreq(c) || b.col_nummu(c) != N) return false;
    const double freq = b.freq(c, fi);
    const double wl = C_LIGHT / (freq * 1.e3);
    const double* hl = w.hgt_lev + (size_t)c * (Lm + 1);
    const double* tl = w.temp_lev + (size_t)c * (Lm + 1);
    const double zdiff = fabs(hl[z + 1] - hl[z]);
    const double gas = fmax(w.kgas[((size_t)c * Fm + fi) * Lm + z], 0.0);
    const double planck0 = planck(tl[z + 1], wl), planck1 = planck(tl[z], wl);
    const int nleg = w.m_nleg[item];
    const double kext = w.m_kext[item], salb = w.m_salb[item];
    double* Rb = S.mat(0);
    double* Tb = S.mat(1);
    double* Gb = S.mat(2);
    double* Yb = S.mat(4);
    double ext = 0.0, emis = 0.0;
    int status = 0;
    // ---------------- scatcnv (src/scatcnv.f90) into P1 (Tb) and P2 (Rb)
    if (nleg > 0) {
      ext = kext;
      emis = (1.0 - salb) * kext;
      const double cst = kext * salb / (4.0 * 3.1415926535897932384);
      const double* lg = w.m_legen ? w.m_legen + (size_t)item * 3 * MAXNLEG : nullptr;
      const float* lg32 = w.m_legen32 ? w.m_legen32 + (size_t)item * 3 * MAXNLEG : nullptr;
      double* coef = Gb;          // [3][MAXNLEG] (S.mat(2) provides that many; for n = 16 the next matrix)
      double* cphi = Yb;          // [KMAX]
      double* sphi = Yb + KMAX;   // [KMAX]
      const int numpts = 2 * ((nleg + 1) / 2) + 4;
      const int K = numpts / 2 + 1;
      for (int l = t; l <= nleg; l += T) {
#pragma unroll
        for (int k = 0; k < 3; k++)
          coef[k * MAXNLEG + l] = cst * (lg ? lg[k * MAXNLEG + l] : (double)lg32[k * MAXNLEG + l]);
      }
      const double* W = w.wtab[nmu_index(N)];
      if (W) {
        // phase matrices from the azimuth weight tables (k_scat_weights)
        team_sync();
        constexpr int C2 = 2 * N * N, CPT = C2 / T;
        static_assert(C2 % T == 0, "combos per thread");
        const double* Wp = W + scat_weight_offset(N, (numpts - 4) / 2);
        double acc[CPT][4];
#pragma unroll
        for (int u = 0; u < CPT; u++) acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0;
        for (int l = 0; l <= nleg; l++) {
          const double c0 = coef[l], c1 = coef[MAXNLEG + l], c2 = coef[2 * MAXNLEG + l];
          const double* Wl = Wp + (size_t)l * 5 * C2 + t;
#pragma unroll
          for (int u = 0; u < CPT; u++) {
            const double* Wc = Wl + u * T;
            acc[u][0] = fma(c0, Wc[0], acc[u][0]);
            acc[u][1] = fma(c1, Wc[C2], acc[u][1]);
            acc[u][2] = fma(c1, Wc[2 * C2], acc[u][2]);
            acc[u][3] = fma(c0, Wc[3 * C2], acc[u][3]);
            acc[u][3] = fma(c2, Wc[4 * C2], acc[u][3]);
          }
        }
#pragma unroll
        for (int u = 0; u < CPT; u++) {
          const int it = t + u * T;
          const int q = it / (N * N), j1 = (it / N) % N, j2 = it % N;
          double* Qm = (q == 0) ? Tb : Rb;
          const int row0 = 2 * j2, col0 = 2 * j1;
          Qm[(col0 + 0) * LD + row0 + 0] = acc[u][0];
          Qm[(col0 + 1) * LD + row0 + 0] = acc[u][1];
          Qm[(col0 + 0) * LD + row0 + 1] = acc[u][2];
          Qm[(col0 + 1) * LD + row0 + 1] = acc[u][3];
        }
      } else {
        for (int k = t; k < K; k += T) {
          const double delphi = (TWO_PI * k) / numpts;
          cphi[k] = cos(delphi);
          sphi[k] = sin(delphi);
        }
        team_sync();
        for (int it = t; it < 2 * N * N; it += T) {
          const int q = it / (N * N), j1 = (it / N) % N, j2 = it % N;
          const double mu1 = (q == 0) ? S.mu[j1] : -S.mu[j1];
          const double mu2 = S.mu[j2];
          const double st1 = sqrt(1. - mu1 * mu1), st2 = sqrt(1. - mu2 * mu2);
          const double sqm = sqrt((1. - mu1 * mu1) * (1. - mu2 * mu2));
          double a11 = 0, a12 = 0, a21 = 0, a22 = 0, m11 = 0, m12 = 0, m21 = 0, m22 = 0;
          for (int k = 0; k < K; k++) {
            const double cosphi = cphi[k], sinphi = sphi[k];
            const double cs = mu1 * mu2 + sqm * cosphi;
            // SUM_LEGENDRE, DOSUM = (1,1,1,0,0,0)
            double s0 = coef[0], s1 = coef[MAXNLEG], s2 = coef[2 * MAXNLEG];
            double pl1 = 1.0, pl2 = 0.0;
            for (int L = 1; L <= nleg; L++) {
              const double pl = fma(c_leg_a[L] * cs, pl1, -c_leg_b[L] * pl2);
              s0 = fma(coef[L], pl, s0);
              s1 = fma(coef[MAXNLEG + L], pl, s1);
              s2 = fma(coef[2 * MAXNLEG + L], pl, s2);
              pl2 = pl1;
              pl1 = pl;
            }
            // ROTATE_PHASE_MATRIX (NSTOKES=2)
            const double ss = sqrt(fmax(0.0, 1. - cs * cs));
            double sin1, sin2, cos1, cos2;
            if (ss == 0.0) {
              sin1 = 0; sin2 = 0; cos1 = 1; cos2 = -1;
            } else {
              const double r = 1.0 / ss;
              sin1 = st2 * sinphi * r;
              sin2 = st1 * sinphi * r;
              cos1 = (st1 * mu2 - st2 * mu1 * cosphi) * r;
              cos2 = (st2 * mu1 - st1 * mu2 * cosphi) * r;
            }
            const double sin21 = 2.0 * sin1 * cos1, cos21 = 1.0 - 2.0 * (sin1 * sin1);
            const double sin22 = 2.0 * sin2 * cos2, cos22 = 1.0 - 2.0 * (sin2 * sin2);
            const double e11 = s0, e12 = s1 * cos21, e21 = s1 * cos22, e22 = s0 * cos21 * cos22 - s2 * sin21 * sin22;
            // FOURIER_BASIS order 0: points k and numpts-k coincide (MATRIX_SYMMETRY)
            a11 += e11; a12 += e12; a21 += e21; a22 += e22;
            if (k > 0 && k < K - 1) { m11 += e11; m12 += e12; m21 += e21; m22 += e22; }
          }
          double* Q = (q == 0) ? Tb : Rb;
          const int row0 = 2 * j2, col0 = 2 * j1;
          Q[(col0 + 0) * LD + row0 + 0] = (a11 + m11) / numpts;
          Q[(col0 + 1) * LD + row0 + 0] = (a12 + m12) / numpts;
          Q[(col0 + 0) * LD + row0 + 1] = (a21 + m21) / numpts;
          Q[(col0 + 1) * LD + row0 + 1] = (a22 + m22) / numpts;
        }
      }
      team_sync();
      if (!st.lhyd_scattering) {
        for (int e = t; e < MAT; e += T) { Tb[e] = 0.0; Rb[e] = 0.0; }
        team_sync();
      }
      if (!st.lhyd_emission) emis = 0.0;
    } else {
      for (int e = t; e < MAT; e += T) { Tb[e] = 0.0; Rb[e] = 0.0; }
      team_sync();
    }
    // optional save_ssp output of the 4 quadrants (l=1,4 equal; l=2,3 equal)
    if (ssp_scat) {
      const int nn = 2 * b.max_nummu;
      const size_t o = (((size_t)c * Fm + fi) * Lm + z) * 4 * (size_t)nn * nn;
      for (int e = t; e < n * n; e += T) {
        const int row = e / n, col = e % n;
        const double p1 = Tb[col * LD + row], p2 = Rb[col * LD + row];
        ssp_scat[o + 0 * (size_t)nn * nn + (size_t)row * nn + col] = p1;
        ssp_scat[o + 1 * (size_t)nn * nn + (size_t)row * nn + col] = p2;
        ssp_scat[o + 2 * (size_t)nn * nn + (size_t)row * nn + col] = p2;
        ssp_scat[o + 3 * (size_t)nn * nn + (size_t)row * nn + col] = p1;
      }
    }
    // ---------------- CHECK_NORM4 (src/radscat4.f90:87-136)
    if (t < N) {
      double sum = emis - ext;
      for (int j2 = 0; j2 < N; j2++)
        sum = sum + 2.0 * 3.1415926535897932384 * S.wq[j2] * (Tb[(2 * t) * LD + 2 * j2] + Rb[(2 * t) * LD + 2 * j2]);
      S.nrm[t] = fabs(sum);
    }
    team_sync();
    if (t == 0) {
      double mx = 0.0;
      for (int i = 0; i < N; i++) mx = fmax(mx, S.nrm[i]);
      S.stat = (mx > 5.0e-4) ? (PAMTRA_B200_FATAL | PAMTRA_B200_ST_NORM) : 0;
    }
    // ---------------- number of doublings (src/radtran4.f90:319-329)
    const double extinct = ext + gas;
    const double fl = log(fmax(extinct * zdiff, 1.0e-7) / 1.0e-6) / LN2_F32;
    int nd = 0;
    if (fl > 0.0) nd = (int)fl + 1;
    const double num_sub = ldexp(1.0, nd);
    const double delta_z = zdiff / num_sub;
    // ---------------- INITIALIZE4 (src/radintg4.f90:1-45), in place over P1/P2
    {
      const double C = 2.0 * 3.1415926535897932384;
      for (int e = t; e < n * n; e += T) {
        const int col = e / n, row = e % n;
        const int i1 = col & 1, j1 = col >> 1, i2 = row & 1, j2 = row >> 1;
        const double wj1 = S.wq[j1];
        const double tmp = delta_z / S.mu[j2];
        const double gext = (i1 == i2) ? gas : 0.0;
        const double diag = (row == col) ? 1.0 : 0.0;
        double ex = 0.0;
        if (j1 == j2) ex = ((i1 == i2) ? ext : 0.0) + gext;
        Rb[col * LD + row] = C * tmp * wj1 * Rb[col * LD + row];
        Tb[col * LD + row] = diag - tmp * (ex - C * wj1 * Tb[col * LD + row]);
      }
    }
    // INITIAL_SOURCE4 (src/radintg4.f90:51-73)
    if (t < n) {
      const int i = t & 1, jj = t >> 1;
      const double tmp = planck0 * delta_z / S.mu[jj];
      const double v = (i == 0) ? tmp * (emis + gas) : tmp * (0.0 + 0.0);
      S.lin[t] = v;
      S.lin[n + t] = v;
      S.cst[t] = v;
      S.cst[n + t] = v;
    }
    double linfac = (planck0 == 0.0) ? 0.0 : (planck1 / planck0 - 1.0) / num_sub;
    team_sync();
    status |= S.stat;
  it.c = c;
  it.z = z;
  it.fi = fi;
  it.nd = nd;
  it.status = status;
  it.linfac = linfac;
  return true;
}

// Write the layer R, T and S+/S- of an item (FP64, the layout k_adding reads).
template <int N, int T = RTCfg<N>::T>
__device__ __forceinline__ void layer_store(const Work& w, int item, const double* Rb, const double* Tb,
                                            const double* lin) {
  constexpr int n = RTCfg<N>::n, MAT = RTCfg<N>::MAT;
  const int t = threadIdx.x;
  double* out = w.lay + (size_t)item * w.lay_stride;
  for (int e = t; e < MAT; e += T) { out[e] = Rb[e]; out[MAT + e] = Tb[e]; }
  for (int e = t; e < 2 * n; e += T) out[2 * MAT + e] = lin[e];
}

template <int N>
__global__ void __launch_bounds__(RTCfg<N>::T, (N == 16 ? 5 : 1)) k_layer(Batch b, Work w, pamtra_b200_settings st,
                                                       double* __restrict__ ssp_scat) {
  constexpr int n = RTCfg<N>::n, LD = RTCfg<N>::LD, MAT = RTCfg<N>::MAT, T = RTCfg<N>::T;
  (void)LD;
  (void)MAT;
  extern __shared__ double smem_raw[];
  LayerSmem<N>& S = *reinterpret_cast<LayerSmem<N>*>(smem_raw);
  const int t = threadIdx.x;
  const int Fm = b.max_nfreq;
  const int P = min(w.counters[0], w.pmax);
  const int nitems = P * Fm;
  scat_weights_mark_ready<N>(w);
  if (t < N) { S.mu[t] = w.lob_mu[lob_off(N) + t]; S.wq[t] = w.lob_w[lob_off(N) + t]; }
  for (;;) {
    team_sync();
    if (t == 0) S.item = atomicAdd(&w.counters[2 + (N == 8 ? 0 : (N == 16 ? 1 : 2))], 1);
    team_sync();
    const int item = S.item;
    if (item >= nitems) break;
    LayerItem it;
    if (!layer_setup<N>(b, w, st, ssp_scat, S, item, it)) continue;
    const int nd = it.nd, c = it.c, fi = it.fi;
    int status = it.status;
    double linfac = it.linfac;
    double* Rb = S.m[0];
    double* Tb = S.m[1];
    double* Gb = S.m[2];
    double* Wb = S.m[3];
    double* Yb = S.mat(4);  // = Gb's buffer role for N = 16 (see below)
    constexpr bool FOUR = LayerSmem<N>::NM == 4;
    // ---------------- DOUBLING_INTEGRATION4, SYMMETRIC (src/radintg4.f90:174-309)
    // R' = R + T G R T and T' = T G T with G = (I - R R)^-1, as five products
    // per step: W = T G, then R' = R + W (R T) and T' = W T; the source
    // chains use W u for T G u.  R R and R T only read R and T, so they
    // share the first phase.
    constexpr int NV = (4 * n + T - 1) / T;
    int nprod = 5 * nd;  // n x n products issued for this item (counted by thread 0)
    // sources S+ / S- (linear and constant parts), double-buffered so that a
    // step writes the new ones while other threads still read the old
    double *lin = S.lin, *cst = S.cst, *lin_n = S.lin2, *cst_n = S.cst2;
    for (int itd = 0; itd < nd; itd++) {
      mm<n, MM_SET>(Rb, Rb, Gb);  // R+ R-
      if (!FOUR) mm<n, MM_SET>(Rb, Tb, Yb);  // Y = R T
      // v = [S- + f C-, C-, S+, C+]
      for (int o = t; o < 4 * n; o += T) {
        const int r = o % n, k = o / n;
        double v;
        if (k == 0) v = lin[n + r] + linfac * cst[n + r];
        else if (k == 1) v = cst[n + r];
        else if (k == 2) v = lin[r];
        else v = cst[r];
        S.v[k][r] = v;
      }
      team_sync();
      {
        int sg = 0;
        double* gi = inv_iminus<n>(Gb, Wb, S.inv, &sg, &nprod);  // GAMMA = inv(I - R+ R-)
        if (sg) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
        if (gi != Gb) { Wb = Gb; Gb = gi; }
      }
      // W = T G;  u = [S+ + R v0, C+ + R v1, v0 + R v2, C- + R v3]
      mm<n, MM_SET>(Tb, Gb, Wb);
      for (int o = t; o < 4 * n; o += T) {
        const int r = o % n, k = o / n;
        const double a = mv_row<n>(Rb, S.v[k], r);
        double u;
        if (k == 0) u = lin[r] + a;
        else if (k == 1) u = cst[r] + a;
        else if (k == 2) u = S.v[0][r] + a;
        else u = cst[n + r] + a;
        S.u[k][r] = u;
      }
      team_sync();
      // new sources from W u, then R' = R + W Y and T' = W T (into the G
      // buffer): nothing of this phase reads what it writes.  With four
      // matrices Y = R T goes into G's buffer here (G is consumed), and T' is
      // formed in place in T.
      if (FOUR) mm<n, MM_SET>(Rb, Tb, Gb);
#pragma unroll
      for (int s = 0; s < NV; s++) {
        const int o = t + s * T;
        if (o < 4 * n) {
          const int r = o % n, k = o / n;
          const double a = mv_row<n>(Wb, S.u[k], r);
          if (k == 0) lin_n[r] = (lin[r] + a) + linfac * cst[r];
          else if (k == 1) cst_n[r] = cst[r] + a;
          else if (k == 2) lin_n[n + r] = lin[n + r] + a;
          else cst_n[n + r] = cst[n + r] + a;
        }
      }
      if (FOUR) {
        team_sync();                           // Y complete
        mm<n, MM_ACC>(Wb, Gb, Rb, Rb);         // R' = R + W Y
        mm<n, MM_SET, true>(Wb, Tb, Tb);       // T' = W T (reads W and T, barrier, writes T)
      } else {
        mm<n, MM_ACC>(Wb, Yb, Rb, Rb);
        mm<n, MM_SET>(Wb, Tb, Gb);
        { double* tmp = Tb; Tb = Gb; Gb = tmp; }
      }
      { double* tmp = lin; lin = lin_n; lin_n = tmp; }
      { double* tmp = cst; cst = cst_n; cst_n = tmp; }
      linfac = 2.0 * linfac;
      team_sync();
    }
    layer_store<N>(w, item, Rb, Tb, lin);
    if (t == 0) {
      w.lay_nd[item] = nd;
      if (status) atomicOr(&w.status[(size_t)c * Fm + fi], status);
      if (nprod) atomicAdd(reinterpret_cast<unsigned long long*>(w.counters + COUNTER_PRODUCTS),
                           (unsigned long long)nprod);
    }
  }
}

// ============================================================== adding kernel
// Ten n x n matrices per column-frequency unit.  For N <= 16 all of them live
// in shared memory; for N = 32 (n = 64, 34 KB per matrix) the first six do and
// the last four (G, X, Y, Z) live in a per-CTA slice of global scratch
// (Work::add_scr), which stays L2-resident.
template <int N>
struct AddSmem {
  static constexpr int n = RTCfg<N>::n, MAT = RTCfg<N>::MAT;
  static constexpr int NS = (N == 32) ? 6 : 10;  // matrices in shared memory
  double m[NS][MAT];
  double sp[n], sm[n], s2p[n], s2m[n], t1[n], t2[n], nsp[n], nsm[n];
  double wv[n], wv2[n], u1[n], u2[n];
  double sky[n], gnd[n], uprad[n], dnrad[n];
  double mu[N], wq[N];
  InvScratch<n> inv;
  int unit;
};

template <int n>
__device__ __forceinline__ void ew_ident(double* A) {  // A = I
  constexpr int LD = Team<n>::LD, T = Team<n>::T;
  for (int e = threadIdx.x; e < n * n; e += T) {
    const int col = e / n, row = e % n;
    A[col * LD + row] = (row == col) ? 1.0 : 0.0;
  }
}
template <int n>
__device__ __forceinline__ void ew_zero(double* A) {
  constexpr int LD = Team<n>::LD, T = Team<n>::T;
  for (int e = threadIdx.x; e < n * n; e += T) A[(e / n) * LD + e % n] = 0.0;
}
template <int n>
__device__ __forceinline__ void ew_diag(double* A, const double* d) {
  constexpr int LD = Team<n>::LD, T = Team<n>::T;
  for (int e = threadIdx.x; e < n * n; e += T) {
    const int col = e / n, row = e % n;
    A[col * LD + row] = (row == col) ? d[col] : 0.0;
  }
}

// End of the adding for one (column, frequency) unit: the stack (Rp, Rm, Tp,
// Tm with sources S.sp / S.sm, or a clear stack t1 / sp / sm when sstate <= 1)
// on the surface, the internal radiances at the output levels, TB, status.
// R2, T2, G, X, Y are scratch matrices (G and X may be swapped by the
// inverses).
template <int N>
__device__ __forceinline__ void adding_finish(const Batch& b, const Work& w, const pamtra_b200_settings& st,
                                              const pamtra_b200_outputs& out, AddSmem<N>& S, int c, int fi,
                                              int L, double wl, int sstate, int status, double* Rp, double* Rm,
                                              double* Tp, double* Tm, double* R2, double* T2, double* G,
                                              double* X, double* Y) {
  constexpr int n = RTCfg<N>::n, LD = RTCfg<N>::LD, MAT = RTCfg<N>::MAT, T = RTCfg<N>::T;
  const int t = threadIdx.x;
  const int Fm = b.max_nfreq;
  // materialise a clear (or empty) stack
  if (sstate <= 1) {
    if (sstate == 0 && t < n) { S.t1[t] = 1.0; S.sp[t] = 0.0; S.sm[t] = 0.0; }
    team_sync();
    ew_diag<n>(Tp, S.t1);
    ew_diag<n>(Tm, S.t1);
    ew_zero<n>(Rp);
    ew_zero<n>(Rm);
    team_sync();
  }
  // surface (src/sfc_matrices.f90; default emissivity sfc_optics.f90:79-81)
  // and sky (src/surface.f90:169-195)
  const char refl = (char)b.sfc_refl[c];
  const double e = st.emissivity, rr = 1.0 - e;
  const double pg = planck(w.gtemp[c], wl), psky = planck(SKY_TEMP, wl);
  for (int ee = t; ee < n * n; ee += T) {  // R2 := surface R- (R+ = 0), T2 := I
    const int col = ee / n, row = ee % n;
    double v = 0.0;
    if (refl == 'S' || refl == 'F') {
      const double r1 = (rr + rr) / 2.0, r2 = (rr - rr) / 2.0;
      if ((row >> 1) == (col >> 1)) v = ((row & 1) == (col & 1)) ? r1 : r2;
    } else if (refl == 'L') {
      if ((row & 1) == 0 && (col & 1) == 0) v = 2.0 * rr * S.mu[col >> 1] * S.wq[col >> 1];
    }
    R2[col * LD + row] = v;
    T2[col * LD + row] = (row == col) ? 1.0 : 0.0;
  }
  if (refl != 'S' && refl != 'F' && refl != 'L') status |= PAMTRA_B200_WARNING;
  if (t < n) {
    const int i = t & 1;
    double gv = 0.0;
    if (refl == 'S' || refl == 'F') {
      const double r1 = (rr + rr) / 2.0, r2 = (rr - rr) / 2.0;
      gv = (i == 0) ? (1.0 - r1) * pg : -r2 * pg;
    } else if (refl == 'L') {
      gv = (i == 0) ? e * pg : 0.0;
    }
    S.gnd[t] = gv;
    S.sky[t] = (i == 0) ? (1.0 - 0.0) * psky : 0.0;
    S.s2m[t] = 0.0;  // the surface carries no source in the adding
  }
  team_sync();
  // output levels: L+1 -> (stack, surface); 1 -> (empty, stack on surface)
  int lev_order[2] = {-1, -1};
  for (int io = 0; io < b.noutlevels; io++) {
    const int lev = w.outlev[(size_t)c * b.noutlevels + io];
    if (lev == L + 1) lev_order[0] = io;
    else if (lev == 1) lev_order[1] = io;
    else status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE;  // intermediate levels not supported
  }
  for (int pass = 0; pass < 2; pass++) {
    const int io = lev_order[pass];
    if (io < 0) continue;
    if (pass == 1) {
      // down stack for level 1: (stack) on top of (surface), minus side only
      mm<n, MM_SET>(R2, Rp, G);  // GAMMAm = inv(I - Rsfc R1p)
      team_sync();
      {
        int sg = 0;
        double* gi = inv_iminus<n>(G, X, S.inv, &sg);
        if (sg) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
        if (gi != G) { X = G; G = gi; }
      }
      mm<n, MM_SET>(R2, Tp, X);
      if (t < n) S.wv[t] = 0.0 + mv_row<n>(R2, S.sp, t);
      team_sync();
      mm<n, MM_SET>(G, X, Y);
      if (t < n) S.wv2[t] = mv_row<n>(G, S.wv, t);
      team_sync();
      mm<n, MM_ACC>(Tm, Y, Rm, Rm);
      mm<n, MM_SET>(G, T2, X);
      if (t < n) S.nsm[t] = S.sm[t] + mv_row<n>(Tm, S.wv2, t);
      team_sync();
      mm<n, MM_SET>(Tm, X, Y);  // new T- in Y
      team_sync();
      // up side: empty (R+ = 0, T+ = I, S+ = 0); down side: (new R-, new T-, new S-)
      ew_zero<n>(Rp);
      ew_ident<n>(Tp);
      for (int ee = t; ee < MAT; ee += T) { R2[ee] = Rm[ee]; T2[ee] = Y[ee]; }
      if (t < n) { S.sp[t] = 0.0; S.s2m[t] = S.nsm[t]; }
      team_sync();
    }
    // INTERNAL_RADIANCE4 (src/radintg4.f90:119-172): up = (Rp, Tp, sp), down = (R2, T2, s2m)
    mm<n, MM_SET>(Rp, R2, X);
    if (t < n) S.wv[t] = mv_row<n>(T2, S.gnd, t);
    team_sync();
    double* Ginv;
    {
      int sg = 0;
      Ginv = inv_iminus<n>(X, G, S.inv, &sg);
      if (sg) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
    }
    if (t < n) {
      double s = mv_row<n>(Rp, S.wv, t);
      s = mv_row<n>(Tp, S.sky, t) + s;
      s = mv_row<n>(Rp, S.s2m, t) + s;
      s = S.sp[t] + s;
      S.wv2[t] = s;
    }
    team_sync();
    if (t < n) S.dnrad[t] = mv_row<n>(Ginv, S.wv2, t);
    team_sync();
    mm<n, MM_SET>(R2, Rp, X);
    if (t < n) S.wv[t] = mv_row<n>(Tp, S.sky, t);
    team_sync();
    {
      int sg = 0;
      Ginv = inv_iminus<n>(X, G, S.inv, &sg);
      if (sg) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
    }
    if (t < n) {
      double s = mv_row<n>(R2, S.wv, t);
      s = mv_row<n>(T2, S.gnd, t) + s;
      s = mv_row<n>(R2, S.sp, t) + s;
      s = S.s2m[t] + s;
      S.wv2[t] = s;
    }
    team_sync();
    if (t < n) S.uprad[t] = mv_row<n>(Ginv, S.wv2, t);
    team_sync();
    // collect_output + CONVERT_OUTPUT
    if (t < N) {
      const int jj = t;
      double u0 = S.uprad[2 * jj], u1 = S.uprad[2 * jj + 1], d0 = S.dnrad[2 * jj], d1 = S.dnrad[2 * jj + 1];
      if (st.outpol_vh) {
        double iv = 0.5 * (u0 + u1), ih = 0.5 * (u0 - u1);
        u0 = iv; u1 = ih;
        iv = 0.5 * (d0 + d1); ih = 0.5 * (d0 - d1);
        d0 = iv; d1 = ih;
        u0 = 2.0 * u0; u1 = 2.0 * u1; d0 = 2.0 * d0; d1 = 2.0 * d1;
      }
      const int NA = 2 * b.max_nummu;
      double* tbo = out.tb + ((size_t)c * b.noutlevels + io) * NA * Fm * 2;
      const size_t up_i = ((size_t)(N - 1 - jj) * Fm + fi) * 2, dn_i = ((size_t)(N + jj) * Fm + fi) * 2;
      tbo[up_i + 0] = rad_to_tb(u0, wl);
      tbo[up_i + 1] = rad_to_tb(u1, wl);
      tbo[dn_i + 0] = rad_to_tb(d0, wl);
      tbo[dn_i + 1] = rad_to_tb(d1, wl);
    }
    team_sync();
  }
  if (t == 0) {
    if (out.emissivity)
      for (int i = 0; i < 2; i++)
        for (int jj = 0; jj < N; jj++) out.emissivity[(((size_t)c * 2 + i) * Fm + fi) * b.max_nummu + jj] = e;
    if (status) atomicOr(&w.status[(size_t)c * Fm + fi], status);
  }
}

template <int N, bool ONE_INV = false>
__global__ void __launch_bounds__(RTCfg<N>::T) k_adding(Batch b, Work w, pamtra_b200_settings st,
                                                        pamtra_b200_outputs out) {
  constexpr int n = RTCfg<N>::n, LD = RTCfg<N>::LD, MAT = RTCfg<N>::MAT, T = RTCfg<N>::T;
  extern __shared__ double smem_raw[];
  AddSmem<N>& S = *reinterpret_cast<AddSmem<N>*>(smem_raw);
  const int t = threadIdx.x;
  const int Lm = b.max_nlyrs, Fm = b.max_nfreq;
  const int nunits = b.ncol * Fm;
  if (t < N) { S.mu[t] = w.lob_mu[lob_off(N) + t]; S.wq[t] = w.lob_w[lob_off(N) + t]; }
  for (;;) {
    team_sync();
    if (t == 0) S.unit = atomicAdd(&w.counters[5 + (N == 8 ? 0 : (N == 16 ? 1 : 2))], 1);
    team_sync();
    const int unit = S.unit;
    if (unit >= nunits) break;
    const int c = unit / Fm, fi = unit % Fm;
    if (fi >= b.col_nfreq(c) || b.col_nummu(c) != N) continue;
    const int L = b.nlyrs[c];
    const double freq = b.freq(c, fi);
    const double wl = C_LIGHT / (freq * 1.e3);
    const double* hl = w.hgt_lev + (size_t)c * (Lm + 1);
    const double* tl = w.temp_lev + (size_t)c * (Lm + 1);
    int status = w.col_status[c];
    double* mats[10];
#pragma unroll
    for (int q = 0; q < 10; q++)
      mats[q] = (q < AddSmem<N>::NS) ? S.m[q < AddSmem<N>::NS ? q : 0]
                                     : w.add_scr + ((size_t)blockIdx.x * (10 - AddSmem<N>::NS) + (q - AddSmem<N>::NS)) * MAT;
    double *Rp = mats[0], *Rm = mats[1], *Tp = mats[2], *Tm = mats[3];
    double *R2 = mats[4], *T2 = mats[5];
    double *G = mats[6], *X = mats[7], *Y = mats[8], *Z = mats[9];
    // stack state: 0 empty, 1 clear (R = 0, T = diag t1 on both sides), 2 general
    int sstate = 0;
    // The next scattering layer's R, T and S blocks are read into registers
    // while the current combine runs (batched forms, N <= 16: the kernel's
    // occupancy is set by shared memory, so the registers are free).
    constexpr bool PREFETCH = ONE_INV && N <= 16;
    constexpr int PFE = (MAT + T - 1) / T;
    double pfR[PREFETCH ? PFE : 1], pfT[PREFETCH ? PFE : 1], pfS[2];
    int pf_pidx = -1;
    auto prefetch = [&](int kfrom) {
      pf_pidx = -1;
      for (int kk = kfrom; kk < L; kk++) {
        const int p = w.pres_idx[(size_t)c * Lm + (L - 1 - kk)];
        if (p >= 0) { pf_pidx = p; break; }
      }
      if (pf_pidx < 0) return;
      const double* src = w.lay + ((size_t)pf_pidx * Fm + fi) * w.lay_stride;
#pragma unroll
      for (int q = 0; q < PFE; q++) {
        const int e = t + q * T;
        if (e < MAT) { pfR[q] = src[e]; pfT[q] = src[MAT + e]; }
      }
      if (t < n) { pfS[0] = src[2 * MAT + t]; pfS[1] = src[2 * MAT + n + t]; }
    };
    if (PREFETCH) prefetch(0);
    for (int k = 0; k < L; k++) {  // top-down layer index
      const int z = L - 1 - k;
      const int pidx = w.pres_idx[(size_t)c * Lm + z];
      if (pidx < 0) {
        // NONSCATTER_LAYER4 (src/radintg4.f90:79-117)
        if (t < n) {
          const int jj = t >> 1, i = t & 1;
          const double zdiff = fabs(hl[z + 1] - hl[z]);
          const double gas = fmax(w.kgas[((size_t)c * Fm + fi) * Lm + z], 0.0);
          const double dtau = zdiff * gas;
          const double p0 = planck(tl[z + 1], wl), p1 = planck(tl[z], wl);
          S.t2[t] = exp(-dtau / S.mu[jj]);
          double a = 0.0, bq = 0.0;
          if (dtau > 0.0 && i == 0) {
            const double path = dtau / S.mu[jj];
            const double slope = (p1 - p0) / path;
            a = p1 - slope - (p1 - slope * (1.0 + path)) * exp(-path);
            bq = p0 + slope - (p0 + slope * (1.0 + path)) * exp(-path);
          }
          S.s2p[t] = a;
          S.s2m[t] = bq;
        }
        team_sync();
        if (sstate == 0) {
          if (t < n) { S.t1[t] = S.t2[t]; S.sp[t] = S.s2p[t]; S.sm[t] = S.s2m[t]; }
          sstate = 1;
        } else if (sstate == 1) {
          // clear + clear
          if (t < n) {
            const double sp = S.s2p[t] + S.t2[t] * S.sp[t];
            const double sm = S.sm[t] + S.t1[t] * S.s2m[t];
            S.t1[t] = S.t2[t] * S.t1[t];
            S.sp[t] = sp;
            S.sm[t] = sm;
          }
        } else {
          // general stack + clear layer
          if (t < n) S.nsp[t] = S.s2p[t] + S.t2[t] * (S.sp[t] + mv_row<n>(Rp, S.s2m, t));
          else if (t < 2 * n) S.nsm[t - n] = S.sm[t - n] + mv_row<n>(Tm, S.s2m, t - n);
          team_sync();
          for (int e = t; e < n * n; e += T) {
            const int col = e / n, row = e % n, a = col * LD + row;
            const double t2i = S.t2[row], t2j = S.t2[col];
            Rp[a] = t2i * (Rp[a] * t2j);
            Tp[a] = t2i * Tp[a];
            Tm[a] = Tm[a] * t2j;
          }
          if (t < n) { S.sp[t] = S.nsp[t]; S.sm[t] = S.nsm[t]; }
        }
        team_sync();
        continue;
      }
      // scattering layer: its R2, T2, S2 from the arena (prefetched), then the next one's
      if (PREFETCH) {
#pragma unroll
        for (int q = 0; q < PFE; q++) {
          const int e = t + q * T;
          if (e < MAT) { R2[e] = pfR[q]; T2[e] = pfT[q]; }
        }
        if (t < n) { S.s2p[t] = pfS[0]; S.s2m[t] = pfS[1]; }
        prefetch(k + 1);
      } else {
        const double* src = w.lay + ((size_t)pidx * Fm + fi) * w.lay_stride;
        for (int e = t; e < MAT; e += T) { R2[e] = src[e]; T2[e] = src[MAT + e]; }
        for (int e = t; e < n; e += T) { S.s2p[e] = src[2 * MAT + e]; S.s2m[e] = src[2 * MAT + n + e]; }
      }
      team_sync();
      if (sstate == 0) {
        for (int e = t; e < MAT; e += T) { Rp[e] = R2[e]; Rm[e] = R2[e]; Tp[e] = T2[e]; Tm[e] = T2[e]; }
        if (t < n) { S.sp[t] = S.s2p[t]; S.sm[t] = S.s2m[t]; }
        sstate = 2;
        team_sync();
        continue;
      }
      if (sstate == 1) {
        // clear stack (t1, sp, sm) + scattering layer
        if (t < n) S.nsp[t] = S.s2p[t] + mv_row<n>(T2, S.sp, t);
        else if (t < 2 * n) S.nsm[t - n] = S.sm[t - n] + S.t1[t - n] * (S.s2m[t - n] + mv_row<n>(R2, S.sp, t - n));
        for (int e = t; e < n * n; e += T) {
          const int col = e / n, row = e % n, a = col * LD + row;
          const double t1i = S.t1[row], t1j = S.t1[col];
          const double r2 = R2[a], tt = T2[a];
          Rp[a] = r2;
          Rm[a] = t1i * (r2 * t1j);
          Tp[a] = tt * t1j;
          Tm[a] = t1i * tt;
        }
        team_sync();
        if (t < n) { S.sp[t] = S.nsp[t]; S.sm[t] = S.nsm[t]; }
        sstate = 2;
        team_sync();
        continue;
      }
      if (ONE_INV) {
        // ---- COMBINE_LAYERS4 with one inverse.  With Gp = (I - R1p R2)^-1
        // the minus-side inverse Gm = (I - R2 R1p)^-1 satisfies
        //   Gm R2 = R2 Gp   and   Gm = I + R2 Gp R1p,
        // so R1m' = R1m + T1m Gm R2 T1p = R1m + (T1m R2)(Gp T1p),
        //    T1m' = T1m Gm T2 = T1m (T2 + R2 (Gp R1p T2)),
        //    Gm w = w + R2 Gp (R1p w) for the S- chain:
        // ten products and one inverse per combine instead of twelve and two.
        // Products that share their left factor run in one pass (mm2), and the
        // two source chains of a phase run on different warps:
        //   Rp [R2, T2] -> Gp (inverted next), Z = R1p T2
        mm2<n, MM_SET, MM_SET>(Rp, R2, G, nullptr, T2, Z, nullptr);
        if (t < n) S.wv[t] = S.sp[t] + mv_row<n>(Rp, S.s2m, t);                    // S+ chain
        else if (t < 2 * n) S.nsm[t - n] = S.s2m[t - n] + mv_row<n>(R2, S.sp, t - n);  // S- chain: w
        team_sync();
        {
          int sg = 0;
          double* gi = inv_iminus<n>(G, X, S.inv, &sg);
          if (sg) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
          if (gi != G) { X = G; G = gi; }
        }
        //   Gp [Z, T1p] -> Y = Gp R1p T2, X = W = Gp T1p
        mm2<n, MM_SET, MM_SET>(G, Z, Y, nullptr, Tp, X, nullptr);
        if (t < n) S.wv2[t] = mv_row<n>(G, S.wv, t);
        else if (t < 2 * n) S.u1[t - n] = mv_row<n>(Rp, S.nsm, t - n);
        team_sync();
        //   T2 [Y, W] -> new R+ = R2 + T2 Y (into Z), new T+ = T2 W (into Rp: old R+ is dead)
        mm2<n, MM_ACC, MM_SET>(T2, Y, Z, R2, X, Rp, nullptr);
        if (t < n) S.nsp[t] = S.s2p[t] + mv_row<n>(T2, S.wv2, t);
        else if (t < 2 * n) S.u2[t - n] = mv_row<n>(G, S.u1, t - n);
        team_sync();
        mm<n, MM_SET>(Tm, R2, G);  // V = T1m R2 (Gp is dead)
        if (t < n) S.u1[t] = S.nsm[t] + mv_row<n>(R2, S.u2, t);  // Gm w
        team_sync();
        mm<n, MM_ACC>(G, X, Rm, Rm);   // new R- = R1m + V W
        mm<n, MM_ACC>(R2, Y, Tp, T2);  // U = T2 + R2 Y (old T+ is dead)
        if (t < n) S.nsm[t] = S.sm[t] + mv_row<n>(Tm, S.u1, t);
        team_sync();
        mm<n, MM_SET>(Tm, Tp, X);  // new T- = T1m U
        team_sync();
        {
          // roles: new R+ = Z, new R- = Rm, new T+ = Rp, new T- = X
          double *oRp = Rp, *oTp = Tp, *oTm = Tm, *oX = X, *oZ = Z;
          Rp = oZ;
          Tp = oRp;
          Tm = oX;
          Z = oTp;
          X = oTm;
        }
        if (t < n) { S.sp[t] = S.nsp[t]; S.sm[t] = S.nsm[t]; }
        team_sync();
        continue;
      }
      // ---- general COMBINE_LAYERS4 (src/radintg4.f90:447-513), R2p = R2m, T2p = T2m
      mm<n, MM_SET>(Rp, R2, G);  // GAMMAp = inv(I - R1p R2m)
      team_sync();
      {
        int sg = 0;
        double* gi = inv_iminus<n>(G, X, S.inv, &sg);
        if (sg) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
        if (gi != G) { X = G; G = gi; }
      }
      mm<n, MM_SET>(Rp, T2, X);  // RTp = R2p + T2p G R1p T2m
      if (t < n) S.wv[t] = S.sp[t] + mv_row<n>(Rp, S.s2m, t);  // STp chain
      team_sync();
      mm<n, MM_SET>(G, X, Y);
      if (t < n) S.wv2[t] = mv_row<n>(G, S.wv, t);
      team_sync();
      mm<n, MM_ACC>(T2, Y, Z, R2);  // new R+ in Z
      mm<n, MM_SET>(G, Tp, X);      // TTp = T2p G T1p
      if (t < n) S.nsp[t] = S.s2p[t] + mv_row<n>(T2, S.wv2, t);
      team_sync();
      mm<n, MM_SET>(T2, X, Y);  // new T+ in Y
      team_sync();
      mm<n, MM_SET>(R2, Rp, G);  // GAMMAm = inv(I - R2m R1p); Gp is dead
      team_sync();
      {
        int sg = 0;
        double* gi = inv_iminus<n>(G, X, S.inv, &sg);
        if (sg) status |= PAMTRA_B200_FATAL | PAMTRA_B200_ST_PIVOT;
        if (gi != G) { X = G; G = gi; }
      }
      mm<n, MM_SET>(R2, Tp, X);  // RTm = R1m + T1m G R2m T1p
      if (t < n) S.wv[t] = S.s2m[t] + mv_row<n>(R2, S.sp, t);  // STm chain
      team_sync();
      mm<n, MM_SET>(G, X, Rp);  // old R+ is dead
      if (t < n) S.wv2[t] = mv_row<n>(G, S.wv, t);
      team_sync();
      mm<n, MM_ACC>(Tm, Rp, Rm, Rm);  // new R- in place
      mm<n, MM_SET>(G, T2, X);        // TTm = T1m G T2m
      if (t < n) S.nsm[t] = S.sm[t] + mv_row<n>(Tm, S.wv2, t);
      team_sync();
      mm<n, MM_SET>(Tm, X, Tp);  // old T+ is dead: new T- in Tp buffer
      team_sync();
      {
        // roles: new R+ = Z, new R- = Rm, new T+ = Y, new T- = Tp
        double *oRp = Rp, *oTm = Tm;
        Rp = Z;
        Tm = Tp;
        Tp = Y;
        Z = oRp;
        Y = oTm;
      }
      if (t < n) { S.sp[t] = S.nsp[t]; S.sm[t] = S.nsm[t]; }
      team_sync();
    }
    adding_finish<N>(b, w, st, out, S, c, fi, L, wl, sstate, status, Rp, Rm, Tp, Tm, R2, T2, G, X, Y);
  }
}

}  // namespace pb
