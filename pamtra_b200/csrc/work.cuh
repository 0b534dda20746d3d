// Device-side views of a batch (inputs) and of the scratch arena.
#pragma once
#include "common.cuh"

namespace pb {

// Inputs of one batch; copies of the pamtra_b200_columns pointers plus the
// padded sizes.  Passed by value to kernels.
struct Batch {
  int ncol, max_nlyrs, nhydro, max_nfreq, noutlevels, max_nummu, max_nbin, species_stride;
  int default_nummu;
  int nummu_mask;  // quadratures launched: bit 0 N = 8, bit 1 N = 16, bit 2 N = 32
  const pamtra_b200_species* species;
  const int* nlyrs;
  const int* nummu;
  const int* nfreq;
  const double* freqs;
  int freq_per_col;
  const double *hgt_lev, *temp_lev, *press_lev, *relhum_lev;
  const double *hgt, *temp, *press, *relhum;
  const double *hydro_q, *hydro_n, *hydro_reff;
  const double* groundtemp;
  const double* obs_height;
  const int8_t* sfc_refl;
  // full size spectra [C][Lm][H][fs_nbin] (d_bound: fs_nbin + 1); fs_d NULL = derived
  int fs_nbin;
  const double *fs_d, *fs_d_bound, *fs_n, *fs_rho, *fs_mass;

  __device__ __forceinline__ int col_nfreq(int c) const { return nfreq ? nfreq[c] : max_nfreq; }
  __device__ __forceinline__ double freq(int c, int f) const {
    return freq_per_col ? freqs[(size_t)c * max_nfreq + f] : freqs[f];
  }
  __device__ __forceinline__ int col_nummu(int c) const { return nummu ? nummu[c] : default_nummu; }
  __device__ __forceinline__ pamtra_b200_species species_of(int c, int h) const {
    return species[(size_t)c * species_stride + h];
  }
};

// Scratch arena views.  Index conventions:
//   column-level  [c][...]
//   slot          s = (c*Lm + z)*H + h
//   present layer p (compact), unit-layer item i = p*Fm + f
struct Work {
  // atmosphere
  double *hgt_lev, *temp_lev;          // [C][Lm+1]
  double *temp, *press, *rho_vap, *q_hum, *vap;  // [C][Lm]; vap: vapour pressure, Pa
  double* gtemp;                       // [C]
  int* outlev;                         // [C][nout]
  double* kgas;                        // [C][Fm][Lm]
  // size distributions
  int8_t* slot_st;                     // [S] 0 absent, 1 present w/o bins, 2 bins, 3 fatal
  int* slot_nb;                        // [S]
  double *b_d, *b_dd, *b_nd, *b_rho, *b_mass;  // [S][max_nbin]
  // save_psd outputs [S][psd_nbin] (NULL psd_d: not requested)
  double *psd_d, *psd_dd, *psd_n, *psd_mass, *psd_area, *psd_bscat;
  int psd_nbin;
  // compaction
  int* pres_idx;                       // [C][Lm]
  int* plist;                          // [pmax]
  int pmax;
  int* counters;                       // [16] 0: P, 1: mie work, 2-4: layer work, 5-7: adding work,
                                       // 8-9: n x n products of the FP64 layer kernel (uint64)
  // single-scattering per item
  double *m_kext, *m_salb;             // [pmax*Fm]
  double* m_back;                      // [pmax*Fm] volumetric backscattering cross section, m^2/m^3
  double* m_refr;                      // [pmax*Fm][4] refractive index of water (re, im), ice (re, im); NaN: none
  int* m_nleg;                         // [pmax*Fm]
  double* mie_slab;                    // [mie_nslab][MIE_SLAB_STRIDE] per-warp Mie slabs of k_mie
  int mie_nslab;
  double* m_legen;                     // [pmax*Fm][3][MAXNLEG] normalised Legendre coefficients (FP64 storage)
  float* m_legen32;                    // the same in FP32 storage (split-precision form); exactly one is set
  // layer R, T, S per item (R,T padded n x (n+2), symmetric +/-)
  double* lay;                         // [pmax*Fm][lay_stride]
  size_t lay_stride;
  int* lay_nd;                         // [pmax*Fm]
  int lay32;                           // k_layer_tc writes FP32 layer records (add_tc.cuh) for k_adding_tc
  float* add_stk;                      // [C*Fm][STK_FLOATS] FP32 adding stacks, k_adding_tc -> k_adding_finish
  // adding matrices that do not fit in shared memory (N = 32 only)
  double* add_scr;                     // [adding CTAs][4][MAT]
  // scatcnv weight tables per NUMMU index (0: N = 8, 1: 16, 2: 32); null = direct sums
  const double* wtab[3];               // [numpts index][l][5][2 N^2], see scat_weight_offset
  int* wt_need;                        // [3][SCAT_NPI] numpts values seen (set by k_mie)
  int* wt_ready;                       // [3][SCAT_NPI] tables already computed
  // polls of each wait on a tensor-core MMA before it gives up (PAMTRA_B200_ST_TIMEOUT)
  uint32_t spin_limit;
  // status
  int* status;                         // [C][Fm]
  int* col_status;                     // [C]
  // quadrature tables
  const double* gq_x;                  // Gauss-Legendre nodes, packed: nquad=q at offset q*(q-1)/2
  const double* gq_w;
  int gq_max;
  const double* lob_mu;                // Lobatto nodes for N = 8,16,32 at offsets 0, 8, 24
  const double* lob_w;
};

constexpr int COUNTER_PRODUCTS = 8;  // counters[8..9]: 8-byte aligned (the arena slice is 256-aligned)

__host__ __device__ __forceinline__ int lob_off(int N) { return N == 8 ? 0 : (N == 16 ? 8 : 24); }
__host__ __device__ __forceinline__ int nmu_index(int N) { return N == 8 ? 0 : (N == 16 ? 1 : 2); }

// scatcnv weight tables: numpts = 2 * ((nlegen + 1) / 2) + 4 takes SCAT_NPI
// values 4, 6, ..., 204 (index pi = (numpts - 4) / 2); the table of pi holds
// numpts - 3 = 2 pi + 1 Legendre orders x 5 weights x 2 N^2 (mu1, mu2) pairs,
// so it starts 10 N^2 pi^2 doubles into the tables of N.
constexpr int SCAT_NPI = 101;
__host__ __device__ __forceinline__ size_t scat_weight_offset(int N, int pi) {
  return (size_t)10 * N * N * pi * pi;
}
__host__ __device__ __forceinline__ size_t scat_weight_doubles(int N) { return scat_weight_offset(N, SCAT_NPI); }

}  // namespace pb
