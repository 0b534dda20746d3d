/*
 * pamtra_b200.h -- C ABI of the B200-native PAMTRA passive forward path.
 *
 * Boundary being replaced.  The reference crosses from Python into native
 * code through f2py: python/pyPamtra/libWrapper.py:24-235
 * (PamtraFortranWrapper) copies the namelist settings, the descriptor file
 * and the profile into Fortran module globals and calls
 * pypamtralib.run_pamtra() (src/pyPamtraLib.f90:18), which loops
 * frequency x grid and calls run_rt (src/run_rt.f90:1) per column.  Results
 * come back as vars_output.out_* arrays.  Error codes are 0 (success),
 * 1 (warning), 2 (fatal) (src/report_module.f90:11-14).
 *
 * Here the same seam is one re-entrant call per batch of columns on a
 * caller-provided CUDA stream, with plain pointers and sizes.  All array
 * pointers in pamtra_b200_columns / pamtra_b200_outputs are DEVICE pointers
 * (caller-owned), except in pamtra_b200_run_host, which takes HOST pointers
 * and performs the copies itself.  The library owns only its scratch arena,
 * held by the context.
 *
 * Layouts (row-major, C order):
 *   level arrays  [ncol][max_nlyrs+1]   bottom-up, NaN = missing
 *   layer arrays  [ncol][max_nlyrs]     bottom-up, NaN = missing
 *   hydro arrays  [ncol][max_nlyrs][nhydro]
 *   tb            [ncol][noutlevels][2*max_nummu][max_nfreq][2]   (V,H or I,Q)
 *   emissivity    [ncol][2][max_nfreq][max_nummu]
 *   status        [ncol][max_nfreq]   0 ok, 2 fatal, see PAMTRA_B200_ST_*
 */
#ifndef PAMTRA_B200_H
#define PAMTRA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PAMTRA_B200_MAXNLEG 200   /* src/settings.f90:13 maxleg */
#define PAMTRA_B200_MAXBIN 256    /* bins per species slot */

/* error / status codes (src/report_module.f90:11-14, plus per-column detail) */
#define PAMTRA_B200_OK 0
#define PAMTRA_B200_WARNING 1
#define PAMTRA_B200_FATAL 2
#define PAMTRA_B200_ST_NORM 0x100      /* check_norm4 failed (src/radscat4.f90:125) */
#define PAMTRA_B200_ST_PSD 0x200       /* run_drop_size_dist fatal */
#define PAMTRA_B200_ST_MIE 0x400       /* calc_mie_spheres assertion failed */
#define PAMTRA_B200_ST_GAS 0x800       /* rosen98 input range (src/rosen98_gasabs.f90:103-125) */
#define PAMTRA_B200_ST_PIVOT 0x1000    /* singular matrix in an inverse */
#define PAMTRA_B200_ST_NAN 0x2000      /* NaN in extinction / coefficients */
#define PAMTRA_B200_ST_SIZE 0x4000     /* a size limit of this library was exceeded */
#define PAMTRA_B200_ST_TIMEOUT 0x8000  /* a bounded wait on the tensor core gave up */
#define PAMTRA_B200_ST_RANGE 0x10000   /* input outside a model's range (liq_mod 'Ray' outside 0.2 um - 10 cm wavelength) */

/* dist_name codes (src/make_dist_param.f90) */
#define PAMTRA_B200_DIST_EXP 0
#define PAMTRA_B200_DIST_EXP_FIELD_T 1
#define PAMTRA_B200_DIST_MGAMMA 2
#define PAMTRA_B200_DIST_MONO 3
#define PAMTRA_B200_DIST_EXP_RYAN 5
#define PAMTRA_B200_DIST_LOGN 6
#define PAMTRA_B200_DIST_DISABLED 7

/* precision / form of the doubling and adding solves */
#define PAMTRA_B200_PREC_FP64 0          /* FP64 in the reference's operation order: COMBINE_LAYERS4
                                           (src/radintg4.f90:447-513) with its two inverses per
                                           combine; the plain drop-in form */
#define PAMTRA_B200_PREC_3XTF32 1        /* batched split-precision form: layer doubling products
                                           as 3xTF32 tcgen05 MMAs (NUMMU 16 and 32; NUMMU 8 doubles
                                           in FP64); for NUMMU 16 the adding products too (stack in
                                           FP32, the (I - R R)^-1 of each combine, the surface
                                           coupling and the radiances in FP64), for NUMMU 8 and 32
                                           FP64 adding with one inverse per combine; the Legendre
                                           coefficients of the phase matrices are stored in FP32
                                           (computed and expanded in FP64) */
#define PAMTRA_B200_PREC_FP64_BATCHED 2  /* batched form in FP64: as PREC_FP64, but each adding
                                           combine derives the minus-side inverse from the
                                           plus-side one (Gm R2 = R2 Gp, Gm = I + R2 Gp R1p):
                                           one inverse and ten products instead of two and twelve */
#define PAMTRA_B200_PREC_3XTF32_FP64ADD 3 /* as PREC_3XTF32 with the adding in FP64 for every NUMMU
                                           (PREC_FP64_BATCHED's adding) */

/* Settings: the nmlSet keys on the passive Mie path
 * (src/settings.f90:454-573; python/pyPamtra/core.py:89-157). */
typedef struct pamtra_b200_settings {
  double emissivity;                 /* nmlSet['emissivity'] (sfc_optics.f90:79-81) */
  double hydro_threshold;            /* nmlSet['hydro_threshold'] */
  double hydro_softsphere_min_density;
  int32_t lgas_extinction;
  int32_t lhyd_absorption;
  int32_t lhyd_scattering;
  int32_t lhyd_emission;
  int32_t hydro_includehydroinrhoair;
  int32_t hydro_adaptive_grid;
  int32_t conserve_mass_rescale_dsd;
  int32_t hydro_limit_density_area;
  int32_t outpol_vh;                 /* nmlSet['outpol'] == 'VH' */
  int32_t nummu;                     /* default quadrature angles per hemisphere */
  /* active "simple" radar (radar_mode 'simple', src/radar_simulator.f90:161-176) */
  int32_t active;                    /* nmlSet['active']: fill outputs.ze / att_* */
  int32_t radar_attenuation;         /* PAMTRA_B200_ATT_*: nmlSet['radar_attenuation'] */
  double radar_k2;                   /* nmlSet['radar_k2'], |K|^2 of the radar equation */
  int32_t liq_mod;                   /* PAMTRA_B200_LIQ_*: nmlSet['liq_mod'] (src/eps_water.f90:39-63) */
  int32_t gas_mod;                   /* PAMTRA_B200_GAS_*: nmlSet['gas_mod'] (src/get_gasabs.f90:78-102) */
} pamtra_b200_settings;

/* liquid water permittivity models (nmlSet['liq_mod']) */
#define PAMTRA_B200_LIQ_TKC 0  /* Turner, Kneifel and Cadeddu 2016 (default) */
#define PAMTRA_B200_LIQ_ELL 1  /* Ellison 2007 */
#define PAMTRA_B200_LIQ_LIE 2  /* Liebe, Hufford and Manabe 1991 */
#define PAMTRA_B200_LIQ_RAY 3  /* Ray 1972, wavelengths above 1 mm */
#define PAMTRA_B200_LIQ_STO 4  /* Stogryn et al. 1995 */
/* gas absorption models (nmlSet['gas_mod']) */
#define PAMTRA_B200_GAS_R98 0  /* Rosenkranz 1998 (default) */
#define PAMTRA_B200_GAS_L93 1  /* Liebe MPM93 */

/* radar_attenuation codes */
#define PAMTRA_B200_ATT_DISABLED 0
#define PAMTRA_B200_ATT_BOTTOM_UP 1
#define PAMTRA_B200_ATT_TOP_DOWN 2

/* One descriptor-file row (python/pyPamtra/descriptorFile.py:19-20);
 * string fields are encoded: dist (PAMTRA_B200_DIST_*), scat = mie-sphere. */
typedef struct pamtra_b200_species {
  int32_t liq_ice, moment_in, nbin, dist;
  double as_ratio, rho_ms, a_ms, b_ms, alpha_as, beta_as;
  double p_1, p_2, p_3, p_4, d_1, d_2;
} pamtra_b200_species;

/* A batch of columns.  The plain form passes ncol = 1. */
typedef struct pamtra_b200_columns {
  int32_t ncol, max_nlyrs, nhydro, max_nfreq, noutlevels, max_nummu;
  int32_t species_stride;     /* 0: one species table for all columns; nhydro: per column */
  int32_t max_present;        /* upper bound on hydrometeor-bearing layers in the batch, 0 = ncol*max_nlyrs */
  int32_t nummu_mask;         /* bit 0: N=8, bit 1: N=16, bit 2: N=32 present; 0 = settings.nummu only */
  const pamtra_b200_species* species;  /* HOST pointer, [ncol or 1][nhydro] (copied by the library) */
  const int32_t* nlyrs;       /* [ncol] */
  const int32_t* nummu;       /* [ncol] in {8,16,32}; NULL = settings.nummu.  A column whose value is
                                 not 8/16/32, not in nummu_mask or above max_nummu is solved by no
                                 kernel and gets PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE in status */
  const int32_t* nfreq;       /* [ncol]; NULL = max_nfreq for all */
  const double* freqs;        /* [ncol][max_nfreq] GHz, or [max_nfreq] if nfreq == NULL */
  const double *hgt_lev, *temp_lev, *press_lev, *relhum_lev;   /* [ncol][max_nlyrs+1] */
  const double *hgt, *temp, *press, *relhum;                   /* [ncol][max_nlyrs]   */
  const double *hydro_q, *hydro_n, *hydro_reff;                /* [ncol][max_nlyrs][nhydro] */
  const double* groundtemp;   /* [ncol], NaN = lowest level temperature */
  const double* obs_height;   /* [ncol][noutlevels] m */
  const int8_t* sfc_refl;     /* [ncol] 'S', 'L' or 'F' */
  /* full size spectra (nmlSet['hydro_fullspec'], src/hydrometeor_extinction.f90:122-151):
   * when fs_d is not NULL the size distributions are taken from these arrays
   * instead of being derived from hydro_q / hydro_n / hydro_reff.
   * [ncol][max_nlyrs][nhydro][fs_nbin], fs_d_bound [..][fs_nbin + 1]; the
   * bin width is d_bound[i+1] - d_bound[i]; a slot takes part when its
   * number concentrations sum above zero (or hydro_threshold <= 0). */
  int32_t fs_nbin;
  const double *fs_d, *fs_d_bound, *fs_n, *fs_rho, *fs_mass;
} pamtra_b200_columns;

typedef struct pamtra_b200_outputs {
  double* tb;            /* [ncol][noutlevels][2*max_nummu][max_nfreq][2] */
  double* emissivity;    /* [ncol][2][max_nfreq][max_nummu] or NULL */
  double* angles_deg;    /* [2*max_nummu] or NULL (angles of max_nummu) */
  int32_t* status;       /* [ncol][max_nfreq] or NULL */
  /* optional single-scattering output of save_ssp (run_rt.f90:140-146),
   * for all columns/frequencies; NULL to skip */
  double* kextatmo;      /* [ncol][max_nfreq][max_nlyrs] Np/m */
  double* kexttot;       /* [ncol][max_nfreq][max_nlyrs] */
  double* salbedo;       /* [ncol][max_nfreq][max_nlyrs] */
  double* scatter_matrix;/* [ncol][max_nfreq][max_nlyrs][4][n][n], n = 2*max_nummu, row=(i2,j2) */
  int32_t* num_doubles;  /* [ncol][max_nfreq][max_nlyrs] bottom-up, -1 = non-scattering */
  /* simple radar (settings.active), [ncol][max_nfreq][max_nlyrs] bottom-up, NULL to skip:
   * ze dBZ (-9999 where no hydrometeor or no backscatter), att_hydro / att_atmo
   * one-way attenuation in dB (src/radar_simulator.f90:123-176, src/run_rt.f90:119-121) */
  double* ze;
  double* att_hydro;
  double* att_atmo;
  /* save_psd (src/hydrometeor_extinction.f90:303-309): the size bins of the
   * moment-based distributions, [ncol][max_nlyrs][nhydro][psd_nbin]: bin
   * centre (m), width (m), number per bin (1/m3), particle mass (kg) and
   * cross-section area (m2, -99 without an area-size relation); -9999 where
   * a slot carries no particles, for full spectra input and beyond a
   * species' bins.  psd_bscat: backscattering cross section per particle
   * (m2) of each bin at the column's last frequency, for moment-based and
   * full spectra alike, NaN for an empty bin (src/scatProperties.f90:914-917).
   * psd_nbin >= every species' bin count; NULL psd_d skips all six. */
  int32_t psd_nbin;
  double *psd_d, *psd_deltad, *psd_n, *psd_mass, *psd_area, *psd_bscat;
} pamtra_b200_outputs;

typedef struct pamtra_b200_ctx pamtra_b200_ctx;

/* Create / destroy a context bound to a CUDA device.  The context owns a
 * scratch arena that grows to the largest batch seen (cudaMalloc outside
 * any run) and the quadrature tables.  One context may be used from one
 * host thread at a time; use one context per concurrent stream. */
int32_t pamtra_b200_create(int32_t device, pamtra_b200_ctx** out);
int32_t pamtra_b200_destroy(pamtra_b200_ctx* ctx);

/* Scratch bytes a batch needs (so callers can pack batches by free HBM). */
size_t pamtra_b200_workspace_bytes(const pamtra_b200_columns* cols, int32_t precision);

/* Reserve the arena for batches up to this size before capture/serving. */
int32_t pamtra_b200_reserve(pamtra_b200_ctx* ctx, size_t bytes);

/* Run the passive forward model on a batch (replaces run_pamtra,
 * src/pyPamtraLib.f90:18, for the columns given).  Asynchronous on `stream`
 * (a cudaStream_t; NULL = legacy default stream).  Returns 0, or 2 on an
 * argument/launch error; per-column failures are in outputs->status. */
int32_t pamtra_b200_run(pamtra_b200_ctx* ctx, const pamtra_b200_settings* settings,
                        const pamtra_b200_columns* cols, const pamtra_b200_outputs* out,
                        int32_t precision, void* stream);

/* Same with HOST pointers in cols/out: copies inputs to the device, runs,
 * copies outputs back and synchronises the stream. */
int32_t pamtra_b200_run_host(pamtra_b200_ctx* ctx, const pamtra_b200_settings* settings,
                             const pamtra_b200_columns* cols, const pamtra_b200_outputs* out,
                             int32_t precision, void* stream);

/* Launch shapes of the persistent kernels, chosen per workload by the
 * autotuner (pamtra_b200/autotune.py); no counterpart in the reference, whose
 * Fortran has no launch configuration.  params[0]: warps per Mie CTA (2, 4 or
 * 8; 0 = 4), params[1..3]: CTAs per SM of the Mie, layer and adding kernels
 * (0 = as many as fit), params[4]: size bins per Mie work item, the tile of
 * the phase-function sums (4 or 8; 0 = 4).  Results do not depend on the
 * launch shape. */
#define PAMTRA_B200_NLAUNCH 5
int32_t pamtra_b200_set_launch(pamtra_b200_ctx* ctx, const int32_t* params, int32_t n);
int32_t pamtra_b200_get_launch(const pamtra_b200_ctx* ctx, int32_t* params, int32_t n);

/* CUDA-graph form of pamtra_b200_run (no counterpart in the reference): one
 * direct run on `stream` (synchronised) sizes the scratch arena and leaves
 * the species table resident, then the launch sequence of the same call is
 * captured.  pamtra_b200_graph_launch replays it on any stream: the kernels
 * re-read the caller's input buffers, so new values in the same buffers
 * (same shapes, same species table) give new results.  Replays fail with
 * PAMTRA_B200_FATAL once the context's arena has been regrown by a larger
 * batch; capture again then. */
typedef struct pamtra_b200_graph pamtra_b200_graph;
int32_t pamtra_b200_graph_capture(pamtra_b200_ctx* ctx, const pamtra_b200_settings* settings,
                                  const pamtra_b200_columns* cols, const pamtra_b200_outputs* out,
                                  int32_t precision, void* stream, pamtra_b200_graph** graph);
int32_t pamtra_b200_graph_launch(pamtra_b200_graph* graph, void* stream);
int32_t pamtra_b200_graph_destroy(pamtra_b200_graph* graph);

/* Bound on each wait for a tensor-core MMA of the split-precision kernels
 * (no counterpart in the reference, whose Fortran has no device waits).
 * A wait that polls the MMA's completion barrier `polls` times without
 * success gives up: the items that CTA holds or takes afterwards get
 * PAMTRA_B200_FATAL | PAMTRA_B200_ST_TIMEOUT in outputs->status and are not
 * computed, and the CTA lets its last MMA finish before it frees its tensor
 * memory, so the context stays usable.  The default is
 * PAMTRA_B200_WAIT_LIMIT_DEFAULT polls, far above any MMA's latency; 0 makes
 * every wait give up at once (to exercise that path). */
#define PAMTRA_B200_WAIT_LIMIT_DEFAULT (1u << 24)
int32_t pamtra_b200_set_wait_limit(pamtra_b200_ctx* ctx, uint32_t polls);

/* n x n matrix products the FP64 doubling kernels (k_layer<N>) of the last
 * pamtra_b200_run on ctx issued, inverses by Gauss-Jordan counted as one:
 * the executed counterpart of the algorithmic count of DOUBLING_INTEGRATION4
 * (src/radintg4.f90:174-309: six products and one inverse per doubling).
 * The split-precision kernels are not counted.  Waits for `stream`. */
int32_t pamtra_b200_layer_products(pamtra_b200_ctx* ctx, uint64_t* out, void* stream);

/* Number of kernel launches the last pamtra_b200_run issued on ctx. */
int32_t pamtra_b200_last_launch_count(const pamtra_b200_ctx* ctx);

/* Per-stage timing (the reference only prints total runtime, core.py:1567).
 * When enabled, pamtra_b200_run records CUDA events between its stages on
 * its stream; pamtra_b200_stage_ms waits for the last run and returns
 * milliseconds per stage: [0] pre-processing + gas + outputs, [1] size
 * distributions, [2] Mie, [3] layer doubling, [4] adding + radiance. */
#define PAMTRA_B200_NSTAGES 5
int32_t pamtra_b200_set_timing(pamtra_b200_ctx* ctx, int32_t enable);
int32_t pamtra_b200_stage_ms(pamtra_b200_ctx* ctx, float* ms, int32_t n);

/* sizeof of the ABI structs, in order settings, species, columns, outputs,
 * tmatrix_in, tmatrix_out (for bindings to check their struct layouts). */
int32_t pamtra_b200_abi_sizes(size_t* out, int32_t n);

/* ---- single-stage entry points (parity tests of individual routines) ---- */

/* Rosenkranz-98 absorption (src/rosen98_gasabs.f90:2 + get_gasabs.f90:95),
 * element-wise over device arrays; kext in Np/m. */
int32_t pamtra_b200_gas_r98(const double* freq, const double* temp, const double* rho_vap,
                            const double* press, double* kext, int32_t* status, int32_t n, void* stream);

/* TKC water permittivity (src/eps_water.f90:653), element-wise; T in degC. */
int32_t pamtra_b200_eps_water_tkc(const double* t_c, const double* freq, double* eps_re, double* eps_im,
                                  int32_t n, void* stream);

/* get_eps_water (src/eps_water.f90:6-70) for a PAMTRA_B200_LIQ_* model,
 * element-wise: salinity s (ppt), T in degC, f in GHz; status[i] is
 * PAMTRA_B200_FATAL | PAMTRA_B200_ST_RANGE where the model has no value. */
int32_t pamtra_b200_get_eps_water(int32_t liq_mod, const double* s, const double* t_c, const double* freq,
                                  double* eps_re, double* eps_im, int32_t* status, int32_t n, void* stream);

/* MPM93 absorption (src/mpm93.f90, called as src/get_gasabs.f90:78-86),
 * element-wise: pressure and water vapour pressure in Pa, T in K; Np/m. */
int32_t pamtra_b200_gas_l93(const double* freq, const double* press, const double* vap, const double* temp,
                            double* kext, int32_t n, void* stream);

/* ---- T-matrix scattering of spheroids (scat_name 'tmatrix') ----
 * calc_tmatrix (src/tmatrix.f90:14-433) for a batch of (species, layer,
 * frequency) items of nbins bins each: per bin the T-matrix of a spheroid of
 * the bin's aspect ratio and canting angle (tmatrix_amplq, the EBCM solve of
 * src/tmatrix_amplq.lp.f, with NMAX and the Gauss points converged as there),
 * its amplitude matrices over 30 scattering azimuths at the Lobatto angles
 * (calc_single_tmatrix, src/tmatrix.f90:436-684), and the bin sums weighted
 * by ndens * del_d.  Replaces the call at src/scatProperties.f90:289-306.
 * All array pointers are host pointers (on_device = 0: copied in and out, the
 * call returns when the results are on the host) or device pointers
 * (on_device = 1: work queued on `stream`); one call in flight per context.
 * The solve is FP64 where the reference's is REAL*16: it agrees for ice and
 * snow at all sizes and for liquid water up to size parameter ~3 (~6 for
 * aspect ratios 0.7-1.5); larger aspherical drops lose accuracy. */
typedef struct {
  int32_t n_items, nbins, nummu, on_device;  /* nummu in {8, 16, 32} */
  const double* freq;     /* [n_items] Hz */
  const double* ref_re;   /* [n_items] refractive index of water or pure ice (either sign of Im) */
  const double* ref_im;
  const int32_t* phase;   /* [n_items] 1 liquid, -1 ice (mixed with air where density != 917) */
  const double* dmax;     /* [n_items][nbins] maximum dimension (m) */
  const double* del_d;    /* [n_items][nbins] bin width (m) */
  const double* ndens;    /* [n_items][nbins] number density per size (1/m^4); 0 = empty bin */
  const double* density;  /* [n_items][nbins] particle density (kg/m^3) */
  const double* as_ratio; /* [n_items][nbins] aspect ratio (< 1 oblate, > 1 prolate) */
  const double* canting;  /* [n_items][nbins] canting angle beta (deg) */
} pamtra_b200_tmatrix_in;
typedef struct {
  double* scatter_matrix; /* [n_items][2 * nummu * 2 * nummu * 2], Fortran order of scatter_matrix(2,nummu,2,nummu,2) */
  double* extinct_matrix; /* [n_items][2 * 2 * nummu] */
  double* emis_vector;    /* [n_items][2 * nummu] */
  double* sback;          /* [n_items][2 * 2] */
  double* back_spec;      /* [n_items][nbins] "NN" backscattering 4 pi ndens Sback(1,1) (m^-1 per m) */
  int32_t* nmax;          /* [n_items][nbins] converged NMAX (0 empty bin); may be NULL */
  int32_t* status;        /* [n_items] OR of the bins: FATAL | ST_RANGE for an invalid bin or a solve past
                             NMAX 48 / 128 Gauss points (the reference allows 100 / 500) */
} pamtra_b200_tmatrix_out;

int32_t pamtra_b200_tmatrix(pamtra_b200_ctx* ctx, const pamtra_b200_tmatrix_in* in, pamtra_b200_tmatrix_out* out,
                            void* stream);

/* Matrix inverse with partial pivoting of `count` column-major n x n matrices
 * (replaces MINVERT, src/radmat.f90:155), n in {16,32,64}. */
int32_t pamtra_b200_minvert_batched(const double* a, double* ainv, int32_t* status, int32_t n, int32_t count,
                                    void* stream);

/* C = A * B for `count` column-major n x n matrices (replaces MMULT,
 * src/radmat.f90:137, for batches) computed as 3xTF32 split-precision
 * tcgen05 tensor-core products with FP32 accumulation; n = 32.  *err is
 * OR-ed with 1 if a wait on the tensor core timed out. */
int32_t pamtra_b200_mmult_3xtf32_batched(const double* a, const double* b, double* c, int32_t n, int32_t count,
                                         int32_t* err, void* stream);

/* ---- allocation-free single column ----
 * No counterpart in the reference (its Fortran owns module-global arrays).
 * For callers that cannot call cudaMalloc: hosts whose own device memory
 * manager owns all allocations and forbids outside ones, and latency-critical
 * callers that cannot accept the device-wide synchronisation an allocation
 * implies.  Runs the plain form (one column, same kernels as
 * pamtra_b200_run) with all scratch in a fixed static device array of
 * PAMTRA_B200_NOALLOC_SCRATCH_MIB MiB that every GPU loading this library
 * keeps until the process exits.  No context is needed and nothing is
 * allocated: no cudaMalloc, cudaFree, pinned host memory or library
 * allocator.  All pointers in `cols` and `out` are DEVICE pointers,
 * `cols->species` included.  Limits: ncol = 1, max_nlyrs <= 64,
 * max_nfreq <= 4, nhydro <= 4, nbin <= 64 per species, nummu 8 or 16,
 * noutlevels <= 2, no full spectra (fs_d NULL) and no save_psd outputs
 * (psd_d NULL); other requests return
 * PAMTRA_B200_FATAL | PAMTRA_B200_ST_SIZE without running, and so does a
 * quadrature (settings.nummu or nummu_mask) wider than max_nummu.  The first
 * call on a device (with that device current) is the set-up: CUDA loads this
 * library's device code and its static arrays on that device at first use
 * (lazy module loading, the default), which takes device memory for the
 * module and synchronises; the call then resolves the array's device address
 * with cudaGetSymbolAddress, fills the quadrature and line tables and
 * synchronises the stream.  Make that first call once per device outside any
 * no-allocation or latency-critical region, and before any stream capture;
 * later calls allocate nothing and do not synchronise.  Every call shares the one array and
 * clears what must start at zero, so calls that overlap on the GPU (other
 * streams, other host threads) race: serialise them. */
#define PAMTRA_B200_NOALLOC_SCRATCH_MIB 8
#define PAMTRA_B200_NOALLOC_MAX_NLYRS 64
#define PAMTRA_B200_NOALLOC_MAX_NFREQ 4
#define PAMTRA_B200_NOALLOC_MAX_NHYDRO 4
#define PAMTRA_B200_NOALLOC_MAX_NBIN 64
int32_t pamtra_b200_run_noalloc(const pamtra_b200_settings* settings, const pamtra_b200_columns* cols,
                                const pamtra_b200_outputs* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* PAMTRA_B200_H */
