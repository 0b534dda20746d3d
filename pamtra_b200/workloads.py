"""Seeded synthetic workloads of the named shapes (shared by tests, smoke and
bench).  No dataset is involved: the reference publishes none for this path.

``golden_pam`` rebuilds the reference's golden regression column
(tests/_scenario.py:14-38 of the reference): rain (exp, N0 = 8e6, 30 bins)
at 1 g/kg in layer 1 and snow (exp_field_t) at 0.5 g/kg in layer 2 of a
U.S. standard atmosphere on hgt_lev = 0..3 km, at 10.65 and 35.5 GHz.

``c1_pam`` is the single-column workload: 50 layers over 0-12 km, seeded
standard-atmosphere T/p jitter, RH 40-95 %, cloud liquid (exp, 40 bins over
2-100 um, 0.3 g/kg) and rain (Marshall-Palmer, 50 bins over 0.1-6 mm,
0.5 g/kg) in layers 5-25, specular surface with emissivity 0.5 at 290 K.

``c2_pam`` is the batched workload: ``ncol`` seeded columns of 50 layers with
the same two species and mixing ratios log-uniform over 0.01-2 g/kg.

``uneven_batch`` is the uneven workload: layer counts uniform over 40-150,
1-5 species per column drawn from cloud water, cloud ice, snow, graupel and
rain with exponential or modified-gamma size distributions (mu uniform over
0-4), 20-80 bins each, ice densities 100-900 kg/m3 (soft spheres, Sihvola
mixing), 8-32 frequencies per column from 10-183 GHz and NUMMU from
{8, 16, 32}, all per column.

``target_batch`` is the 150-layer, 16-angle, 4-species shape: 150 layers
over 0-15 km with cloud water, cloud ice, snow and rain in overlapping bands.

``mie_heavy_batch`` is the Mie-heavy workload: 100 layers over 0-12 km, rain,
snow, graupel and cloud ice with 200 bins each (sizes up to 10 mm, size
parameters up to about 19 at 190 GHz), at 89, 157, 176.31 and 190.31 GHz.
"""

import warnings

import numpy as np

from . import batch as _batch
from . import core, importer, meteoSI, packing

GOLDEN_FREQS = [10.65, 35.5]
C1_FREQS = [23.8, 31.4, 89.0]
C2_FREQS = [23.8, 31.4, 89.0, 150.0]

RAIN_GOLDEN = ("rwc_q", -99.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 3, 30, "exp", -99.0, -99.0, 8.0e6, -99.0,
               1.0e-5, 6.0e-3, "mie-sphere", "khvorostyanov01_drops", -99.0)
SNOW_GOLDEN = ("swc_q", -99.0, -1, -99.0, 0.038, 2.0, 0.3971, 1.88, 3, 30, "exp_field_t", -99.0, -99.0, -99.0,
               -99.0, 0.51e-10, 2.0e-2, "mie-sphere", "heymsfield10_particles", -99.0)
# cloud liquid: exponential PSD with fixed effective radius p_2 = 10 um
CLOUD_C1 = ("cwc_q", -99.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 3, 40, "exp", -99.0, 1.0e-5, -99.0, -99.0,
            2.0e-6, 1.0e-4, "mie-sphere", "corPowerLaw_24388657.6_2.0", -99.0)
# rain: Marshall-Palmer (exponential, N0 = 8e6 m^-4)
RAIN_C1 = ("rwc_q", -99.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 3, 50, "exp", -99.0, -99.0, 8.0e6, -99.0,
           1.0e-4, 6.0e-3, "mie-sphere", "khvorostyanov01_drops", -99.0)


def golden_pam():
    warnings.simplefilter("ignore")
    pam = core.pyPamtra()
    pam.df.addHydrometeor(RAIN_GOLDEN)
    pam.df.addHydrometeor(SNOW_GOLDEN)
    pam = importer.createUsStandardProfile(pam, hgt_lev=[0.0, 1000.0, 2000.0, 3000.0])
    pam.nmlSet["randomseed"] = 10
    pam.p["hydro_q"][0, 0, 1, 0] = 1e-3
    pam.p["hydro_q"][0, 0, 2, 1] = 5e-4
    return pam


def _columns(ncol, nlay, seed, q_cloud=None, q_rain=None):
    rng = np.random.default_rng(seed)
    hgt_lev = np.linspace(0.0, 12000.0, nlay + 1)
    _, p0, t0 = meteoSI.usStandard(hgt_lev)
    temp_lev = t0[None, :] + rng.uniform(-1.0, 1.0, (ncol, nlay + 1))
    press_lev = p0[None, :] * (1.0 + rng.uniform(-0.005, 0.005, (ncol, nlay + 1)))
    relhum_lev = rng.uniform(40.0, 95.0, (ncol, nlay + 1))
    hydro_q = np.zeros((ncol, nlay, 2))
    cloud = slice(5, 26)
    if q_cloud is None:
        hydro_q[:, cloud, 0] = 10 ** rng.uniform(np.log10(1e-5), np.log10(2e-3), (ncol, 21))
        hydro_q[:, cloud, 1] = 10 ** rng.uniform(np.log10(1e-5), np.log10(2e-3), (ncol, 21))
    else:
        hydro_q[:, cloud, 0] = q_cloud
        hydro_q[:, cloud, 1] = q_rain
    return dict(hgt_lev=np.repeat(hgt_lev[None, :], ncol, 0), temp_lev=temp_lev, press_lev=press_lev,
                relhum_lev=relhum_lev, hydro_q=hydro_q)


def _pam_from(cols, ncol, nlay):
    warnings.simplefilter("ignore")
    pam = core.pyPamtra()
    pam.df.addHydrometeor(CLOUD_C1)
    pam.df.addHydrometeor(RAIN_C1)
    pam.nmlSet["hydro_adaptive_grid"] = False
    pam.nmlSet["emissivity"] = 0.5
    pam.createProfile(hgt_lev=cols["hgt_lev"].reshape(ncol, 1, nlay + 1),
                      temp_lev=cols["temp_lev"].reshape(ncol, 1, nlay + 1),
                      press_lev=cols["press_lev"].reshape(ncol, 1, nlay + 1),
                      relhum_lev=cols["relhum_lev"].reshape(ncol, 1, nlay + 1),
                      hydro_q=cols["hydro_q"].reshape(ncol, 1, nlay, 2),
                      groundtemp=290.0, sfc_refl="S",
                      obs_height=np.tile([833000.0, 0.0], (ncol, 1, 1)))
    return pam


def c1_pam(seed=1):
    return _pam_from(_columns(1, 50, seed, q_cloud=3e-4, q_rain=5e-4), 1, 50)


def c2_pam(ncol=4096, seed=2):
    return _pam_from(_columns(ncol, 50, seed), ncol, 50)


# ------------------------------------------------------------------ packed (per-column) workloads
# species kinds: (liq_ice, d_1, d_2, effective radius p_2 of the gamma forms, band bottom/top in m)
_KINDS = {
    "cwc": (1, 2.0e-6, 1.0e-4, 1.0e-5, 500.0, 6000.0),
    "iwc": (-1, 1.0e-5, 2.0e-3, 5.0e-5, 6000.0, 12000.0),
    "swc": (-1, 1.0e-4, 1.0e-2, 5.0e-4, 3000.0, 10000.0),
    "gwc": (-1, 1.0e-4, 8.0e-3, 4.0e-4, 2000.0, 8000.0),
    "rwc": (1, 1.0e-4, 6.0e-3, 3.0e-4, 0.0, 4000.0),
}
_KIND_ORDER = ("cwc", "iwc", "swc", "gwc", "rwc")


def _species_row(kind, rng, nbin=None, gamma=None, rho=None):
    li, d1, d2, reff, _, _ = _KINDS[kind]
    r = np.zeros((), dtype=packing.SPECIES_DTYPE)
    for k in ("as_ratio", "rho_ms", "a_ms", "b_ms", "alpha_as", "beta_as", "p_1", "p_2", "p_3", "p_4"):
        r[k] = -99.0
    r["liq_ice"] = li
    r["moment_in"] = 3
    r["nbin"] = int(rng.integers(20, 81)) if nbin is None else nbin
    use_gamma = (rng.random() < 0.5) if gamma is None else gamma
    if li == -1:
        r["rho_ms"] = float(rng.uniform(100.0, 900.0)) if rho is None else rho
    if use_gamma:
        r["dist"] = packing.DIST_CODES["mgamma"]
        r["p_2"] = reff
        r["p_3"] = float(rng.uniform(0.0, 4.0))
        r["p_4"] = 1.0
    else:
        r["dist"] = packing.DIST_CODES["exp"]
        if kind == "rwc":
            r["p_3"] = 8.0e6  # Marshall-Palmer intercept
        else:
            r["p_2"] = reff
    r["d_1"], r["d_2"] = d1, d2
    return r


def _settings(nummu=16):
    warnings.simplefilter("ignore")
    nml = dict(core.pyPamtra().nmlSet)
    nml["hydro_adaptive_grid"] = False
    nml["emissivity"] = 0.5
    return packing.settings_from_nml(nml, nummu)


def _atmosphere(rng, nl, top):
    h = np.linspace(0.0, top, nl + 1)
    _, p0, t0 = meteoSI.usStandard(h)
    t = t0 + rng.uniform(-1.0, 1.0, nl + 1)
    p = p0 * (1.0 + rng.uniform(-0.005, 0.005, nl + 1))
    rh = rng.uniform(40.0, 95.0, nl + 1)
    return h, t, p, rh


def _packed(st, species, stride, nly, freqs_list, nummu, kinds_list, qs, top, rng, Lm, H, per_freq):
    C = len(nly)
    F = max(len(f) for f in freqs_list)
    host = dict()
    for k in ("hgt_lev", "temp_lev", "press_lev", "relhum_lev"):
        host[k] = np.full((C, Lm + 1), np.nan)
    for k in ("hgt", "temp", "press", "relhum"):
        host[k] = np.full((C, Lm), np.nan)
    hq = np.zeros((C, Lm, H))
    for c in range(C):
        nl = int(nly[c])
        h, t, p, rh = _atmosphere(rng, nl, top[c])
        host["hgt_lev"][c, :nl + 1], host["temp_lev"][c, :nl + 1] = h, t
        host["press_lev"][c, :nl + 1], host["relhum_lev"][c, :nl + 1] = p, rh
        host["hgt"][c, :nl] = 0.5 * (h[1:] + h[:-1])
        mid = host["hgt"][c, :nl]
        for j, kind in enumerate(kinds_list[c]):
            if kind is None:
                continue
            lo, hi = _KINDS[kind][4], _KINDS[kind][5]
            band = (mid >= lo) & (mid <= hi)
            hq[c, :nl, j] = np.where(band, qs[c][j] * 10 ** rng.uniform(-0.5, 0.5, nl), 0.0)
    host["hydro_q"] = hq
    host["hydro_n"] = np.zeros_like(hq)
    host["hydro_reff"] = np.zeros_like(hq)
    host["nlyrs"] = np.ascontiguousarray(np.asarray(nly, dtype=np.int32))
    host["groundtemp"] = np.full(C, 290.0)
    host["obs_height"] = np.tile([833000.0, 0.0], (C, 1))
    host["sfc_refl"] = np.full(C, ord("S"), dtype=np.int8)
    host["ncol"], host["max_nlyrs"], host["noutlevels"], host["nhydro"] = C, Lm, 2, H
    host["max_nfreq"] = F
    if per_freq:
        fr = np.zeros((C, F))
        for c, f in enumerate(freqs_list):
            fr[c, :len(f)] = f
        host["freqs"] = fr
        host["nfreq"] = np.asarray([len(f) for f in freqs_list], dtype=np.int32)
    else:
        host["freqs"] = np.asarray(freqs_list[0], dtype=np.float64)
    if nummu is not None:
        host["nummu"] = np.asarray(nummu, dtype=np.int32)
    return _batch.pack_columns(st, species, host, stride)


def uneven_batch(ncol=16384, seed=3, nummu_choices=(8, 16, 32), nfreq_range=(8, 32)):
    """Seeded uneven batch (per-column layers, species, frequencies, NUMMU)."""
    rng = np.random.default_rng(seed)
    H = 5
    st = _settings(16)
    nly = rng.integers(40, 151, ncol)
    top = nly * 100.0  # 100 m layers
    nummu = rng.choice(np.asarray(nummu_choices), ncol)
    sp = np.empty(ncol * H, dtype=packing.SPECIES_DTYPE)
    kinds_list, qs, freqs_list = [], [], []
    for c in range(ncol):
        nk = int(rng.integers(1, 6))
        chosen = sorted(rng.choice(H, nk, replace=False).tolist())
        kl = [None] * H
        qq = [0.0] * H
        for j in range(H):
            if j in chosen:
                kl[j] = _KIND_ORDER[j]
                sp[c * H + j] = _species_row(_KIND_ORDER[j], rng)
                qq[j] = 10 ** rng.uniform(-5.0, np.log10(2e-3))
            else:
                sp[c * H + j] = packing.disabled_species()
        kinds_list.append(kl)
        qs.append(qq)
        nf = int(rng.integers(nfreq_range[0], nfreq_range[1] + 1))
        freqs_list.append(np.sort(rng.uniform(10.0, 183.0, nf)))
    return _packed(st, sp, H, nly, freqs_list, nummu, kinds_list, qs, top, rng, int(nly.max()), H, True)


TARGET_FREQS = [23.8, 31.4, 89.0, 150.0]


def target_batch(ncol=1024, seed=4):
    """150-layer, NUMMU = 16 columns with four species (cloud water, cloud
    ice, snow, rain), shared species table and frequencies."""
    rng = np.random.default_rng(seed)
    st = _settings(16)
    kinds = ["cwc", "iwc", "swc", "rwc"]
    sp = np.empty(4, dtype=packing.SPECIES_DTYPE)
    for j, k in enumerate(kinds):
        sp[j] = _species_row(k, np.random.default_rng(100 + j), nbin=40, gamma=(k != "rwc"), rho=300.0)
    nly = np.full(ncol, 150)
    top = np.full(ncol, 15000.0)
    qs = [[10 ** rng.uniform(-5.0, np.log10(2e-3)) for _ in kinds] for _ in range(ncol)]
    return _packed(st, sp, 0, nly, [TARGET_FREQS], None, [kinds] * ncol, qs, top, rng, 150, 4, False)


MIE_HEAVY_FREQS = [89.0, 157.0, 176.31, 190.31]


def mie_heavy_batch(ncol=2048, seed=6):
    """Mie-heavy columns: 100 layers, four species of 200 bins (rain up to
    6 mm, snow up to 10 mm, graupel up to 8 mm, cloud ice up to 2 mm), shared
    species table and frequencies 89/157/176.31/190.31 GHz."""
    rng = np.random.default_rng(seed)
    st = _settings(16)
    kinds = ["rwc", "swc", "gwc", "iwc"]
    sp = np.empty(4, dtype=packing.SPECIES_DTYPE)
    for j, k in enumerate(kinds):
        sp[j] = _species_row(k, np.random.default_rng(200 + j), nbin=200, gamma=(k != "rwc"), rho=400.0)
    nly = np.full(ncol, 100)
    top = np.full(ncol, 12000.0)
    qs = [[10 ** rng.uniform(-5.0, np.log10(2e-3)) for _ in kinds] for _ in range(ncol)]
    return _packed(st, sp, 0, nly, [MIE_HEAVY_FREQS], None, [kinds] * ncol, qs, top, rng, 100, 4, False)


# ------------------------------------------------------------------ full size spectra
ICE_FS = ("ice", 1.0, -1, 200.0, -99.0, -99.0, np.pi / 4.0, 2.0, 0, 40, "exp", 3000.0, 3e8, -99.0, -99.0, 100e-6,
          1000e-6, "mie-sphere", "heymsfield10_particles", 0.0)
RAIN_FS = ("rain", 1.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 0, 40, "exp", 2000.0, 8e6, -99.0, -99.0, 100e-6,
           6000e-6, "mie-sphere", "khvorostyanov01_drops", 0.0)


def fullspec_pam(ncol=4, nlay=30, seed=7):
    """Columns whose size distributions are given as full spectra
    (``nmlSet['hydro_fullspec']``): soft ice spheres (200 kg/m3, 100-1000 um)
    and rain (100 um - 6 mm), 40 bins each, on per-(column, layer) bin edges
    with exponential spectra of seeded slope and intercept; about a quarter
    of the (layer, species) slots are left empty."""
    warnings.simplefilter("ignore")
    rng = np.random.default_rng(seed)
    cols = _columns(ncol, nlay, seed, q_cloud=0.0, q_rain=0.0)
    pam = core.pyPamtra()
    pam.df.addHydrometeor(ICE_FS)
    pam.df.addHydrometeor(RAIN_FS)
    pam.nmlSet["hydro_adaptive_grid"] = False
    pam.nmlSet["emissivity"] = 0.5
    pam.createProfile(hgt_lev=cols["hgt_lev"].reshape(ncol, 1, nlay + 1),
                      temp_lev=cols["temp_lev"].reshape(ncol, 1, nlay + 1),
                      press_lev=cols["press_lev"].reshape(ncol, 1, nlay + 1),
                      relhum_lev=cols["relhum_lev"].reshape(ncol, 1, nlay + 1),
                      hydro_q=np.zeros((ncol, 1, nlay, 2)), groundtemp=290.0, sfc_refl="S",
                      obs_height=np.tile([833000.0, 0.0], (ncol, 1, 1)))
    pam.nmlSet["hydro_fullspec"] = True
    pam.df.addFullSpectra()
    fs = pam.df.dataFullSpec
    nb = pam.df.fs_nbin
    for h, (d1, d2, rho) in enumerate(((100e-6, 1000e-6, 200.0), (100e-6, 6000e-6, 1000.0))):
        jit = rng.uniform(0.9, 1.1, (ncol, 1, nlay, 1))
        edges = np.exp(np.linspace(np.log(d1), np.log(d2), nb + 1))[None, None, None, :] * jit
        fs["d_bound_ds"][..., h, :] = edges
        d = 0.5 * (edges[..., 1:] + edges[..., :-1])
        fs["d_ds"][..., h, :] = d
        lam = 10 ** rng.uniform(3.0, 4.0, (ncol, 1, nlay, 1))
        n0 = 10 ** rng.uniform(6.0, 8.0, (ncol, 1, nlay, 1))
        n = n0 * np.exp(-lam * d) * np.diff(edges, axis=-1)
        n *= (rng.uniform(size=(ncol, 1, nlay, 1)) > 0.25)
        fs["n_ds"][..., h, :] = n
        fs["rho_ds"][..., h, :] = rho
        fs["mass_ds"][..., h, :] = np.pi / 6.0 * rho * d ** 3
        fs["area_ds"][..., h, :] = np.pi / 4.0 * d ** 2
        fs["as_ratio"][..., h, :] = 1.0
    return pam
