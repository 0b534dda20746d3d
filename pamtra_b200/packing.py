"""Host-side packer: turns the pyPamtra session state (``nmlSet``, descriptor
table, profile dict ``p``) into the flat column-major-by-column arrays the
C-ABI takes.  This replaces the module-global copies that the reference's
``PamtraFortranWrapper`` performs (python/pyPamtra/libWrapper.py:24-207).

Columns are the flattened (ngridx, ngridy) grid in C order.
"""

import ctypes

import numpy as np

# dist_name codes shared with the native library (include/pamtra_b200.h)
DIST_CODES = {"exp": 0, "exp_field_t": 1, "mgamma": 2, "mono": 3, "exp_cosmo_snow": 4,
              "exp_ryan": 5, "logn": 6, "disabled": 7}
# scat_name codes: only Mie spheres are on this path
SCAT_CODES = {"mie-sphere": 0, "disabled": 1}

# nmlSet['liq_mod'] / nmlSet['gas_mod'] codes (PAMTRA_B200_LIQ_* / _GAS_*)
LIQ_MODS = {"TKC": 0, "Ell": 1, "Lie": 2, "Ray": 3, "Sto": 4}
GAS_MODS = {"R98": 0, "L93": 1}

MAXNLEG = 200
# radar_attenuation codes (PAMTRA_B200_ATT_*)
RADAR_ATTENUATION = {"disabled": 0, "bottom-up": 1, "top-down": 2}


class Settings(ctypes.Structure):
    """Mirror of ``pamtra_b200_settings`` (include/pamtra_b200.h)."""
    _fields_ = [
        ("emissivity", ctypes.c_double),
        ("hydro_threshold", ctypes.c_double),
        ("hydro_softsphere_min_density", ctypes.c_double),
        ("lgas_extinction", ctypes.c_int32),
        ("lhyd_absorption", ctypes.c_int32),
        ("lhyd_scattering", ctypes.c_int32),
        ("lhyd_emission", ctypes.c_int32),
        ("hydro_includehydroinrhoair", ctypes.c_int32),
        ("hydro_adaptive_grid", ctypes.c_int32),
        ("conserve_mass_rescale_dsd", ctypes.c_int32),
        ("hydro_limit_density_area", ctypes.c_int32),
        ("outpol_vh", ctypes.c_int32),
        ("nummu", ctypes.c_int32),
        ("active", ctypes.c_int32),
        ("radar_attenuation", ctypes.c_int32),
        ("radar_k2", ctypes.c_double),
        ("liq_mod", ctypes.c_int32),
        ("gas_mod", ctypes.c_int32),
    ]


class Species(ctypes.Structure):
    """Mirror of ``pamtra_b200_species``: one descriptor-file row."""
    _fields_ = [
        ("liq_ice", ctypes.c_int32),
        ("moment_in", ctypes.c_int32),
        ("nbin", ctypes.c_int32),
        ("dist", ctypes.c_int32),
        ("as_ratio", ctypes.c_double),
        ("rho_ms", ctypes.c_double),
        ("a_ms", ctypes.c_double),
        ("b_ms", ctypes.c_double),
        ("alpha_as", ctypes.c_double),
        ("beta_as", ctypes.c_double),
        ("p_1", ctypes.c_double),
        ("p_2", ctypes.c_double),
        ("p_3", ctypes.c_double),
        ("p_4", ctypes.c_double),
        ("d_1", ctypes.c_double),
        ("d_2", ctypes.c_double),
    ]


SPECIES_DTYPE = np.dtype([(name, np.int32 if ct is ctypes.c_int32 else np.float64)
                          for name, ct in Species._fields_])
assert SPECIES_DTYPE.itemsize == ctypes.sizeof(Species)


def settings_from_nml(nmlSet, nummu=16):
    """Validate the namelist keys this path honours and build the settings
    struct.  Options whose reference branch is not on the passive Mie path
    raise NotImplementedError instead of silently changing behaviour."""
    gas = str(nmlSet.get("gas_mod", "R98")).strip()
    if gas not in GAS_MODS:
        # settings.f90:286-287
        raise ValueError("gas_mod has to be L93 or R98")
    liq = str(nmlSet.get("liq_mod", "TKC")).strip()
    if liq not in LIQ_MODS:
        # eps_water.f90:59-63
        raise ValueError("Do not know liq_mod: %s" % liq)
    outpol = str(nmlSet.get("outpol", "VH")).strip()
    if outpol not in ("VH", "IQ"):
        raise ValueError("outpol must be VH or IQ")
    s = Settings()
    s.emissivity = float(nmlSet["emissivity"])
    s.hydro_threshold = float(nmlSet["hydro_threshold"])
    s.hydro_softsphere_min_density = float(nmlSet["hydro_softsphere_min_density"])
    s.lgas_extinction = int(bool(nmlSet["lgas_extinction"]))
    s.lhyd_absorption = int(bool(nmlSet["lhyd_absorption"]))
    s.lhyd_scattering = int(bool(nmlSet["lhyd_scattering"]))
    s.lhyd_emission = int(bool(nmlSet["lhyd_emission"]))
    s.hydro_includehydroinrhoair = int(bool(nmlSet["hydro_includehydroinrhoair"]))
    s.hydro_adaptive_grid = int(bool(nmlSet["hydro_adaptive_grid"]))
    s.conserve_mass_rescale_dsd = int(bool(nmlSet["conserve_mass_rescale_dsd"]))
    s.hydro_limit_density_area = int(bool(nmlSet["hydro_limit_density_area"]))
    s.outpol_vh = int(outpol == "VH")
    s.nummu = int(nummu)
    s.active = int(bool(nmlSet.get("active", False)))
    att = str(nmlSet.get("radar_attenuation", "disabled")).strip()
    if att not in RADAR_ATTENUATION:
        raise ValueError("radar_attenuation must be one of %s" % sorted(RADAR_ATTENUATION))
    s.radar_attenuation = RADAR_ATTENUATION[att]
    s.radar_k2 = float(nmlSet.get("radar_k2", 0.93))
    s.liq_mod = LIQ_MODS[liq]
    s.gas_mod = GAS_MODS[gas]
    if s.active and str(nmlSet.get("radar_mode", "simple")).strip() != "simple":
        raise NotImplementedError("radar_mode %r: only 'simple' is on this path" % nmlSet["radar_mode"])
    return s


def disabled_species():
    """A species slot that takes no part (dist ``disabled``), used to pad
    columns with fewer species in a batch with per-column species tables."""
    r = np.zeros((), dtype=SPECIES_DTYPE)
    for k in ("as_ratio", "rho_ms", "a_ms", "b_ms", "alpha_as", "beta_as", "p_1", "p_2", "p_3", "p_4", "d_1", "d_2"):
        r[k] = -99.0
    r["liq_ice"], r["moment_in"], r["nbin"] = 1, 3, 2
    r["dist"] = DIST_CODES["disabled"]
    return r


def species_from_df(data, fullspec=False):
    """Descriptor recarray -> structured array of ``pamtra_b200_species``.
    With ``fullspec`` (sizes from ``dataFullSpec``) ``dist_name`` is not read
    (src/hydrometeor_extinction.f90:122-151); a species whose ``scat_name`` is
    'disabled' still marks its layers as carrying hydrometeors but adds no
    scattering (src/scatProperties.f90:203)."""
    out = np.zeros(len(data), dtype=SPECIES_DTYPE)
    for i, row in enumerate(data):
        dist = str(row["dist_name"]).strip()
        scat = str(row["scat_name"]).strip()
        if fullspec:
            dist = "exp"
        if dist not in DIST_CODES or dist == "exp_cosmo_snow":
            raise NotImplementedError("dist_name %r is not on this path" % dist)
        if scat == "tmatrix":
            raise NotImplementedError(
                "scat_name 'tmatrix' inside runPamtra is not wired into the forward run yet; the species' "
                "single-scattering matrices are available from pamtra_b200.tmatrix.calc_tmatrix")
        if scat not in SCAT_CODES:
            raise NotImplementedError("scat_name %r is not on this path (mie-sphere only)" % scat)
        out[i]["liq_ice"] = int(row["liq_ice"])
        out[i]["moment_in"] = int(row["moment_in"])
        out[i]["nbin"] = int(row["nbin"])
        out[i]["dist"] = DIST_CODES["disabled"] if scat == "disabled" else DIST_CODES[dist]
        for k in ("as_ratio", "rho_ms", "a_ms", "b_ms", "alpha_as", "beta_as", "p_1", "p_2", "p_3", "p_4",
                  "d_1", "d_2"):
            out[i][k] = float(row[k])
    return out


FULLSPEC_KEYS = ("d_ds", "d_bound_ds", "n_ds", "rho_ds", "mass_ds")


def fullspec_columns(cols, dataFullSpec):
    """Add the full spectra of ``dataFullSpec`` (descriptorFile.addFullSpectra)
    to packed ``cols`` as ``fs_d``, ``fs_d_bound``, ``fs_n``, ``fs_rho``,
    ``fs_mass``: C-contiguous float64, one row per column,
    [max_nlyrs][nhydro][nbin] (``fs_d_bound``: nbin + 1), plus ``fs_nbin``."""
    ncol, L = cols["ncol"], cols["max_nlyrs"]
    nh = cols["hydro_q"].shape[-1]
    for k in FULLSPEC_KEYS:
        if k not in dataFullSpec:
            raise ValueError("hydro_fullspec: dataFullSpec[%r] is missing" % k)
    nb = int(np.asarray(dataFullSpec["d_ds"]).shape[-1])
    for k in FULLSPEC_KEYS:
        tail = nb + 1 if k == "d_bound_ds" else nb
        a = np.asarray(dataFullSpec[k], dtype=np.float64)
        if a.size != ncol * L * nh * tail:
            raise ValueError("hydro_fullspec: dataFullSpec[%r] has shape %s, expected (ngridx, ngridy, %d, %d, %d)"
                             % (k, a.shape, L, nh, tail))
        cols["fs_" + k[:-3]] = np.ascontiguousarray(a.reshape(ncol, L, nh, tail))
    cols["fs_nbin"] = nb
    return cols


def profile_columns(p, nhydro):
    """Profile dict -> dict of C-contiguous float64/int arrays, one row per
    column (flattened x, y)."""
    nx, ny, L = int(p["ngridx"]), int(p["ngridy"]), int(p["max_nlyrs"])
    ncol = nx * ny

    def col(key, tail, fill=np.nan):
        if key in p and isinstance(p[key], np.ndarray) and p[key].size > 0:
            a = np.asarray(p[key], dtype=np.float64).reshape((ncol,) + tail)
        else:
            a = np.full((ncol,) + tail, fill)
        return np.ascontiguousarray(a)

    cols = dict()
    cols["nlyrs"] = np.ascontiguousarray(np.asarray(p["nlyrs"]).reshape(ncol).astype(np.int32))
    for k in ("hgt_lev", "temp_lev", "press_lev", "relhum_lev"):
        cols[k] = col(k, (L + 1,))
    for k in ("hgt", "temp", "press", "relhum"):
        cols[k] = col(k, (L,))
    for k in ("hydro_q", "hydro_n", "hydro_reff"):
        cols[k] = col(k, (L, nhydro), fill=0.0) if nhydro > 0 else np.zeros((ncol, L, 0))
    cols["groundtemp"] = col("groundtemp", ())
    nout = int(p["noutlevels"])
    cols["obs_height"] = col("obs_height", (nout,))
    refl = np.asarray(p["sfc_refl"]).reshape(ncol)
    refl = np.array([(r.decode() if isinstance(r, bytes) else str(r))[:1] or 'S' for r in refl])
    cols["sfc_refl"] = np.ascontiguousarray(np.frombuffer("".join(refl).encode(), dtype=np.int8).copy())
    sfc_type = np.asarray(p.get("sfc_type", np.full(ncol, -9999))).reshape(ncol)
    if np.any((sfc_type == 0) | (sfc_type == 1)):
        raise NotImplementedError("sfc_type 0/1 (ocean/land emissivity models) is not on this path")
    cols["ncol"] = ncol
    cols["max_nlyrs"] = L
    cols["noutlevels"] = nout
    return cols
