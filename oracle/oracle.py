"""ctypes front end of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  It runs the C++ restatement in ``pamtra_oracle.cpp`` column by
column, mirroring ``PamtraFortranWrapper`` (python/pyPamtra/libWrapper.py:24)
of the reference.
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
MAXNLEG = 200

_lib = None


class OrcSettings(ctypes.Structure):
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


class OrcFullspec(ctypes.Structure):
    _fields_ = [("nbin", ctypes.c_int32), ("d", ctypes.c_void_p), ("d_bound", ctypes.c_void_p),
                ("n", ctypes.c_void_p), ("rho", ctypes.c_void_p), ("mass", ctypes.c_void_p),
                ("as_ratio", ctypes.c_void_p), ("canting", ctypes.c_void_p)]


PSD_KEYS = ("psd_d", "psd_deltad", "psd_n", "psd_mass", "psd_area", "psd_bscat")


class OrcDebug(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in
                ("kextatmo", "kexttot", "salbedo", "nlegen", "legen", "present", "scatter_matrix", "ext",
                 "emis", "num_doubles", "back", "ze", "att_hydro", "att_atmo")] + \
        [("psd_nbin", ctypes.c_int32)] + [(k, ctypes.c_void_p) for k in PSD_KEYS]


def build():
    """Compile the oracle with its Makefile (g++ only)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        l = ctypes.CDLL(LIB)
        dp = ctypes.POINTER(ctypes.c_double)
        l.orc_run_column.restype = ctypes.c_int
        l.orc_run_column.argtypes = [ctypes.POINTER(OrcSettings), ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                     dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, dp, ctypes.c_double, ctypes.c_int,
                                     dp, ctypes.c_char, ctypes.c_int, dp, dp, dp, dp,
                                     ctypes.POINTER(OrcDebug)]
        l.orc_run_column_fs.restype = ctypes.c_int
        l.orc_run_column_fs.argtypes = l.orc_run_column.argtypes + [ctypes.POINTER(OrcFullspec)]
        l.orc_run_column_tm.restype = ctypes.c_int
        l.orc_run_column_tm.argtypes = l.orc_run_column_fs.argtypes + [ctypes.c_void_p, dp]
        l.orc_gas_r98.restype = ctypes.c_int
        l.orc_gas_r98.argtypes = [ctypes.c_double] * 4 + [dp]
        l.orc_get_eps_water.restype = ctypes.c_int
        l.orc_get_eps_water.argtypes = [ctypes.c_int] + [ctypes.c_double] * 3 + [dp, dp]
        l.orc_gas_l93.restype = ctypes.c_double
        l.orc_gas_l93.argtypes = [ctypes.c_double] * 4
        l.orc_eps_water_tkc.restype = None
        l.orc_eps_water_tkc.argtypes = [ctypes.c_double, ctypes.c_double, dp, dp]
        l.orc_lobatto.argtypes = [ctypes.c_int, dp, dp]
        fp = ctypes.POINTER(ctypes.c_float)
        l.orc_tmatrix_single.restype = ctypes.c_int
        l.orc_tmatrix_single.argtypes = [ctypes.c_int] + [ctypes.c_double] * 6 + [dp] * 4
        l.orc_tmatrix_tmat.restype = ctypes.c_int
        l.orc_tmatrix_tmat.argtypes = [ctypes.c_double] * 5 + [ctypes.c_int, fp, fp]
        l.orc_tmatrix_species.restype = ctypes.c_int
        l.orc_tmatrix_species.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_int] + [dp] * 11
        l.orc_layer_start.restype = ctypes.c_int
        l.orc_layer_start.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4 + [dp, ctypes.c_double, ctypes.c_double,
                                                                                ctypes.c_void_p, ctypes.c_void_p] + \
            [dp] * 4
        l.orc_miecalc.restype = ctypes.c_int
        l.orc_miecalc.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int] + [dp] * 4
        l.orc_minvert.restype = ctypes.c_int
        l.orc_minvert.argtypes = [ctypes.c_int, dp, dp]
        l.orc_e_sat.argtypes = [ctypes.c_double, dp]
        _lib = l
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def settings(pk_settings):
    """Copy a pamtra_b200.packing.Settings into the oracle's struct."""
    s = OrcSettings()
    for name, _ in OrcSettings._fields_:
        setattr(s, name, getattr(pk_settings, name))
    return s


def run_column(st, species, cols, c, freqs, debug=False, psd_nbin=0, scat_code=None, canting=None,
               fs_as_ratio=None, fs_canting=None):
    """Run column ``c`` of packed ``cols`` (pamtra_b200.packing.profile_columns).
    ``debug`` True returns all intermediates, "radar" only the simple-radar
    outputs (back, ze, att_hydro, att_atmo; filled when ``st.active``).
    ``psd_nbin`` > 0 adds the save_psd bins, [L][nhydro][psd_nbin].
    ``scat_code`` (per species, 1 = T-matrix spheroid of the species' aspect
    ratio, 0 = Mie sphere) and ``canting`` (deg, per species) select the
    scattering model of scatProperties.f90:289-367; with full spectra the
    T-matrix species take ``fs_as_ratio`` / ``fs_canting`` of this column,
    [L][nhydro][nbin] (hydrofs_as_ratio / hydrofs_canting, :257-265)."""
    l = lib()
    L = int(cols["nlyrs"][c])
    Lmax = int(cols["max_nlyrs"])
    H = len(species)
    N = st.nummu
    nf = len(freqs)
    nout = int(cols["noutlevels"])
    f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))
    hl = {k: f64(cols[k][c, :L + 1]) for k in ("hgt_lev", "temp_lev", "press_lev", "relhum_lev")}
    ly = {k: f64(cols[k][c, :L]) for k in ("hgt", "temp", "press", "relhum")}
    hq = {k: f64(cols[k][c, :L, :]) if H else np.zeros(1) for k in ("hydro_q", "hydro_n", "hydro_reff")}
    obs = f64(cols["obs_height"][c])
    fr = f64(freqs)
    tb = np.zeros((nout, 2 * N, nf, 2))
    em = np.zeros((2, nf, N))
    ang = np.zeros(2 * N)
    dbg = None
    out_dbg = None
    if debug == "radar":
        out_dbg = dict(back=np.zeros((nf, L)), ze=np.zeros((nf, L)), att_hydro=np.zeros((nf, L)),
                       att_atmo=np.zeros((nf, L)))
        dbg = OrcDebug(**{k: v.ctypes.data for k, v in out_dbg.items()})
    elif debug:
        n = 2 * N
        out_dbg = dict(kextatmo=np.zeros((nf, L)), kexttot=np.zeros((nf, L)), salbedo=np.zeros((nf, L)),
                       nlegen=np.zeros((nf, L), np.int32), legen=np.zeros((nf, L, 3, MAXNLEG)),
                       present=np.zeros(L, np.int32), scatter_matrix=np.zeros((nf, L, 4, n, n)),
                       ext=np.zeros((nf, L)), emis=np.zeros((nf, L)), num_doubles=np.zeros((nf, L), np.int32),
                       back=np.zeros((nf, L)), ze=np.zeros((nf, L)), att_hydro=np.zeros((nf, L)),
                       att_atmo=np.zeros((nf, L)))
        dbg = OrcDebug(**{k: v.ctypes.data for k, v in out_dbg.items()})
    if psd_nbin > 0:
        if out_dbg is None:
            out_dbg = dict()
            dbg = OrcDebug()
        for k in PSD_KEYS:
            out_dbg[k] = np.full((L, H, psd_nbin), -9999.0)
            setattr(dbg, k, out_dbg[k].ctypes.data)
        dbg.psd_nbin = psd_nbin
    sp = np.ascontiguousarray(species)
    refl = bytes([int(cols["sfc_refl"][c]) & 0xFF])
    args = [ctypes.byref(st), sp.ctypes.data if H else None, H, L,
            _p(hl["hgt_lev"]), _p(hl["temp_lev"]), _p(hl["press_lev"]), _p(hl["relhum_lev"]),
            _p(ly["hgt"]), _p(ly["temp"]), _p(ly["press"]), _p(ly["relhum"]),
            _p(hq["hydro_q"]), _p(hq["hydro_n"]), _p(hq["hydro_reff"]),
            float(cols["groundtemp"][c]), nout, _p(obs), refl, nf, _p(fr), _p(tb), _p(em),
            _p(ang), ctypes.byref(dbg) if dbg is not None else None]
    if cols.get("fs_d") is not None:
        # full spectra of this column, [L][H][nbin] (+1 for the bin bounds)
        fsa = {k: f64(cols[k][c, :L]) for k in ("fs_d", "fs_d_bound", "fs_n", "fs_rho", "fs_mass")}
        fs = OrcFullspec(int(cols["fs_nbin"]), *[fsa[k].ctypes.data for k in
                                                  ("fs_d", "fs_d_bound", "fs_n", "fs_rho", "fs_mass")])
        if scat_code is not None:
            keep = [f64(fs_as_ratio) if fs_as_ratio is not None else None,
                    f64(fs_canting) if fs_canting is not None else None]
            fs.as_ratio = keep[0].ctypes.data if keep[0] is not None else None
            fs.canting = keep[1].ctypes.data if keep[1] is not None else None
            sc = np.ascontiguousarray(np.asarray(scat_code, dtype=np.int32))
            ct = f64(canting if canting is not None else np.zeros(H))
            err = l.orc_run_column_tm(*(args + [ctypes.byref(fs), sc.ctypes.data, _p(ct)]))
        else:
            err = l.orc_run_column_fs(*(args + [ctypes.byref(fs)]))
    elif scat_code is not None:
        sc = np.ascontiguousarray(np.asarray(scat_code, dtype=np.int32))
        ct = f64(canting if canting is not None else np.zeros(H))
        err = l.orc_run_column_tm(*(args + [None, sc.ctypes.data, _p(ct)]))
    else:
        err = l.orc_run_column(*args)
    return err, tb, em, ang, out_dbg


def run_pamtra(pam, freqs, nummu=16, debug=False):
    """Oracle counterpart of ``pyPamtra.runPamtra``: returns a results dict with
    ``tb`` (ngridx, ngridy, noutlevels, 2N, nfreq, 2), ``emissivity``,
    ``angles_deg`` and the error code."""
    from pamtra_b200 import packing
    st = settings(packing.settings_from_nml(pam.nmlSet, nummu))
    fullspec = bool(pam.nmlSet.get("hydro_fullspec", False))
    sp = packing.species_from_df(pam.df.data, fullspec)
    cols = packing.profile_columns(pam.p, pam.df.nhydro)
    if fullspec:
        packing.fullspec_columns(cols, pam.df.dataFullSpec)
    nx, ny = int(pam.p["ngridx"]), int(pam.p["ngridy"])
    nout = int(cols["noutlevels"])
    N = nummu
    tb = np.full((nx * ny, nout, 2 * N, len(freqs), 2), -9999.0)
    em = np.full((nx * ny, 2, len(freqs), N), -9999.0)
    err_all = 0
    ang = None
    dbgs = []
    Lm, nf = int(cols["max_nlyrs"]), len(freqs)
    H = len(sp)
    # save_psd: bins of the moment-based distributions (-9999 for full spectra)
    # and per-bin backscattering cross sections
    psd_nbin = max(2, int(np.max(pam.df.data["nbin"]))) if pam.nmlSet.get("save_psd", False) and H else 0
    psd = {k: np.full((nx * ny, Lm, H, psd_nbin), -9999.0) for k in PSD_KEYS} if psd_nbin else None
    ze = np.full((nx * ny, Lm, nf), -9999.0)
    ath = np.zeros((nx * ny, Lm, nf))
    ata = np.zeros((nx * ny, Lm, nf))
    for c in range(nx * ny):
        err, t, e, a, d = run_column(st, sp, cols, c, freqs, debug or ("radar" if st.active else False),
                                     psd_nbin=psd_nbin)
        err_all = max(err_all, err)
        tb[c], em[c], ang = t, e, a
        if st.active:
            L = int(cols["nlyrs"][c])
            ze[c, :L], ath[c, :L], ata[c, :L] = d["ze"].T, d["att_hydro"].T, d["att_atmo"].T
        if psd is not None:
            L = int(cols["nlyrs"][c])
            for k in PSD_KEYS:
                psd[k][c, :L] = d[k]
        dbgs.append(d)
    r = dict(tb=tb.reshape(nx, ny, nout, 2 * N, len(freqs), 2),
             emissivity=em.reshape(nx, ny, 2, len(freqs), N), angles_deg=ang)
    if st.active:
        r["Ze"] = ze.reshape(nx, ny, Lm, nf, 1, 1)
        r["Att_hydro"] = ath.reshape(nx, ny, Lm, nf, 1)
        r["Att_atmo"] = ata.reshape(nx, ny, Lm, nf)
    if psd is not None:
        for k in PSD_KEYS:
            r[k] = psd[k].reshape(nx, ny, Lm, H, psd_nbin)
    if debug:
        r["debug"] = dbgs
    return r, err_all


def gas_r98(f, T, rhowv, p):
    k = ctypes.c_double()
    err = lib().orc_gas_r98(f, T, rhowv, p, ctypes.byref(k))
    return err, k.value


LIQ_MODS = {"TKC": 0, "Ell": 1, "Lie": 2, "Ray": 3, "Sto": 4}


def get_eps_water(liq_mod, s, T_c, f):
    """(errorstatus, eps) of get_eps_water (src/eps_water.f90:6-70)."""
    re, im = ctypes.c_double(), ctypes.c_double()
    err = lib().orc_get_eps_water(LIQ_MODS[liq_mod], s, T_c, f, ctypes.byref(re), ctypes.byref(im))
    return err, complex(re.value, im.value)


def gas_l93(f, press, vap, T):
    """MPM93 absorption in Np/m (pressures in Pa, T in K)."""
    return lib().orc_gas_l93(f, press, vap, T)


def eps_water_tkc(T_c, f):
    re, im = ctypes.c_double(), ctypes.c_double()
    lib().orc_eps_water_tkc(T_c, f, ctypes.byref(re), ctypes.byref(im))
    return complex(re.value, im.value)


def lobatto(n):
    mu, w = np.zeros(n), np.zeros(n)
    lib().orc_lobatto(n, _p(mu), _p(w))
    return mu, w


def minvert(A):
    A = np.asfortranarray(np.asarray(A, dtype=np.float64))
    out = np.zeros_like(A, order="F")
    err = lib().orc_minvert(A.shape[0], _p(A), _p(out))
    return err, out


# ---------------------------------------------------------------- T-matrix branch


def tmatrix_tmat(lam, mrr, mri, axi, as_ratio):
    """Single-precision T-matrix of one spheroid (tmatrix_amplq, quad solve):
    complex array [m = 0..nmax][block 11, 12, 21, 22][n1][n2], or None."""
    cap = 101 * 4 * 100 * 100
    re = np.zeros(cap, np.float32)
    im = np.zeros(cap, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    nmax = lib().orc_tmatrix_tmat(lam, mrr, mri, axi, as_ratio, cap, re.ctypes.data_as(fp), im.ctypes.data_as(fp))
    if nmax <= 0:
        return None
    n = (nmax + 1) * 4 * nmax * nmax
    return (re[:n] + 1j * im[:n].astype(np.complex64)).reshape(nmax + 1, 4, nmax, nmax)


def tmatrix_single(nummu, frequency, mrr, mri, axi, as_ratio, beta=0.0):
    """calc_single_tmatrix of one particle: dict of scatter_matrix
    (Fortran order (2, nummu, 2, nummu, 2)), extinct_matrix (2, 2, nummu),
    emis_vector (2, nummu), sback (2, 2); None on the reference's error."""
    scat = np.zeros(2 * nummu * 2 * nummu * 2)
    ext = np.zeros(4 * nummu)
    emis = np.zeros(2 * nummu)
    sb = np.zeros(4)
    r = lib().orc_tmatrix_single(nummu, frequency, mrr, mri, axi, as_ratio, beta, _p(scat), _p(ext), _p(emis),
                                 _p(sb))
    if r:
        return None
    return {"scatter_matrix": scat.reshape((2, nummu, 2, nummu, 2), order="F"),
            "extinct_matrix": ext.reshape((2, 2, nummu), order="F"),
            "emis_vector": emis.reshape((2, nummu), order="F"), "sback": sb.reshape((2, 2), order="F")}


def tmatrix_species(nummu, frequency, ref_re, ref_im, phase, dmax, del_d, ndens, density, as_ratio, canting):
    """calc_tmatrix of one species at one frequency over its bins (arrays of
    equal length); same keys as tmatrix_single plus back_spec per bin."""
    nb = len(dmax)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dmax, del_d, ndens, density, as_ratio, canting)]
    scat = np.zeros(2 * nummu * 2 * nummu * 2)
    ext = np.zeros(4 * nummu)
    emis = np.zeros(2 * nummu)
    back = np.zeros(nb)
    sb = np.zeros(4)
    r = lib().orc_tmatrix_species(nummu, frequency, ref_re, ref_im, phase, nb, *[_p(a) for a in arrs], _p(scat),
                                  _p(ext), _p(emis), _p(back), _p(sb))
    if r:
        return None
    return {"scatter_matrix": scat.reshape((2, nummu, 2, nummu, 2), order="F"),
            "extinct_matrix": ext.reshape((2, 2, nummu), order="F"),
            "emis_vector": emis.reshape((2, nummu), order="F"), "sback": sb.reshape((2, 2), order="F"),
            "back_spec": back}


def miecalc(x, mr, mi):
    """Mie coefficients (a_n, b_n) of the oracle's miecalc (index m = mr - i mi)."""
    ar, ai, br, bi = (np.zeros(10000) for _ in range(4))
    n = lib().orc_miecalc(x, mr, mi, 10000, _p(ar), _p(ai), _p(br), _p(bi))
    return (ar[:n] + 1j * ai[:n]), (br[:n] + 1j * bi[:n])


_twins = {}


def _twin_tmat(kind):
    """orc64_tmatrix_tmat (FP64 twin) or orcdd_tmatrix_tmat (double-double twin)."""
    if kind not in _twins:
        lib()
        name, prefix = {"f64": ("liboracle_tm64.so", "orc64"), "dd": ("liboracle_tmdd.so", "orcdd")}[kind]
        path = os.path.join(HERE, "_build", name)
        if not os.path.exists(path):
            build()
        fn = getattr(ctypes.CDLL(path), prefix + "_tmatrix_tmat")
        fp = ctypes.POINTER(ctypes.c_float)
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_double] * 5 + [ctypes.c_int, fp, fp]
        _twins[kind] = fn
    return _twins[kind]


def tmatrix_tmat64(lam, mrr, mri, axi, as_ratio, kind="f64"):
    """As tmatrix_tmat, from a twin of the solve: ``kind`` "f64" runs the same
    steps in double precision (the precision of the CUDA path), "dd" in
    double-double; for measuring how far each departs from REAL*16."""
    cap = 101 * 4 * 100 * 100
    re = np.zeros(cap, np.float32)
    im = np.zeros(cap, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    nmax = _twin_tmat(kind)(lam, mrr, mri, axi, as_ratio, cap, re.ctypes.data_as(fp), im.ctypes.data_as(fp))
    if nmax <= 0:
        return None
    n = (nmax + 1) * 4 * nmax * nmax
    return (re[:n] + 1j * im[:n].astype(np.complex64)).reshape(nmax + 1, 4, nmax, nmax)


def layer_start(N, zdiff, gas, planck0, planck1, scat, ext_k, emis_k, tm_ext=None, tm_emis=None):
    """The oracle's start of a scattering layer (doubling count, INITIAL_SOURCE4,
    INITIALIZE4): scat [4][2N][2N] row-major; returns (num_doubles, R, T
    [2][2N][2N] column-major, lin [2][2N], linfactor)."""
    n = 2 * N
    sc = np.ascontiguousarray(scat, dtype=np.float64)
    R = np.zeros(2 * n * n)
    T = np.zeros(2 * n * n)
    lin = np.zeros(2 * n)
    lf = ctypes.c_double(0.0)
    te = None if tm_ext is None else np.ascontiguousarray(tm_ext, dtype=np.float64)
    tv = None if tm_emis is None else np.ascontiguousarray(tm_emis, dtype=np.float64)
    nd = lib().orc_layer_start(N, zdiff, gas, planck0, planck1, _p(sc), ext_k, emis_k,
                               te.ctypes.data if te is not None else None,
                               tv.ctypes.data if tv is not None else None, _p(R), _p(T), _p(lin), ctypes.byref(lf))
    return nd, R, T, lin, lf.value
