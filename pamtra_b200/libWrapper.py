"""Native seam, replacing the reference's f2py seam
``PamtraFortranWrapper`` (python/pyPamtra/libWrapper.py:24-235).

Same signature and return value ``(results, pamError[, module])``; results
carry the passive keys of ``pyPamtra.r`` (``tb``, ``emissivity``,
``angles_deg``; with ``save_ssp`` also ``kextatmo``, ``scatter_matrix``,
``extinct_matrix``, ``emis_vector``); with ``active`` (radar_mode 'simple')
``Ze``, ``Att_hydro``, ``Att_atmo`` and ``radar_hgt``; with ``save_psd`` the
``psd_*`` bins and per-bin backscatter; the other active keys
filled with -9999 as the reference does for unallocated outputs
(libWrapper.py:214-223).
"""

import numpy as np

from . import __version__
from . import packing
from ._native import PREC_FP64, engine

missingNumber = -9999.0

PSD_KEYS = ("psd_d", "psd_deltad", "psd_n", "psd_mass", "psd_area", "psd_bscat")
ACTIVE_KEYS = ["Ze", "Att_hydro", "Att_atmo", "radar_hgt", "radar_moments", "radar_edges", "radar_slopes",
               "radar_quality", "radar_snr", "radar_spectra", "radar_vel", "psd_d", "psd_deltad", "psd_n",
               "psd_mass", "psd_area", "psd_bscat"]


def present_bound(cols, df_data, hydro_threshold=None):
    """Upper bound on the number of (column, layer) pairs that can carry
    hydrometeors (src/hydrometeor_extinction.f90:276-283 presence test; for
    full spectra the test of lines 142-148)."""
    if len(df_data) == 0:
        return 0
    L = cols["max_nlyrs"]
    valid = np.arange(L)[None, :] < cols["nlyrs"][:, None]
    if cols.get("fs_d") is not None:
        if hydro_threshold is not None and hydro_threshold <= 0:
            return int(np.sum(valid))
        nsum = cols["fs_n"].sum(axis=-1)  # (ncol, L, H)
        return int(np.sum(np.any(nsum > 0, axis=-1) & valid))
    if np.any(np.asarray(df_data["moment_in"]) == 0):
        return int(np.sum(cols["nlyrs"]))
    any_q = np.zeros(cols["hydro_q"].shape[:2], dtype=bool)
    for k in ("hydro_q", "hydro_n", "hydro_reff"):
        a = cols[k]
        any_q |= np.any((a != 0) | np.isnan(a), axis=-1)
    return int(np.sum(any_q & valid))


def host_inputs(cols, freqs):
    """Dict of contiguous host arrays for pamtra_b200_run_host."""
    arrs = dict(cols)
    arrs["freqs"] = np.ascontiguousarray(np.asarray(freqs, dtype=np.float64))
    arrs["max_nfreq"] = len(freqs)
    nh = cols["hydro_q"].shape[-1]
    arrs["nhydro"] = nh
    for k in ("hydro_q", "hydro_n", "hydro_reff"):
        arrs[k] = np.ascontiguousarray(cols[k].reshape(cols["ncol"], cols["max_nlyrs"], nh))
    return arrs


def PamtraFortranWrapper(sets, nmlSets, descriptorFile, descriptorFile4D, descriptorFileFS, profile,
                         returnModule=True, device=0, precision=PREC_FP64, nummu=16):
    """Run the passive forward model for every column of ``profile`` at
    ``sets['freqs']`` on the GPU (host buffers in, host arrays out)."""
    if descriptorFile4D:
        raise NotImplementedError("4D descriptor fields are not on this path")
    if not nmlSets.get("passive", True):
        raise NotImplementedError("passive=False: only the passive path is built")
    freqs = list(sets["freqs"])
    nf = len(freqs)
    st = packing.settings_from_nml(nmlSets, nummu)
    fullspec = bool(nmlSets.get("hydro_fullspec", False))
    sp = packing.species_from_df(descriptorFile, fullspec)
    nhydro = len(sp)
    cols = packing.profile_columns(profile, nhydro)
    if fullspec:
        # full spectra replace the moment-based size distributions
        # (libWrapper.py:191-202 of the reference)
        if not descriptorFileFS:
            raise ValueError("hydro_fullspec needs the arrays of descriptorFile.addFullSpectra()")
        packing.fullspec_columns(cols, descriptorFileFS)
    arrs = host_inputs(cols, freqs)
    ncol, L, nout = cols["ncol"], cols["max_nlyrs"], cols["noutlevels"]
    N = nummu
    out = dict(tb=np.zeros((ncol, nout, 2 * N, nf, 2)), emissivity=np.zeros((ncol, 2, nf, N)),
               angles_deg=np.zeros(2 * N), status=np.zeros((ncol, nf), dtype=np.int32))
    save_ssp = bool(nmlSets.get("save_ssp", False))
    if save_ssp:
        out["kextatmo"] = np.zeros((ncol, nf, L))
        out["kexttot"] = np.zeros((ncol, nf, L))
        out["salbedo"] = np.zeros((ncol, nf, L))
        out["scatter_matrix"] = np.zeros((ncol, nf, L, 4, 2 * N, 2 * N))
    if st.active:
        for k in ("ze", "att_hydro", "att_atmo"):
            out[k] = np.zeros((ncol, nf, L))
    # save_psd: bins of the moment-based size distributions, sized as
    # src/vars_output.f90:175-193 (max descriptor nbin, at least 2)
    psd_nbin = max(2, int(np.max(descriptorFile["nbin"]))) if nmlSets.get("save_psd", False) and nhydro else 0
    if psd_nbin:
        for k in PSD_KEYS:
            out[k] = np.zeros((ncol, L, nhydro, psd_nbin))
    mask = {8: 1, 16: 2, 32: 4}[N]
    eng = engine(device)
    c = eng.make_columns(arrs, sp, nmu_mask=mask, max_present=present_bound(cols, descriptorFile, st.hydro_threshold),
                         max_nummu=N)
    o = eng.make_outputs(out)
    eng.run_host(st, c, o, precision)

    nx, ny = int(profile["ngridx"]), int(profile["ngridy"])
    results = dict()
    results["tb"] = out["tb"].reshape(nx, ny, nout, 2 * N, nf, 2)
    results["emissivity"] = out["emissivity"].reshape(nx, ny, 2, nf, N)
    results["angles_deg"] = out["angles_deg"]
    results["status"] = out["status"].reshape(nx, ny, nf)
    for k in ACTIVE_KEYS:
        results[k] = -9999 if k == "radar_quality" else missingNumber
    if psd_nbin:
        for k in PSD_KEYS:
            results[k] = out[k].reshape(nx, ny, L, nhydro, psd_nbin)
        if str(list(sets.get("radar_pol", ["NN"]))[0]).strip() in ("HV", "VH"):
            # psd_bscat is taken for the first polarisation; Mie spheres have no
            # cross-polar backscatter (src/scatProperties.f90:746-756)
            b = results["psd_bscat"]
            results["psd_bscat"] = np.where(b == missingNumber, b, 0.0 * b)
    if st.active:
        # simple radar (src/radar_simulator.f90:161-176): Ze per polarisation;
        # Mie spheres give the same backscatter for NN/HH/VV and none for HV/VH
        # (src/scatProperties.f90:746-756)
        pols = list(sets.get("radar_pol", ["NN"]))
        ze = out["ze"].transpose(0, 2, 1)  # (ncol, L, nf)
        zp = np.stack([ze if p.strip() in ("NN", "HH", "VV") else np.full_like(ze, missingNumber) for p in pols],
                      axis=-1)
        results["Ze"] = zp.reshape(nx, ny, L, nf, len(pols), 1)
        results["Att_hydro"] = out["att_hydro"].transpose(0, 2, 1).reshape(nx, ny, L, nf, 1)
        results["Att_atmo"] = out["att_atmo"].transpose(0, 2, 1).reshape(nx, ny, L, nf)
        hgt = cols["hgt"].copy()
        lev = cols["hgt_lev"]
        mid = 0.5 * (lev[:, 1:] + lev[:, :-1])
        hgt = np.where(np.isnan(hgt), mid, hgt)
        valid = np.arange(L)[None, :] < cols["nlyrs"][:, None]
        results["radar_hgt"] = np.where(valid, hgt, missingNumber).reshape(nx, ny, L)
    if save_ssp:
        # the reference keeps the values of the last column and frequency computed
        # (src/run_rt.f90:140-146, loop order pyPamtraLib.f90:119-133)
        last = ncol - 1
        nl = int(cols["nlyrs"][last])
        results["kextatmo"] = out["kextatmo"][last, nf - 1, :nl].copy()
        sm = out["scatter_matrix"][last, nf - 1, :nl]  # [L][4][row][col]
        # (L, i2, j2, i1, j1, quadrant): row = i2 + 2*j2, col = i1 + 2*j1
        sm6 = sm.reshape(nl, 4, N, 2, N, 2).transpose(0, 3, 2, 5, 4, 1)
        results["scatter_matrix"] = np.ascontiguousarray(sm6)
        kt = out["kexttot"][last, nf - 1, :nl]
        sa = out["salbedo"][last, nf - 1, :nl]
        ext = np.zeros((nl, 2, 2, N, 2))
        emv = np.zeros((nl, 2, N, 2))
        has = np.any(sm.reshape(nl, -1) != 0, axis=1) | (kt > 0)
        for z in range(nl):
            if has[z]:
                ext[z, 0, 0, :, :] = kt[z]
                ext[z, 1, 1, :, :] = kt[z]
                emv[z, 0, :, :] = (1.0 - sa[z]) * kt[z]
        results["extinct_matrix"] = ext
        results["emis_vector"] = emv
        results["kexttot_all"] = out["kexttot"].reshape(nx, ny, nf, L)
        results["salbedo_all"] = out["salbedo"].reshape(nx, ny, nf, L)
        results["kextatmo_all"] = out["kextatmo"].reshape(nx, ny, nf, L)
    results["pamtraVersion"] = "pamtra_b200 " + __version__
    results["pamtraHash"] = ""
    stt = out["status"]
    pamError = 2 if np.any(stt & 2) else (1 if np.any(stt & 1) else 0)
    if returnModule:
        return results, pamError, eng
    return results, pamError
