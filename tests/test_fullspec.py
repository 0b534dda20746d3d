"""Full size spectra input (``nmlSet['hydro_fullspec']``,
src/hydrometeor_extinction.f90:122-151 of the reference).

CPU: the descriptor arrays have the reference's shapes
(tests/test_descriptor_file.py:105-114); the oracle given the bins that
the moment-based path builds for a species reproduces that path's
brightness temperatures; an empty spectrum is clear sky.
GPU: the CUDA path through the pyPamtra surface against the oracle, 1e-6 K.
"""
import copy
import warnings

import numpy as np
import pytest

from pamtra_b200 import core, importer
from pamtra_b200 import workloads as wl

TB_TOL = 1e-6  # K


def test_add_full_spectra_shapes():
    pam = wl.fullspec_pam(ncol=2, nlay=6)
    sh4 = pam._shape4D
    nb = pam.df.fs_nbin
    assert nb == 40
    for k in ("rho_ds", "d_ds", "n_ds", "mass_ds", "area_ds", "as_ratio", "canting", "fallvelocity",
              "rg_kappa_ds", "rg_beta_ds", "rg_gamma_ds", "rg_zeta_ds"):
        assert pam.df.dataFullSpec[k].shape == sh4 + (nb,)
    assert pam.df.dataFullSpec["d_bound_ds"].shape == sh4 + (nb + 1,)
    with pytest.raises(AssertionError):
        pam.df.addHydrometeor(("x",) + wl.ICE_FS[1:])


def _merged_grid(d1, d2, nw):
    """Bin edges of the non-adaptive size grid (src/make_dist.f90:90-130):
    a linear and a logarithmic grid of about nw / 2 points each, merged in
    ascending order."""
    nlin = nlog = int(nw / 2.0)
    if nlin + nlog == nw:
        nlin -= 1
    w = (d2 - d1) / (nlin + 1)
    lin = [d1 + w * i for i in range(1, nlin + 2)]
    w = (np.log(d2) - np.log(d1)) / (nlog + 1)
    lg = [np.exp(w * (i - 1) + np.log(d1)) for i in range(1, nlog + 2)]
    return np.array(sorted(lin + lg, key=float))


def _one_species_pam(fullspec):
    warnings.simplefilter("ignore")
    pam = core.pyPamtra()
    pam.df.addHydrometeor(wl.ICE_FS)
    pam = importer.createUsStandardProfile(pam, hgt_lev=[0.0, 1000.0, 2000.0, 3000.0])
    pam.nmlSet["hydro_adaptive_grid"] = False
    pam.nmlSet["conserve_mass_rescale_dsd"] = False
    pam.p["hydro_q"][:] = 0.002
    if fullspec:
        pam.nmlSet["hydro_fullspec"] = True
        pam.df.addFullSpectra()
    return pam


def test_oracle_fullspec_reproduces_moment_path(oracle_mod):
    """Exponential ice (N0 = 3e8, lambda = 3000, moment_in 0, 40 bins over
    100-1000 um, rho 200 kg/m3) through the moment-based size distribution,
    and the same bins handed over as a full spectrum: number per bin is the
    trapezoid of the distribution over the bin (src/make_dist.f90:250-290),
    mass pi/6 rho d^3."""
    freqs = [35.5, 89.0]
    ref, err = oracle_mod.run_pamtra(_one_species_pam(False), freqs)
    assert err == 0
    pam = _one_species_pam(True)
    nb = pam.df.fs_nbin
    edges = _merged_grid(wl.ICE_FS[15] + 1e-8, wl.ICE_FS[16], nb)
    f = 3e8 * np.exp(-3000.0 * edges)
    fs = pam.df.dataFullSpec
    fs["d_bound_ds"][:] = edges
    d = 0.5 * (edges[1:] + edges[:-1])
    fs["d_ds"][:] = d
    fs["n_ds"][:] = (f[:-1] + f[1:]) / 2.0 * np.diff(edges)
    fs["rho_ds"][:] = 200.0
    fs["mass_ds"][:] = np.pi / 6.0 * 200.0 * d ** 3
    got, err = oracle_mod.run_pamtra(pam, freqs)
    assert err == 0
    assert np.max(np.abs(got["tb"] - ref["tb"])) < 1e-6
    # and the spectrum is what is used: twice the particles, other TBs
    fs["n_ds"][:] *= 2.0
    got2, _ = oracle_mod.run_pamtra(pam, freqs)
    assert np.max(np.abs(got2["tb"] - ref["tb"])) > 1.0


def test_oracle_fullspec_empty_is_clear_sky(oracle_mod):
    freqs = [89.0]
    pam = _one_species_pam(True)  # n_ds all zero: no layer carries hydrometeors
    got, err = oracle_mod.run_pamtra(pam, freqs)
    assert err == 0
    clear = _one_species_pam(False)
    clear.p["hydro_q"][:] = 0.0
    clear.df.data["moment_in"] = 3
    ref, err = oracle_mod.run_pamtra(clear, freqs)
    assert err == 0
    assert np.max(np.abs(got["tb"] - ref["tb"])) < 1e-9


@pytest.mark.gpu
def test_fullspec_gpu_matches_oracle(oracle_mod, native):
    freqs = [23.8, 89.0, 150.0]
    pam = wl.fullspec_pam(ncol=6, nlay=30)
    ref, err = oracle_mod.run_pamtra(copy.deepcopy(pam), freqs)
    assert err == 0
    pam.runPamtra(freqs)
    assert pam.fortError == 0
    assert np.max(np.abs(pam.r["tb"] - ref["tb"])) < TB_TOL
    # the spectra are not a no-op
    assert np.ptp(pam.r["tb"][:, 0, 0, :, 2, 0]) > 1.0


@pytest.mark.gpu
def test_fullspec_gpu_disabled_species(oracle_mod, native):
    """A species with scat_name 'disabled' marks its layers as carrying
    hydrometeors but scatters nothing (src/scatProperties.f90:203)."""
    freqs = [89.0]
    pam = wl.fullspec_pam(ncol=3, nlay=20, seed=11)
    pam.df.data["scat_name"][1] = "disabled"
    ref, err = oracle_mod.run_pamtra(copy.deepcopy(pam), freqs)
    assert err == 0
    pam.runPamtra(freqs)
    assert pam.fortError == 0
    assert np.max(np.abs(pam.r["tb"] - ref["tb"])) < TB_TOL


def test_fullspec_packing_and_presence():
    from pamtra_b200 import libWrapper, packing
    pam = wl.fullspec_pam(ncol=3, nlay=8, seed=5)
    cols = packing.profile_columns(pam.p, pam.df.nhydro)
    packing.fullspec_columns(cols, pam.df.dataFullSpec)
    assert cols["fs_nbin"] == 40 and cols["fs_d"].shape == (3, 8, 2, 40)
    assert cols["fs_d_bound"].shape == (3, 8, 2, 41)
    # presence: layers where any species' spectrum sums above zero, or all with threshold <= 0
    nsum = pam.df.dataFullSpec["n_ds"].reshape(3, 8, 2, 40).sum(-1)
    assert libWrapper.present_bound(cols, pam.df.data) == int(np.sum(np.any(nsum > 0, axis=-1)))
    assert libWrapper.present_bound(cols, pam.df.data, hydro_threshold=0.0) == 3 * 8
    bad = dict(pam.df.dataFullSpec)
    del bad["mass_ds"]
    with pytest.raises(ValueError):
        packing.fullspec_columns(packing.profile_columns(pam.p, pam.df.nhydro), bad)
    bad = dict(pam.df.dataFullSpec, d_bound_ds=pam.df.dataFullSpec["d_ds"])
    with pytest.raises(ValueError):
        packing.fullspec_columns(packing.profile_columns(pam.p, pam.df.nhydro), bad)


def test_oracle_fullspec_psd_outputs(oracle_mod):
    """With full spectra the bins are not saved (the reference saves them in
    the moment-based branch only), the per-bin backscatter is."""
    pam = wl.fullspec_pam(ncol=1, nlay=6, seed=9)
    pam.nmlSet["save_psd"] = True
    r, err = oracle_mod.run_pamtra(pam, [89.0])
    assert err == 0
    assert np.all(r["psd_d"] == -9999)
    n = pam.df.dataFullSpec["n_ds"].reshape(r["psd_bscat"].shape)
    b = r["psd_bscat"]
    assert np.all(b[n > 0] > 0)
