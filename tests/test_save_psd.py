"""save_psd outputs (src/hydrometeor_extinction.f90:303-309,
src/scatProperties.f90:914-917, src/vars_output.f90:175-193 of the reference).

CPU: the oracle's bins follow the descriptor (contiguous bins; with a fixed
grid the edges of src/make_dist.f90; masses a d^b, areas alpha d^beta
capped at d^2); slots without particles stay -9999.  GPU: the facade's
psd_* arrays against the oracle's.
"""
import copy

import numpy as np
import pytest

from pamtra_b200 import workloads as wl
from test_fullspec import _merged_grid

KEYS = ("psd_d", "psd_deltad", "psd_n", "psd_mass", "psd_area", "psd_bscat")


def _golden_psd():
    pam = wl.golden_pam()
    pam.nmlSet["save_psd"] = True
    return pam


def test_oracle_psd_golden_bins(oracle_mod):
    pam = _golden_psd()
    r, err = oracle_mod.run_pamtra(pam, wl.GOLDEN_FREQS)
    assert err == 0
    nb = 30
    assert r["psd_d"].shape == (1, 1, 3, 2, nb)
    # rain in layer 1 only, snow in layer 2 only
    assert np.all(r["psd_d"][0, 0, 0] == -9999) and np.all(r["psd_d"][0, 0, 1, 1] == -9999)
    rain_d, snow_d = r["psd_d"][0, 0, 1, 0], r["psd_d"][0, 0, 2, 1]
    # rain: the adaptive grid (the default) places the bins; they are
    # contiguous: each centre lies half a width past the previous edge
    dd = r["psd_deltad"][0, 0, 1, 0]
    assert np.all(dd > 0) and np.all(np.diff(rain_d) > 0)
    np.testing.assert_allclose(rain_d[1:] - rain_d[:-1], (dd[1:] + dd[:-1]) / 2, rtol=1e-9)
    np.testing.assert_allclose(r["psd_mass"][0, 0, 1, 0], np.pi / 6 * 1000.0 * rain_d ** 3, rtol=1e-13)
    assert np.all(r["psd_area"][0, 0, 1, 0] == -99.0)  # no area-size relation for rain
    # snow: m = 0.038 d^2, area = 0.3971 d^1.88 (capped at d^2)
    np.testing.assert_allclose(r["psd_mass"][0, 0, 2, 1], 0.038 * snow_d ** 2, rtol=1e-13)
    np.testing.assert_allclose(r["psd_area"][0, 0, 2, 1], np.minimum(0.3971 * snow_d ** 1.88, snow_d ** 2),
                               rtol=1e-13)
    # per-particle backscatter at the last frequency: positive where there are particles
    b = r["psd_bscat"][0, 0, 1, 0]
    n = r["psd_n"][0, 0, 1, 0]
    assert np.all(b[n > 0] > 0) and np.all(np.isnan(b[n == 0]))


def test_oracle_psd_fixed_grid_and_mass(oracle_mod):
    """Non-adaptive grid: the bin edges are the merged linear/log grid over
    [d_1 + 1e-8, d_2]; bins past a species' count stay -9999."""
    pam = wl.c1_pam()
    pam.nmlSet["save_psd"] = True
    r, err = oracle_mod.run_pamtra(pam, wl.C1_FREQS)
    assert err == 0
    for h, row in enumerate((wl.CLOUD_C1, wl.RAIN_C1)):
        nb = row[9]
        edges = _merged_grid(row[15] + 1e-8, row[16], nb)
        d = r["psd_d"][0, 0, 10, h, :nb]
        np.testing.assert_allclose(d, (edges[1:] + edges[:-1]) * 0.5, rtol=1e-13)
        np.testing.assert_allclose(r["psd_deltad"][0, 0, 10, h, :nb], np.diff(edges), rtol=1e-10)
        if nb < r["psd_d"].shape[-1]:
            assert np.all(r["psd_d"][0, 0, 10, h, nb:] == -9999)
    assert np.all(r["psd_n"][0, 0, 5:26, 1] >= 0) and np.all(r["psd_d"][0, 0, 26:] == -9999)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["golden", "c1", "fullspec"])
def test_save_psd_gpu_matches_oracle(oracle_mod, native, case):
    if case == "golden":
        pam, freqs = _golden_psd(), wl.GOLDEN_FREQS
    elif case == "c1":
        pam, freqs = wl.c1_pam(), wl.C1_FREQS
    else:
        pam, freqs = wl.fullspec_pam(ncol=3, nlay=12), [89.0, 150.0]
    pam.nmlSet["save_psd"] = True
    ref, err = oracle_mod.run_pamtra(copy.deepcopy(pam), freqs)
    assert err == 0
    pam.runPamtra(freqs)
    assert pam.fortError == 0
    for k in KEYS:
        assert pam.r[k].shape == ref[k].shape, k
        np.testing.assert_allclose(pam.r[k], ref[k], rtol=1e-9 if k == "psd_bscat" else 1e-13, atol=0,
                                   equal_nan=True, err_msg=k)
    if case == "fullspec":
        assert np.all(pam.r["psd_d"] == -9999)
        assert np.any(np.isfinite(pam.r["psd_bscat"]) & (pam.r["psd_bscat"] > 0))
