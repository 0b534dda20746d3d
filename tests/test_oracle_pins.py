"""The oracle against the reference's own known answers (CPU only)."""
import os

import numpy as np
import pytest

from pamtra_b200.workloads import GOLDEN_FREQS, golden_pam, c1_pam, C1_FREQS

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rain_snow_reference.npz")


def test_golden_tb_pinned(oracle_mod):
    # reference tests/test_regression.py:42-43 uses rtol 1e-5
    r, err = oracle_mod.run_pamtra(golden_pam(), GOLDEN_FREQS)
    assert err == 0
    ref = np.load(GOLDEN)["tb"]
    assert r["tb"].shape == ref.shape
    np.testing.assert_allclose(r["tb"], ref, rtol=1e-5)
    # the restatement reproduces the fixture far below the reference's tolerance
    assert np.max(np.abs(r["tb"] - ref) / np.abs(ref)) < 1e-7


def test_golden_sky_entries(oracle_mod):
    # TOA downwelling is the 2.73 K cosmic background (constants.f90 sky_temp)
    r, _ = oracle_mod.run_pamtra(golden_pam(), GOLDEN_FREQS)
    np.testing.assert_allclose(r["tb"][0, 0, 0, 16:, :, :], 2.73, rtol=1e-12)


def test_tkc_known_answer(oracle_mod):
    # reference tests/test_fortran_functions.py:23-33
    e = oracle_mod.eps_water_tkc(20.0, 10.0)
    np.testing.assert_allclose(e.real, 60.6084, rtol=1e-3)
    np.testing.assert_allclose(e.imag, 32.9184, rtol=1e-3)


@pytest.mark.parametrize("n", [8, 16, 32])
def test_lobatto(oracle_mod, n):
    mu, w = oracle_mod.lobatto(n)
    assert mu[-1] == 1.0
    assert np.all(np.diff(mu) > 0)
    np.testing.assert_allclose(w.sum(), 1.0, rtol=1e-13)
    # exact for polynomials up to degree 4n-3 on [-1,1] (even parts)
    np.testing.assert_allclose(np.sum(w * mu ** 2), 1.0 / 3.0, rtol=1e-13)


def test_minvert(oracle_mod):
    rng = np.random.default_rng(0)
    for n in (16, 32, 64):
        a = rng.normal(size=(n, n)) + 0.1 * np.eye(n)
        err, inv = oracle_mod.minvert(a)
        assert err == 0
        np.testing.assert_allclose(inv @ a, np.eye(n), atol=1e-10)
    # needs pivoting: zero leading diagonal
    a = np.array([[0.0, 1.0], [1.0, 0.0]])
    a = np.kron(np.eye(8), a)
    err, inv = oracle_mod.minvert(a)
    assert err == 0
    np.testing.assert_allclose(inv, np.linalg.inv(a), atol=1e-15)
    err, _ = oracle_mod.minvert(np.zeros((16, 16)))
    assert err != 0


def test_gas_range_errors(oracle_mod):
    assert oracle_mod.gas_r98(0.0, 280.0, 0.0, 1e5)[0] == 2
    assert oracle_mod.gas_r98(801.0, 280.0, 0.0, 1e5)[0] == 2
    assert oracle_mod.gas_r98(50.0, 99.0, 0.0, 1e5)[0] == 2
    assert oracle_mod.gas_r98(50.0, 280.0, 0.0, 1.3e5)[0] == 2


def test_gas_physics(oracle_mod):
    # O2 complex near 60 GHz is opaque; the 22.235 GHz line grows with vapour
    _, k60 = oracle_mod.gas_r98(60.0, 288.0, 0.0, 101325.0)
    _, k30 = oracle_mod.gas_r98(30.0, 288.0, 0.0, 101325.0)
    assert k60 > 100 * k30 > 0
    _, kd = oracle_mod.gas_r98(22.235, 288.0, 0.0, 101325.0)
    _, kw = oracle_mod.gas_r98(22.235, 288.0, 0.01, 101325.0)
    assert kw > 10 * kd


def test_blackbody_surface(oracle_mod):
    # no gas, no hydrometeors, emissivity 1: upwelling TOA TB = ground temperature
    pam = golden_pam()
    pam.p["hydro_q"][:] = 0.0
    pam.nmlSet["lgas_extinction"] = False
    pam.nmlSet["emissivity"] = 1.0
    r, err = oracle_mod.run_pamtra(pam, [30.0])
    assert err == 0
    np.testing.assert_allclose(r["tb"][0, 0, 0, :16, 0, :], 288.15, rtol=1e-9)
    # emissivity 0: the surface mirrors the sky
    pam.nmlSet["emissivity"] = 0.0
    r, err = oracle_mod.run_pamtra(pam, [30.0])
    np.testing.assert_allclose(r["tb"][0, 0, 0, :16, 0, :], 2.73, rtol=1e-9)


def test_c1_oracle_runs(oracle_mod):
    r, err = oracle_mod.run_pamtra(c1_pam(), C1_FREQS, debug=True)
    assert err == 0
    tb = r["tb"]
    assert np.all((tb > 2.7) & (tb < 330))
    d = r["debug"][0]
    assert list(np.nonzero(d["present"])[0]) == list(range(5, 26))
    assert np.all(d["num_doubles"][:, 5:26] > 0)


def test_oracle_simple_radar_matches_golden(oracle_mod):
    # the reference's golden scenario runs the active 'simple' radar beside
    # the passive path (nmlSet active=True, radar_mode='simple'); its Ze and
    # Att_hydro pin the oracle's restatement of radar_simulator at the
    # reference test's tolerance (tests/test_regression.py:34-39)
    from pamtra_b200.workloads import golden_pam, GOLDEN_FREQS
    pam = golden_pam()
    assert pam.nmlSet["active"] and pam.nmlSet["radar_mode"] == "simple"
    r, err = oracle_mod.run_pamtra(pam, GOLDEN_FREQS)
    assert err == 0
    gold = np.load(GOLDEN)
    np.testing.assert_allclose(r["Ze"], gold["Ze"], rtol=1e-5)
    np.testing.assert_allclose(r["Att_hydro"], gold["Att_hydro"], rtol=1e-5)
    assert (r["Ze"][0, 0, 1:3] > -9999).all() and np.all(r["Ze"][0, 0, 0] == -9999)
