"""Liquid water permittivity models (nmlSet['liq_mod'], src/eps_water.f90)
and the MPM93 gas model (nmlSet['gas_mod'] = 'L93', src/mpm93.f90).

The reference pins only TKC (tests/test_fortran_functions.py:23-33:
eps = 60.6084 + 32.9184j at 20 degC, 10 GHz, rtol 1e-3); it holds no
golden values for the other models, so their oracle restatements are
checked for physical consistency here (every model within 1.5 % of the
TKC pin at that point; MPM93 within 3 % of Rosenkranz-98 at the centres
of the 22, 60 and 183 GHz lines, where both are dominated by the same line
strengths) and the CUDA path is held to the oracle.
"""
import copy

import numpy as np
import pytest

from pamtra_b200 import packing
from pamtra_b200 import workloads as wl

MODELS = ["TKC", "Ell", "Lie", "Ray", "Sto"]


@pytest.mark.parametrize("liq_mod", MODELS)
def test_oracle_water_models_near_tkc_pin(oracle_mod, liq_mod):
    err, eps = oracle_mod.get_eps_water(liq_mod, 0.0, 20.0, 10.0)
    assert err == 0
    tol = 1e-3 if liq_mod == "TKC" else 1.5e-2
    np.testing.assert_allclose(eps.real, 60.6084, rtol=tol)
    np.testing.assert_allclose(eps.imag, 32.9184, rtol=tol)


def test_oracle_ray_range(oracle_mod):
    # 0.2 um .. 10 cm: table below 1 mm (f above 299.79 GHz), formula above
    assert oracle_mod.get_eps_water("Ray", 0.0, 10.0, 150.0)[0] == 0
    assert oracle_mod.get_eps_water("Ray", 0.0, 10.0, 350.0)[0] == 0
    assert oracle_mod.get_eps_water("Ray", 0.0, 10.0, 1.4e6)[0] == 0  # 0.214 um
    assert oracle_mod.get_eps_water("Ray", 0.0, 10.0, 1.6e6)[0] == 2  # below 0.2 um
    assert oracle_mod.get_eps_water("Ray", 0.0, 10.0, 2.0)[0] == 2  # above 10 cm


def _ray_table():
    import re
    from pathlib import Path
    text = (Path(__file__).resolve().parents[1] / "oracle" / "ray_table.inc").read_text()
    tabs = {}
    for name in ("ray_wl", "ray_rn", "ray_cn"):
        body = re.search(r"%s\[RAY_NUMWAT\] = \{(.*?)\};" % name, text, re.S).group(1)
        tabs[name] = np.array([float(v.rstrip("f")) for v in body.replace(",", " ").split()], dtype=np.float32)
    return tabs


def test_ray_table_shape():
    t = _ray_table()
    wl = t["ray_wl"].astype(np.float64)
    assert all(len(v) == 518 for v in t.values())
    assert wl[0] == np.float32(0.2) and wl[-1] == 1000.0 and np.all(np.diff(wl) > 0)
    # Hale and Querry: visible water n about 1.33, almost transparent
    vis = (wl > 0.4) & (wl < 0.7)
    assert np.all(np.abs(t["ray_rn"][vis] - 1.333) < 0.01) and np.all(t["ray_cn"][vis] < 1e-7)


def test_oracle_ray_table_interpolation(oracle_mod):
    """The table branch at and between table wavelengths: eps = (rn + i cn)^2
    of the linear interpolation in the interval ending at the first table
    wavelength >= wl (src/eps_water.f90:522-537), with the wavelength from
    the frequency as the reference forms it (single-precision constants)."""
    t = _ray_table()
    wl = t["ray_wl"].astype(np.float64)
    rn, cn = t["ray_rn"].astype(np.float64), t["ray_cn"].astype(np.float64)
    c = float(np.float32(1.e6) * np.float32(2.99792458e8))
    rng = np.random.default_rng(5)
    for f in list(rng.uniform(300.0, 1.4e6, 60)) + [c / (wl[100] * 1e9), c / (wl[-1] * 1e9)]:
        w = c / (f * 1e9)
        i2 = max(1, int(np.searchsorted(wl, w, side="left")))
        i1 = i2 - 1
        fac = (w - wl[i1]) / (wl[i2] - wl[i1])
        n = complex(rn[i1] + fac * (rn[i2] - rn[i1]), cn[i1] + fac * (cn[i2] - cn[i1]))
        err, eps = oracle_mod.get_eps_water("Ray", 0.0, 10.0, f)
        assert err == 0
        np.testing.assert_allclose([eps.real, eps.imag], [(n * n).real, (n * n).imag], rtol=1e-12, atol=1e-300)


def test_oracle_ray_continuity_at_1mm(oracle_mod):
    # the Downing-Williams value at 1000 um and Ray's formula just above agree
    # within a few percent at room temperature (the table has no temperature)
    fcut = float(np.float32(1.e6) * np.float32(2.99792458e8)) / 1000.0 / 1e9
    below = oracle_mod.get_eps_water("Ray", 0.0, 20.0, fcut * 1.0001)[1]
    above = oracle_mod.get_eps_water("Ray", 0.0, 20.0, fcut * 0.9999)[1]
    assert abs(np.sqrt(below) - np.sqrt(above)) / abs(np.sqrt(above)) < 0.05


def test_oracle_salinity_lowers_static_permittivity(oracle_mod):
    for m in ("Ell", "Sto"):
        e0 = oracle_mod.get_eps_water(m, 0.0, 15.0, 1.4)[1]
        e35 = oracle_mod.get_eps_water(m, 35.0, 15.0, 1.4)[1]
        assert e35.real < e0.real and e35.imag > e0.imag  # sea water: ionic conductivity


def test_oracle_mpm93_vs_r98(oracle_mod):
    for (T, p, e) in ((288.15, 101325.0, 1000.0), (250.0, 50000.0, 50.0), (300.0, 100000.0, 3000.0)):
        rv = e / (T * 461.5)
        for f in (22.235, 60.0, 183.31):
            np.testing.assert_allclose(oracle_mod.gas_l93(f, p, e, T), oracle_mod.gas_r98(f, T, rv, p)[1], rtol=3e-2)
        for f in (10.0, 31.4, 89.0, 150.0, 250.0):
            r = oracle_mod.gas_l93(f, p, e, T) / oracle_mod.gas_r98(f, T, rv, p)[1]
            assert 0.7 < r < 1.4, (f, r)


def test_settings_codes():
    pam = wl.c1_pam()
    for i, m in enumerate(MODELS):
        pam.nmlSet["liq_mod"] = m
        assert packing.settings_from_nml(pam.nmlSet).liq_mod == i
    pam.nmlSet["gas_mod"] = "L93"
    assert packing.settings_from_nml(pam.nmlSet).gas_mod == 1
    pam.nmlSet["liq_mod"] = "XYZ"
    with pytest.raises(ValueError):
        packing.settings_from_nml(pam.nmlSet)
    pam.nmlSet["liq_mod"] = "TKC"
    pam.nmlSet["gas_mod"] = "MPM"
    with pytest.raises(ValueError):
        packing.settings_from_nml(pam.nmlSet)


@pytest.mark.gpu
def test_model_kernels_match_oracle(oracle_mod, native):
    import torch
    rng = np.random.default_rng(8)
    n = 301
    dev = torch.device("cuda", 0)
    lib = native.load()
    s = rng.choice([0.0, 35.0], n)
    tc = rng.uniform(-30.0, 40.0, n)
    fr = np.concatenate([rng.uniform(3.5, 500.0, n - 40), 10 ** rng.uniform(2.7, 6.2, 40)])  # table branch too
    td = [torch.from_numpy(x).to(dev) for x in (s, tc, fr)]
    for i, m in enumerate(MODELS):
        er = torch.zeros(n, dtype=torch.float64, device=dev)
        ei = torch.zeros(n, dtype=torch.float64, device=dev)
        st = torch.zeros(n, dtype=torch.int32, device=dev)
        assert lib.pamtra_b200_get_eps_water(i, *[x.data_ptr() for x in td], er.data_ptr(), ei.data_ptr(),
                                             st.data_ptr(), n, None) == 0
        torch.cuda.synchronize()
        ref = [oracle_mod.get_eps_water(m, a, b, c) for a, b, c in zip(s, tc, fr)]
        ok = np.array([r[0] == 0 for r in ref])
        assert np.array_equal(st.cpu().numpy() != 0, ~ok), m
        e = np.array([r[1] for r in ref])
        np.testing.assert_allclose(er.cpu().numpy()[ok], e.real[ok], rtol=1e-12, err_msg=m)
        np.testing.assert_allclose(ei.cpu().numpy()[ok], e.imag[ok], rtol=1e-12, err_msg=m)
    f = rng.uniform(1.0, 400.0, n)
    T = rng.uniform(190.0, 310.0, n)
    p = rng.uniform(100.0, 1.1e5, n)
    e = rng.uniform(0.0, 0.05, n) * p
    tt = [torch.from_numpy(x).to(dev) for x in (f, p, e, T)]
    k = torch.zeros(n, dtype=torch.float64, device=dev)
    assert lib.pamtra_b200_gas_l93(*[x.data_ptr() for x in tt], k.data_ptr(), n, None) == 0
    torch.cuda.synchronize()
    ref = np.array([oracle_mod.gas_l93(*v) for v in zip(f, p, e, T)])
    np.testing.assert_allclose(k.cpu().numpy(), ref, rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("liq_mod,gas_mod", [("Ell", "R98"), ("Lie", "R98"), ("Ray", "R98"), ("Sto", "R98"),
                                             ("TKC", "L93")])
def test_models_column_matches_oracle(oracle_mod, native, liq_mod, gas_mod):
    pam = wl.c1_pam()
    pam.nmlSet["liq_mod"] = liq_mod
    pam.nmlSet["gas_mod"] = gas_mod
    ref, err = oracle_mod.run_pamtra(copy.deepcopy(pam), wl.C1_FREQS)
    assert err == 0
    pam.runPamtra(wl.C1_FREQS)
    assert pam.fortError == 0
    assert np.max(np.abs(pam.r["tb"] - ref["tb"])) < 1e-6
    base, _ = oracle_mod.run_pamtra(wl.c1_pam(), wl.C1_FREQS)
    assert np.max(np.abs(ref["tb"] - base["tb"])) > 1e-3  # the model is not a no-op


def test_ray_tables_agree():
    # the device copy (pamtra_b200/csrc/ray_table.cuh) and the oracle's
    # (oracle/ray_table.inc) come from one generator run: same literals
    import re
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    dev = (root / "pamtra_b200" / "csrc" / "ray_table.cuh").read_text()
    orc = (root / "oracle" / "ray_table.inc").read_text()
    for name in ("ray_wl", "ray_rn", "ray_cn"):
        vals = [re.search(r"%s\[RAY_NUMWAT\] = \{(.*?)\};" % name, t, re.S).group(1).split() for t in (dev, orc)]
        assert vals[0] == vals[1] and len(vals[0]) == 518, name
