"""pyPamtra-compatible host logic (CPU only)."""
import numpy as np
import pytest

import pamtra_b200 as pb
from pamtra_b200 import meteoSI, packing, libWrapper
from pamtra_b200.workloads import golden_pam, c2_pam, RAIN_GOLDEN, SNOW_GOLDEN


def test_us_standard():
    rho, p, T = meteoSI.usStandard(np.array([0.0, 11000.0]))
    assert T[0] == 288.15 and p[0] == 101325.0
    # 11 km geometric is just below the tropopause in geopotential height
    assert 216.65 < T[1] < 217.0


def test_create_profile_defaults():
    pam = golden_pam()
    p = pam.p
    assert p["ngridx"] == 1 and p["ngridy"] == 1 and p["max_nlyrs"] == 3
    np.testing.assert_allclose(p["hgt"][0, 0], [500.0, 1500.0, 2500.0])
    assert np.isnan(p["groundtemp"][0, 0])
    np.testing.assert_allclose(p["obs_height"][0, 0], [833000.0, 0.0])
    assert p["sfc_refl"][0, 0] in (b"S", "S")
    assert p["hydro_q"].shape == (1, 1, 3, 2)
    assert p["noutlevels"] == 2


def test_create_profile_requires_fields():
    pam = pb.pyPamtra()
    with pytest.raises(TypeError):
        pam.createProfile(hgt_lev=[0.0, 1.0, 2.0], temp_lev=[280.0, 279.0, 278.0])
    with pytest.raises(TypeError):
        pam.createProfile(hgt_lev=[0, 1, 2], temp_lev=[1, 1, 1], press_lev=[1, 1, 1], relhum_lev=[0, 0, 0], foo=1)


def test_check_data_limits():
    pam = golden_pam()
    pam.p["temp_lev"][0, 0, 0] = 400.0
    with pytest.raises(ValueError):
        pam._checkData()
    pam = golden_pam()
    pam.p["hydro_q"][0, 0, 0, 0] = 0.1
    with pytest.raises(ValueError):
        pam._checkData()


def test_descriptor_roundtrip(tmp_path):
    pam = pb.pyPamtra()
    pam.df.addHydrometeor(RAIN_GOLDEN)
    pam.df.addHydrometeor(SNOW_GOLDEN)
    f = tmp_path / "desc.txt"
    pam.df.writeFile(str(f))
    pam2 = pb.pyPamtra()
    pam2.df.readFile(str(f))
    assert pam2.df.nhydro == 2
    for name in ("liq_ice", "nbin", "dist_name", "p_3", "d_2", "scat_name"):
        assert list(pam2.df.data[name]) == list(pam.df.data[name])
    with pytest.raises(AssertionError):
        pam2.df.addHydrometeor(RAIN_GOLDEN)
    pam2.df.removeHydrometeor("rwc_q")
    assert pam2.df.nhydro == 1


def test_packing_codes():
    pam = golden_pam()
    sp = packing.species_from_df(pam.df.data)
    assert sp["dist"].tolist() == [packing.DIST_CODES["exp"], packing.DIST_CODES["exp_field_t"]]
    assert sp["liq_ice"].tolist() == [1, -1]
    st = packing.settings_from_nml(pam.nmlSet)
    assert st.emissivity == 0.6 and st.outpol_vh == 1 and st.nummu == 16
    assert packing.settings_from_nml(dict(pam.nmlSet, gas_mod="L93")).gas_mod == packing.GAS_MODS["L93"]
    assert packing.settings_from_nml(dict(pam.nmlSet, liq_mod="Ell")).liq_mod == packing.LIQ_MODS["Ell"]
    with pytest.raises(ValueError):
        packing.settings_from_nml(dict(pam.nmlSet, gas_mod="MPM"))


def test_present_bound_covers_hydrometeor_layers():
    pam = c2_pam(64)
    cols = packing.profile_columns(pam.p, 2)
    nb = libWrapper.present_bound(cols, pam.df.data)
    assert nb == 64 * 21


def test_species_struct_size():
    import ctypes
    assert ctypes.sizeof(packing.Species) == 16 + 12 * 8
    assert packing.SPECIES_DTYPE.itemsize == ctypes.sizeof(packing.Species)
