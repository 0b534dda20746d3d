"""T-matrix branch (scat_name 'tmatrix', src/tmatrix.f90 + src/tmatrix_amplq.lp.f).

CPU tests pin the quad-precision oracle by the sphere limit: for aspect ratio
1 the T-matrix is diagonal with T11 = -b_n and T22 = -a_n (the Mie
coefficients of the oracle's miecalc, itself pinned to the reference's golden
fixture), and the extinction and backscattering cross-sections follow.  The
reference stores T in single precision (REAL*4 common /TMAT/), so the pins
hold to float rounding (a few 1e-7 relative).

GPU tests compare ``pamtra_b200_tmatrix`` (FP64 solve, single-precision T as
the reference stores it) with the oracle (REAL*16 solve like the reference)
bin by bin and summed, over spheres, oblate and prolate spheroids, soft ice
spheroids, canted particles (the full AMPL path), empty and invalid bins and
NUMMU 8/16/32.  Tolerance: 2e-6 of each output array's largest magnitude
(T rounded to single precision by both sides; FP64 vs REAL*16 solve).
"""
import numpy as np
import pytest

C = 299792458.0


def _mie_cross(oracle_mod, f, mr, mi, axi):
    k = 2 * np.pi * f / C
    a, b = oracle_mod.miecalc(k * axi, mr, -mi)
    n = np.arange(1, len(a) + 1)
    cext = 2 * np.pi / k ** 2 * np.sum((2 * n + 1) * np.real(a + b))
    cback = np.pi / k ** 2 * abs(np.sum((2 * n + 1) * (-1.0) ** n * (a - b))) ** 2
    return a, b, cext, cback


SPHERES = [(89e9, 1.78, 0.003, 0.5e-3), (150e9, 6.5, 2.8, 1.0e-3), (35e9, 1.3, 0.001, 3e-3)]


@pytest.mark.parametrize("case", SPHERES)
def test_oracle_sphere_tmatrix_is_mie(oracle_mod, case):
    f, mr, mi, axi = case
    T = oracle_mod.tmatrix_tmat(C / f, mr, mi, axi, 1.0)
    a, b, _, _ = _mie_cross(oracle_mod, f, mr, mi, axi)
    nmax = T.shape[2]
    n = min(nmax, len(a))
    for m in range(0, 3):
        for blk, coef in ((0, b), (3, a)):
            d = np.array([T[m, blk, k, k] for k in range(max(m - 1, 0), n)])
            ref = -coef[max(m - 1, 0):n]
            assert np.max(np.abs(d - ref)) <= 3e-7 * np.max(np.abs(coef)), (m, blk)
        # the sphere does not couple orders or the two polarisation blocks
        off = T[m, 0] - np.diag(np.diag(T[m, 0]))
        assert np.max(np.abs(off)) < 1e-20
        assert np.max(np.abs(T[m, 1])) < 1e-20 and np.max(np.abs(T[m, 2])) < 1e-20


@pytest.mark.parametrize("case", SPHERES)
def test_oracle_sphere_cross_sections(oracle_mod, case):
    f, mr, mi, axi = case
    r = oracle_mod.tmatrix_single(16, f, mr, mi, axi, 1.0)
    _, _, cext, cback = _mie_cross(oracle_mod, f, mr, mi, axi)
    ext = r["extinct_matrix"]
    # forward extinction is the same at every incidence and unpolarised
    assert np.allclose(ext[0, 0, :], cext, rtol=5e-7, atol=0)
    assert np.max(np.abs(ext[0, 1, :])) < 1e-12 * cext
    assert abs(4 * np.pi * r["sback"][0, 0] / cback - 1) < 2e-6
    # a sphere does not depolarise the backscattered wave
    assert abs(r["sback"][0, 1]) < 1e-12 * r["sback"][0, 0]


def test_oracle_spheroid_symmetries(oracle_mod):
    """Upright spheroid: the extinction matrix is symmetric, its 11 element
    at nadir incidence equals the sphere-like unpolarised one, and an oblate
    particle extinguishes horizontal polarisation more at grazing angles."""
    r = oracle_mod.tmatrix_single(16, 89e9, 1.78, 0.003, 0.8e-3, 0.6)
    ext = r["extinct_matrix"]
    assert np.allclose(ext[0, 1, :], ext[1, 0, :], rtol=0, atol=0)
    assert np.allclose(ext[0, 0, :], ext[1, 1, :], rtol=0, atol=0)
    # at nadir (mu = 1) the polarisation term vanishes for an upright particle
    assert abs(ext[0, 1, -1]) < 1e-6 * ext[0, 0, -1]
    assert abs(ext[0, 1, 0]) > 1e-3 * ext[0, 0, 0]


# ---------------------------------------------------------------- GPU parity

def _run_gpu(items, nbins, nummu):
    from pamtra_b200 import tmatrix as ptm
    arr = {k: np.array([it[k] for it in items], dtype=np.float64).reshape(len(items), nbins)
           for k in ("dmax", "del_d", "ndens", "density", "as_ratio", "canting")}
    return ptm.calc_tmatrix_batch(np.array([it["freq"] for it in items]), np.array([it["ref"] for it in items]),
                                  np.array([it["phase"] for it in items], dtype=np.int32), arr["dmax"], arr["del_d"],
                                  arr["ndens"], arr["density"], arr["as_ratio"], arr["canting"], nummu=nummu)


def _oracle_item(oracle_mod, it, nummu):
    return oracle_mod.tmatrix_species(nummu, it["freq"], it["ref"].real, it["ref"].imag, it["phase"],
                                      it["dmax"], it["del_d"], it["ndens"], it["density"], it["as_ratio"],
                                      it["canting"])


def _item(freq, ref, phase, dmax, ndens, density, as_ratio, canting, del_d=1e-4):
    nb = len(dmax)
    return {"freq": freq, "ref": complex(ref), "phase": phase, "dmax": list(dmax), "del_d": [del_d] * nb,
            "ndens": list(ndens), "density": [density] * nb if np.isscalar(density) else list(density),
            "as_ratio": [as_ratio] * nb if np.isscalar(as_ratio) else list(as_ratio),
            "canting": [canting] * nb if np.isscalar(canting) else list(canting)}


def _compare(out, refs, nummu, tol=2e-6):
    for i, ref in enumerate(refs):
        assert ref is not None
        assert int(out["status"][i]) == 0
        g = {"scatter_matrix": out["scatter_matrix"][i].reshape((2, nummu, 2, nummu, 2), order="F"),
             "extinct_matrix": out["extinct_matrix"][i].reshape((2, 2, nummu), order="F"),
             "emis_vector": out["emis_vector"][i].reshape((2, nummu), order="F"),
             "sback": out["sback"][i].reshape((2, 2), order="F"), "back_spec": out["back_spec"][i]}
        for k in g:
            scale = np.max(np.abs(ref[k]))
            err = np.max(np.abs(g[k] - ref[k]))
            assert err <= tol * scale + 1e-300, (i, k, err, scale)


@pytest.mark.gpu
def test_gpu_tmatrix_matches_oracle(oracle_mod):
    items = [
        # rain: oblate drops
        _item(89e9, 1.78 - 0.003j, 1, [0.4e-3, 1.2e-3, 2.0e-3], [1e7, 5e6, 0.0], 1000.0, [0.95, 0.8, 0.6], 0.0),
        # water sphere, strongly absorbing
        _item(150e9, 6.5 - 2.8j, 1, [0.6e-3, 1.6e-3], [2e6, 1e6], 1000.0, 1.0, 0.0),
        # soft ice spheroids (mixed with air), prolate and oblate
        _item(35e9, 1.78 - 0.0005j, -1, [1e-3, 3e-3, 5e-3], [1e6, 3e5, 1e5], [600.0, 300.0, 150.0],
              [0.6, 1.5, 0.7], 0.0),
    ]
    # items have different bin counts: pad to three bins with empty ones
    for it in items:
        while len(it["dmax"]) < 3:
            for k in ("dmax", "del_d", "density", "as_ratio", "canting"):
                it[k].append(it[k][-1])
            it["ndens"].append(0.0)
    out = _run_gpu(items, 3, 16)
    refs = [_oracle_item(oracle_mod, it, 16) for it in items]
    _compare(out, refs, 16)
    assert int(out["nmax"][0, 2]) == 0  # empty bin skipped


@pytest.mark.gpu
def test_gpu_tmatrix_canted_full_amplitude_path(oracle_mod):
    items = [_item(89e9, 1.78 - 0.003j, 1, [1.0e-3, 1.8e-3], [1e6, 5e5], 1000.0, [0.8, 0.65], [20.0, 45.0])]
    out = _run_gpu(items, 2, 16)
    _compare(out, [_oracle_item(oracle_mod, it, 16) for it in items], 16)


@pytest.mark.gpu
@pytest.mark.parametrize("nummu", [8, 32])
def test_gpu_tmatrix_nummu(oracle_mod, nummu):
    items = [_item(50e9, 1.78 - 0.001j, -1, [2e-3, 4e-3], [1e6, 2e5], 400.0, 0.6, 0.0)]
    out = _run_gpu(items, 2, nummu)
    _compare(out, [_oracle_item(oracle_mod, it, nummu) for it in items], nummu)


@pytest.mark.gpu
def test_gpu_tmatrix_sphere_limit_is_mie(oracle_mod):
    f, mr, mi, axi = SPHERES[0]
    it = _item(f, complex(mr, -mi), 1, [2 * axi], [1.0], 1000.0, 1.0, 0.0, del_d=1.0)
    out = _run_gpu([it], 1, 16)
    _, _, cext, cback = _mie_cross(oracle_mod, f, mr, mi, axi)
    ext = out["extinct_matrix"][0].reshape((2, 2, 16), order="F")
    assert np.allclose(ext[0, 0, :], cext, rtol=5e-7, atol=0)
    assert abs(out["back_spec"][0, 0] / cback - 1) < 2e-6


@pytest.mark.gpu
def test_gpu_tmatrix_invalid_bins_report_status():
    from pamtra_b200 import _native
    items = [_item(89e9, 1.78 - 0.003j, 1, [1e-3, 1e-3], [1e6, 1e6], 1000.0, [0.8, -1.0], 0.0),
             _item(89e9, 1.78 - 0.003j, 1, [1e-3, 1e-3], [1e6, 1e6], 1000.0, 0.8, 0.0)]
    out = _run_gpu(items, 2, 16)
    assert int(out["status"][0]) == (2 | _native.ST_RANGE)
    assert int(out["status"][1]) == 0
    assert np.all(np.isfinite(out["scatter_matrix"]))


@pytest.mark.gpu
def test_gpu_tmatrix_device_inputs_match_host(oracle_mod):
    import torch
    from pamtra_b200 import tmatrix as ptm
    items = [_item(89e9, 1.78 - 0.003j, 1, [0.8e-3, 1.5e-3], [2e6, 1e6], 1000.0, [0.9, 0.7], 0.0)]
    host = _run_gpu(items, 2, 16)
    dev = torch.device("cuda", 0)
    t = {k: torch.tensor([it[k] for it in items], dtype=torch.float64, device=dev)
         for k in ("dmax", "del_d", "ndens", "density", "as_ratio", "canting")}
    out = ptm.calc_tmatrix_batch(torch.tensor([89e9], device=dev, dtype=torch.float64),
                                 torch.tensor([1.78 - 0.003j], dtype=torch.complex128, device=dev),
                                 torch.tensor([1], device=dev),
                                 t["dmax"], t["del_d"], t["ndens"], t["density"], t["as_ratio"], t["canting"])
    torch.cuda.synchronize()
    for k in ("scatter_matrix", "extinct_matrix", "emis_vector", "sback", "back_spec"):
        assert np.array_equal(out[k].cpu().numpy(), host[k])


def test_oracle_nonabsorbing_spheroid_conserves_energy(oracle_mod):
    """mri = 0: extinction equals the scattering integrated over the sphere,
    so the emission vector vanishes up to the quadrature and the
    single-precision T."""
    r = oracle_mod.tmatrix_single(16, 89e9, 1.78, 0.0, 0.8e-3, 0.6)
    assert np.max(np.abs(r["emis_vector"][0])) < 5e-6 * np.max(r["extinct_matrix"][0, 0])


def test_oracle_upside_down_spheroid_is_the_same_particle(oracle_mod):
    """Canting 180 deg turns the spheroid over: the same particle, reached
    through the rotated geometry of AMPL."""
    r1 = oracle_mod.tmatrix_single(16, 89e9, 1.78, 0.003, 0.8e-3, 0.6, beta=0.0)
    r2 = oracle_mod.tmatrix_single(16, 89e9, 1.78, 0.003, 0.8e-3, 0.6, beta=180.0)
    for k in ("scatter_matrix", "extinct_matrix", "emis_vector", "sback"):
        assert np.max(np.abs(r1[k] - r2[k])) <= 1e-12 * np.max(np.abs(r1[k])), k


def test_oracle_reciprocity_of_the_azimuth_averaged_phase_function(oracle_mod):
    """Z11 averaged over azimuth is symmetric in the incident and scattered
    polar angles (reciprocity), to the single-precision T."""
    S = oracle_mod.tmatrix_single(16, 89e9, 1.78, 0.003, 0.8e-3, 0.6)["scatter_matrix"]
    for kk in (0, 1):
        z = S[0, :, 0, :, kk]
        assert np.max(np.abs(z - z.T)) <= 1e-5 * np.max(np.abs(z))


@pytest.mark.gpu
def test_gpu_upright_and_overturned_paths_agree():
    """Canting 0 takes the separable amplitude sums, canting 180 the full AMPL
    evaluation per azimuth; both describe the same particle."""
    a = _run_gpu([_item(89e9, 1.78 - 0.003j, 1, [0.8e-3, 1.6e-3], [2e6, 1e6], 1000.0, 0.6, 0.0)], 2, 16)
    b = _run_gpu([_item(89e9, 1.78 - 0.003j, 1, [0.8e-3, 1.6e-3], [2e6, 1e6], 1000.0, 0.6, 180.0)], 2, 16)
    for k in ("scatter_matrix", "extinct_matrix", "emis_vector", "sback", "back_spec"):
        assert np.max(np.abs(a[k] - b[k])) <= 5e-6 * np.max(np.abs(a[k])), k


# ---------------------------------------------------------------- forward run (oracle)

def _golden_column():
    from pamtra_b200 import packing
    from pamtra_b200 import workloads as wl
    pam = wl.golden_pam()
    return (packing.settings_from_nml(pam.nmlSet, 16), packing.species_from_df(pam.df.data, False),
            packing.profile_columns(pam.p, pam.df.nhydro))


def test_oracle_forward_tmatrix_entry_keeps_mie_columns(oracle_mod):
    st, sp, cols = _golden_column()
    st = oracle_mod.settings(st)
    e0, tb0, _, _, _ = oracle_mod.run_column(st, sp, cols, 0, [35.5])
    e1, tb1, _, _, _ = oracle_mod.run_column(st, sp, cols, 0, [35.5], scat_code=[0] * len(sp))
    assert e0 == 0 and e1 == 0
    assert np.array_equal(tb0, tb1)


def test_oracle_forward_tmatrix_spheres_reproduce_mie(oracle_mod):
    """Both species as T-matrix spheres (aspect ratio 1): the layer matrices
    come from the amplitude sums instead of scatcnv's Legendre series, and the
    brightness temperatures agree with the Mie run."""
    st, sp, cols = _golden_column()
    st = oracle_mod.settings(st)
    e0, tb0, _, _, _ = oracle_mod.run_column(st, sp, cols, 0, [35.5])
    sp2 = sp.copy()
    sp2["as_ratio"] = 1.0
    e2, tb2, _, _, _ = oracle_mod.run_column(st, sp2, cols, 0, [35.5], scat_code=[1] * len(sp))
    assert e0 == 0 and e2 == 0
    assert np.max(np.abs(tb2 - tb0)) < 1e-4


def test_oracle_forward_oblate_spheroids_polarise(oracle_mod):
    """Oblate rain and snow: CHECK_NORM4 holds with the T-matrix matrices,
    and the upwelling radiation is polarised well beyond the Mie run's."""
    st, sp, cols = _golden_column()
    st = oracle_mod.settings(st)
    e0, tb0, _, _, _ = oracle_mod.run_column(st, sp, cols, 0, [89.0])
    sp2 = sp.copy()
    sp2["as_ratio"] = [0.7, 0.6]
    e2, tb2, _, _, _ = oracle_mod.run_column(st, sp2, cols, 0, [89.0], scat_code=[1, 1])
    assert e0 == 0 and e2 == 0
    assert np.all(np.isfinite(tb2))
    pol_tm = np.max(np.abs(tb2[-1, :16, 0, 0] - tb2[-1, :16, 0, 1]))
    pol_mie = np.max(np.abs(tb0[-1, :16, 0, 0] - tb0[-1, :16, 0, 1]))
    assert pol_tm > 1.0 and pol_tm > 3 * pol_mie


def test_tmatrix_species_in_run_pamtra_points_to_calc_tmatrix():
    from pamtra_b200 import packing
    from pamtra_b200 import workloads as wl
    pam = wl.golden_pam()
    data = pam.df.data.copy()
    data["scat_name"][0] = "tmatrix"
    with pytest.raises(NotImplementedError, match="calc_tmatrix"):
        packing.species_from_df(data, False)


@pytest.mark.parametrize("case", [
    # (size parameter, aspect ratio, index, bound on the T difference, inside the FP64 envelope)
    (10.0, 0.5, (1.78, 0.003), 1e-6, True),     # ice / snow: FP64 holds to x = 14 (2e-7)
    (10.0, 2.0, (1.78, 0.003), 1e-6, True),
    (3.0, 0.7, (5.5, 2.9), 1e-6, True),         # liquid water: small drops
    (6.0, 0.5, (5.5, 2.9), 1e-4, False),        # large, strongly oblate drops: FP64 loses digits
])
def test_fp64_solve_envelope(oracle_mod, case):
    """The CUDA path solves the EBCM system in FP64, the reference in REAL*16.
    The double-precision twin of the oracle's solve (the same steps) against
    the REAL*16 one marks where FP64 suffices: everywhere for ice and snow
    indices, for liquid water only up to moderate size and asphericity."""
    x, asr, (mr, mi), bound, inside = case
    lam = C / 89e9
    axi = x * lam / (2 * np.pi)
    tq = oracle_mod.tmatrix_tmat(lam, mr, mi, axi, asr)
    td = oracle_mod.tmatrix_tmat64(lam, mr, mi, axi, asr)
    assert tq is not None and td is not None and tq.shape == td.shape
    d = np.max(np.abs(tq - td)) / np.max(np.abs(tq))
    if inside:
        assert d <= bound, d
    else:
        assert d > bound, d


@pytest.mark.parametrize("x, asr", [(6.0, 0.5), (10.0, 0.7)])
def test_double_double_solve_reproduces_real16(oracle_mod, x, asr):
    """Where FP64 fails (large aspherical water drops), the same steps in
    double-double arithmetic give the REAL*16 single-precision T-matrix."""
    lam = C / 89e9
    axi = x * lam / (2 * np.pi)
    tq = oracle_mod.tmatrix_tmat(lam, 5.5, 2.9, axi, asr)
    tdd = oracle_mod.tmatrix_tmat64(lam, 5.5, 2.9, axi, asr, kind="dd")
    td = oracle_mod.tmatrix_tmat64(lam, 5.5, 2.9, axi, asr, kind="f64")
    assert tq is not None and tdd is not None and tq.shape == tdd.shape
    scale = np.max(np.abs(tq))
    assert np.max(np.abs(tdd - tq)) <= 1e-6 * scale
    assert td is None or td.shape != tq.shape or np.max(np.abs(td - tq)) > 1e-4 * scale


def test_tmatrix_entry_rejects_missing_context(native):
    """The C-ABI entry validates its arguments before touching a device."""
    import ctypes
    lib = native.load()
    ti, to = native.TmatrixIn(), native.TmatrixOut()
    ti.n_items, ti.nbins, ti.nummu = 1, 1, 16
    assert lib.pamtra_b200_tmatrix(None, ctypes.byref(ti), ctypes.byref(to), None) == 2


def test_back_hydro_polarisations(oracle_mod):
    """back_hydro per radar polarisation from a species' Sback (recorded for
    vertical incidence from below, as the reference records it): a sphere
    and an upright spheroid (seen along its axis) backscatter HH = VV = NN;
    a spheroid tilted by 60 deg gives positive differential reflectivity;
    with the tilt in the plane of the polarisation basis no cross-polar
    power appears."""
    from pamtra_b200.tmatrix import back_hydro
    sph = oracle_mod.tmatrix_single(16, 9.6e9, 8.9, 1.5, 1.5e-3, 1.0)["sback"]
    nn = back_hydro(sph, "NN")
    assert abs(back_hydro(sph, "HH") / nn - 1) < 1e-12 and abs(back_hydro(sph, "VV") / nn - 1) < 1e-12
    assert abs(back_hydro(sph, "HV")) < 1e-12 * nn and abs(back_hydro(sph, "VH")) < 1e-12 * nn
    up = oracle_mod.tmatrix_single(16, 9.6e9, 8.9, 1.5, 1.5e-3, 0.6)["sback"]
    assert abs(back_hydro(up, "HH") / back_hydro(up, "VV") - 1) < 1e-12
    obl = oracle_mod.tmatrix_single(16, 9.6e9, 8.9, 1.5, 1.5e-3, 0.6, beta=60.0)["sback"]
    zdr = 10 * np.log10(back_hydro(obl, "HH") / back_hydro(obl, "VV"))
    assert 2.0 < zdr < 10.0, zdr
    assert abs(back_hydro(obl, "HV")) < 1e-10 * back_hydro(obl, "HH")
    # the flat C-ABI order is the Fortran order of Sback(2, 2)
    assert back_hydro(np.asarray(obl).ravel(order="F"), "HH") == back_hydro(obl, "HH")
    with pytest.raises(ValueError):
        back_hydro(obl, "XX")


def test_oracle_fullspec_tmatrix_matches_moment_path(oracle_mod):
    """A T-matrix ice species through the moment-based bins, and the same
    bins handed over as a full spectrum whose per-bin aspect ratio is the
    species' (hydrofs_as_ratio, src/scatProperties.f90:257-265): the same
    brightness temperatures."""
    import test_fullspec as tf
    from pamtra_b200 import packing
    freqs = [89.0]
    pam0 = tf._one_species_pam(False)
    st = oracle_mod.settings(packing.settings_from_nml(pam0.nmlSet, 16))
    sp0 = packing.species_from_df(pam0.df.data, False)
    sp0["as_ratio"] = 0.6
    cols0 = packing.profile_columns(pam0.p, pam0.df.nhydro)
    e0, tb0, _, _, _ = oracle_mod.run_column(st, sp0, cols0, 0, freqs, scat_code=[1])
    pam = tf._one_species_pam(True)
    nb = pam.df.fs_nbin
    edges = tf._merged_grid(tf.wl.ICE_FS[15] + 1e-8, tf.wl.ICE_FS[16], nb)
    f = 3e8 * np.exp(-3000.0 * edges)
    fs = pam.df.dataFullSpec
    fs["d_bound_ds"][:] = edges
    d = 0.5 * (edges[1:] + edges[:-1])
    fs["d_ds"][:] = d
    fs["n_ds"][:] = (f[:-1] + f[1:]) / 2.0 * np.diff(edges)
    fs["rho_ds"][:] = 200.0
    fs["mass_ds"][:] = np.pi / 6.0 * 200.0 * d ** 3
    sp = packing.species_from_df(pam.df.data, True)
    cols = packing.profile_columns(pam.p, pam.df.nhydro)
    packing.fullspec_columns(cols, fs)
    L = int(cols["nlyrs"][0])
    e1, tb1, _, _, _ = oracle_mod.run_column(st, sp, cols, 0, freqs, scat_code=[1],
                                             fs_as_ratio=np.full((L, 1, nb), 0.6))
    assert e0 == 0 and e1 == 0
    assert np.max(np.abs(tb1 - tb0)) < 1e-6
    # without per-bin aspect ratios a full-spectrum T-matrix species is refused
    e2, _, _, _, _ = oracle_mod.run_column(st, sp, cols, 0, freqs, scat_code=[1])
    assert e2 == 2


def test_fp64_envelope_marks_large_aspherical_drops():
    from pamtra_b200.tmatrix import fp64_envelope
    # 89 GHz: x = 2 pi axi / lambda with lambda = 3.37 mm
    freq = np.array([89e9, 89e9, 89e9])
    ref = np.array([5.5 - 2.9j, 5.5 - 2.9j, 1.78 - 0.003j])
    phase = np.array([1, 1, -1])
    dmax = np.array([[1e-3, 6e-3], [1e-3, 6e-3], [1e-3, 2e-2]])
    asr = np.array([[0.6, 0.6], [1.0, 1.0], [0.6, 0.6]])
    ok = fp64_envelope(freq, ref, phase, dmax, asr)
    assert ok[0, 0] and not ok[0, 1]      # a 6 mm oblate drop: x ~ 4.7, aspect ratio 0.6
    assert ok[1, 0] and ok[1, 1]          # spheres of the same size stay inside to x = 6
    assert ok[2].all()                    # ice: inside at all sizes


def test_bench_tmatrix_cpu_baseline_all_cores():
    """The all-core CPU figure of the bench's T-matrix line: single-bin oracle
    tasks over a spawned pool (no GPU involved)."""
    import multiprocessing as mp
    import bench
    bins = {"dmax": np.array([0.5e-3, 1.0e-3]), "del_d": np.full(2, 1e-4), "ndens": np.full(2, 1e6),
            "density": np.full(2, 300.0), "as_ratio": np.full(2, 0.6), "canting": np.zeros(2)}
    pool = mp.get_context("spawn").Pool(2)
    try:
        v, ntask, wall, ok = bench.tmatrix_cpu_baseline(pool, 2, bins, min_tasks=4)
    finally:
        pool.close()
        pool.join()
    assert ok and ntask == 16 and v > 0 and wall > 0
