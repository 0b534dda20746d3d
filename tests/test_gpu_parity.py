"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference's golden fixture.

Tolerances: the plain FP64 form must match brightness temperatures within
0.01 K and extinction / phase-matrix entries within 1e-9 relative; these
tests hold it to 1e-6 K and 1e-9 relative.
"""
import copy
import os
import warnings

import numpy as np
import pytest

import pamtra_b200 as pb
from pamtra_b200 import batch as pbatch
from pamtra_b200 import workloads as wl

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "rain_snow_reference.npz")
TB_TOL = 1e-6  # K
REL_TOL = 1e-9


def _tb_close(pam, oracle_mod, freqs, nummu=16):
    ref, err = oracle_mod.run_pamtra(copy.deepcopy(pam), freqs, nummu=nummu)
    assert err == 0
    pam.runPamtra(freqs)
    assert pam.fortError == 0
    d = np.max(np.abs(pam.r["tb"] - ref["tb"]))
    assert d < TB_TOL, d
    return pam


def test_golden_fixture_through_facade(oracle_mod, native):
    pam = wl.golden_pam()
    pam.runPamtra(wl.GOLDEN_FREQS)
    gold = np.load(GOLDEN)["tb"]
    np.testing.assert_allclose(pam.r["tb"], gold, rtol=1e-5)
    ref, _ = oracle_mod.run_pamtra(wl.golden_pam(), wl.GOLDEN_FREQS)
    assert np.max(np.abs(pam.r["tb"] - ref["tb"])) < TB_TOL
    np.testing.assert_allclose(pam.r["angles_deg"], ref["angles_deg"], rtol=1e-12)
    np.testing.assert_allclose(pam.r["emissivity"], 0.6)


def test_c1_tb_and_single_scattering(oracle_mod, native):
    pam = wl.c1_pam()
    pam.nmlSet["save_ssp"] = True
    pam.runPamtra(wl.C1_FREQS)
    ref, err = oracle_mod.run_pamtra(wl.c1_pam(), wl.C1_FREQS, debug=True)
    assert err == 0 and pam.fortError == 0
    assert np.max(np.abs(pam.r["tb"] - ref["tb"])) < TB_TOL
    d = ref["debug"][0]
    pres = d["present"].astype(bool)
    kt = pam.r["kexttot_all"][0, 0]
    np.testing.assert_allclose(kt[:, pres], d["kexttot"][:, pres], rtol=REL_TOL)
    np.testing.assert_allclose(pam.r["salbedo_all"][0, 0][:, pres], d["salbedo"][:, pres], rtol=REL_TOL)
    np.testing.assert_allclose(pam.r["kextatmo_all"][0, 0], d["kextatmo"], rtol=REL_TOL)
    # phase matrices of the last frequency (save_ssp semantics), relative to the largest entry
    sm = pam.r["scatter_matrix"]  # (L, 2, N, 2, N, 4)
    ro = d["scatter_matrix"][-1]  # (L, 4, n, n), row = i2 + 2 j2, col = i1 + 2 j1
    ro6 = ro.reshape(ro.shape[0], 4, 16, 2, 16, 2).transpose(0, 3, 2, 5, 4, 1)
    for z in np.nonzero(pres)[0]:
        scale = np.max(np.abs(ro6[z]))
        assert np.max(np.abs(sm[z] - ro6[z])) <= REL_TOL * scale
    np.testing.assert_allclose(pam.r["kextatmo"], d["kextatmo"][-1], rtol=REL_TOL)


def test_num_doubles_match(oracle_mod, native):
    b = pbatch.pack_pam(wl.c1_pam(), wl.C1_FREQS)
    import torch
    out = b.alloc_outputs(torch.device("cuda", 0), ssp=True)
    pbatch.run(b, 0, out)
    torch.cuda.synchronize()
    nd = out["num_doubles"].cpu().numpy()[0]
    ref, _ = oracle_mod.run_pamtra(wl.c1_pam(), wl.C1_FREQS, debug=True)
    assert np.array_equal(nd, ref["debug"][0]["num_doubles"])


def test_gas_and_tkc_kernels(oracle_mod, native):
    import torch
    rng = np.random.default_rng(3)
    n = 257
    f = rng.uniform(1.0, 300.0, n)
    T = rng.uniform(190.0, 310.0, n)
    rv = rng.uniform(0.0, 0.02, n)
    p = rng.uniform(100.0, 1.1e5, n)
    dev = torch.device("cuda", 0)
    tt = [torch.from_numpy(x).to(dev) for x in (f, T, rv, p)]
    k = torch.zeros(n, dtype=torch.float64, device=dev)
    st = torch.zeros(n, dtype=torch.int32, device=dev)
    lib = native.load()
    assert lib.pamtra_b200_gas_r98(*[x.data_ptr() for x in tt], k.data_ptr(), st.data_ptr(), n, None) == 0
    torch.cuda.synchronize()
    ref = np.array([oracle_mod.gas_r98(*v)[1] for v in zip(f, T, rv, p)])
    np.testing.assert_allclose(k.cpu().numpy(), ref, rtol=1e-12)
    assert st.cpu().numpy().max() == 0
    tc = torch.from_numpy(rng.uniform(-40.0, 40.0, n)).to(dev)
    fr = torch.from_numpy(rng.uniform(1.0, 500.0, n)).to(dev)
    er = torch.zeros(n, dtype=torch.float64, device=dev)
    ei = torch.zeros(n, dtype=torch.float64, device=dev)
    assert lib.pamtra_b200_eps_water_tkc(tc.data_ptr(), fr.data_ptr(), er.data_ptr(), ei.data_ptr(), n, None) == 0
    torch.cuda.synchronize()
    ref = np.array([oracle_mod.eps_water_tkc(a, b_) for a, b_ in zip(tc.cpu().numpy(), fr.cpu().numpy())])
    np.testing.assert_allclose(er.cpu().numpy(), ref.real, rtol=1e-12)
    np.testing.assert_allclose(ei.cpu().numpy(), ref.imag, rtol=1e-12)


@pytest.mark.parametrize("n", [16, 32, 64])
def test_minvert_kernel(native, n):
    import torch
    rng = np.random.default_rng(n)
    cnt = 7
    a = rng.normal(size=(cnt, n, n)) + 2.0 * np.eye(n)
    a[0] = np.kron(np.eye(n // 2), np.array([[0.0, 1.0], [1.0, 0.0]]))  # needs pivoting
    dev = torch.device("cuda", 0)
    # column-major per matrix
    at = torch.from_numpy(np.ascontiguousarray(a.transpose(0, 2, 1))).to(dev)
    inv = torch.zeros_like(at)
    st = torch.zeros(cnt, dtype=torch.int32, device=dev)
    assert native.load().pamtra_b200_minvert_batched(at.data_ptr(), inv.data_ptr(), st.data_ptr(), n, cnt, None) == 0
    torch.cuda.synchronize()
    got = inv.cpu().numpy().transpose(0, 2, 1)
    np.testing.assert_allclose(got, np.linalg.inv(a), rtol=1e-9, atol=1e-12)
    assert st.cpu().numpy().max() == 0


# ----------------------------------------------------------------- edge cases
def _custom_pam(nlay=30, q=None, species=(wl.CLOUD_C1, wl.RAIN_C1), nml=None, **prof):
    warnings.simplefilter("ignore")
    pam = pb.pyPamtra()
    for s in species:
        pam.df.addHydrometeor(s)
    for k, v in (nml or {}).items():
        pam.nmlSet[k] = v
    hl = np.linspace(0.0, 10000.0, nlay + 1)
    _, p, T = pb.meteoSI.usStandard(hl)
    kw = dict(hgt_lev=hl, temp_lev=T, press_lev=p, relhum_lev=np.full(nlay + 1, 70.0))
    if species:
        hq = np.zeros((nlay, len(species)))
        if q is not None:
            for (z, h), v in q.items():
                hq[z, h] = v
        kw["hydro_q"] = hq
    kw.update(prof)
    pam.createProfile(**kw)
    return pam


CASES = {
    "clear_sky": dict(),
    "top_layer": dict(q={(29, 0): 5e-4, (29, 1): 5e-4}),
    "bottom_layer": dict(q={(0, 1): 1e-3}),
    "single_species_cloud": dict(q={(10, 0): 3e-4, (11, 0): 3e-4}),
    "lambert": dict(q={(5, 1): 1e-3}, sfc_refl="L", groundtemp=280.0),
    "emissivity_one": dict(q={(5, 1): 1e-3}, nml={"emissivity": 1.0}),
    "outpol_iq": dict(q={(5, 1): 1e-3}, nml={"outpol": "IQ"}),
    "no_gas": dict(q={(5, 1): 1e-3}, nml={"lgas_extinction": False}),
    "no_emission": dict(q={(5, 1): 1e-3, (6, 0): 1e-4}, nml={"lhyd_emission": False}),
    "no_absorption_flag": dict(q={(5, 1): 1e-3}, nml={"lhyd_absorption": False}),
    "adaptive_off": dict(q={(5, 1): 1e-3}, nml={"hydro_adaptive_grid": False}),
    "toa_only": dict(q={(5, 1): 1e-3}, obs_height=[833000.0]),
    "surface_first": dict(q={(5, 1): 1e-3}, obs_height=[0.0, 833000.0]),
    "mgamma_ice_mix": dict(q={(8, 0): 2e-4, (9, 0): 2e-4},
                           species=(("gwc_q", -99.0, -1, 400.0, -99.0, -99.0, -99.0, -99.0, 3, 40, "mgamma",
                                     -99.0, 4.0e-4, 2.0, 1.0, 1.0e-5, 5.0e-3, "mie-sphere", "none", -99.0),)),
    "mono": dict(q={(8, 0): 2e-4},
                 species=(("mono_q", -99.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 3, 2, "mono",
                           -99.0, -99.0, -99.0, -99.0, 5.0e-4, -99.0, "mie-sphere", "none", -99.0),)),
    "ice_default_density": dict(q={(12, 0): 3e-4},
                                species=(("iwc_q", -99.0, -1, -99.0, 0.038, 2.0, -99.0, -99.0, 3, 30, "exp_field_t",
                                          -99.0, -99.0, -99.0, -99.0, 1e-5, 5e-3, "mie-sphere", "none", -99.0),)),
    "no_hydrometeor_species": dict(species=()),
}


# cases where the reference itself stops in check_norm4 (src/radscat4.f90:125):
# without hydrometeor emission the emission vector no longer balances the
# absorption part of the extinction
EXPECT_FATAL = {"no_emission"}


@pytest.mark.parametrize("case", sorted(CASES))
def test_edge_case(case, oracle_mod, native):
    kw = dict(CASES[case])
    pam = _custom_pam(**kw)
    if case in EXPECT_FATAL:
        _, err = oracle_mod.run_pamtra(copy.deepcopy(pam), [23.8, 89.0])
        assert err == 2
        pam.runPamtra([23.8, 89.0], failOnError=False)
        assert pam.fortError == 2
        assert np.any(pam.r["status"] & 0x100)
        return
    _tb_close(pam, oracle_mod, [23.8, 89.0])


def test_nummu_8(oracle_mod, native):
    from pamtra_b200.libWrapper import PamtraFortranWrapper
    pam = _custom_pam(q={(5, 1): 1e-3, (6, 0): 2e-4})
    ref, _ = oracle_mod.run_pamtra(copy.deepcopy(pam), [31.4, 150.0], nummu=8)
    pam._prepare_freqs([31.4, 150.0])
    res, err, _ = PamtraFortranWrapper(pam.set, pam.nmlSet, pam.df.data, {}, {}, pam.p, nummu=8)
    assert err == 0
    assert np.max(np.abs(res["tb"] - ref["tb"])) < TB_TOL


def test_nummu_32(oracle_mod, native):
    from pamtra_b200.libWrapper import PamtraFortranWrapper
    pam = _custom_pam(q={(5, 1): 1e-3, (6, 0): 2e-4, (7, 1): 3e-3})
    ref, _ = oracle_mod.run_pamtra(copy.deepcopy(pam), [31.4, 150.0], nummu=32)
    pam._prepare_freqs([31.4, 150.0])
    res, err, _ = PamtraFortranWrapper(pam.set, pam.nmlSet, pam.df.data, {}, {}, pam.p, nummu=32)
    assert err == 0
    assert np.max(np.abs(res["tb"] - ref["tb"])) < TB_TOL


def _oracle_packed_column(oracle_mod, b, c):
    """Oracle TB of column c of a packed batch with per-column settings."""
    h = b.host
    st = copy.copy(b.settings)
    if h.get("nummu") is not None:
        st.nummu = int(h["nummu"][c])
    H = int(h["nhydro"])
    sp = b.species[c * H:(c + 1) * H] if b.species_stride else b.species
    freqs = h["freqs"][c, :int(h["nfreq"][c])] if h.get("nfreq") is not None else h["freqs"]
    err, tb, _, _, _ = oracle_mod.run_column(oracle_mod.settings(st), sp, h, c, list(freqs))
    return err, tb, int(st.nummu), len(freqs)


def test_uneven_batch_against_oracle(oracle_mod, native):
    # per-column layer counts, species sets, PSD forms, ice densities,
    # frequency lists and NUMMU in one launch sequence
    import torch
    b = wl.uneven_batch(9, seed=11, nfreq_range=(2, 4))
    assert b.nummu_mask == 7
    out = pbatch.run(b, 0)
    torch.cuda.synchronize()
    tb = out["tb"].cpu().numpy()
    status = out["status"].cpu().numpy()
    for c in range(b.ncol):
        err, t, N, nf = _oracle_packed_column(oracle_mod, b, c)
        assert err == 0 and not np.any(status[c, :nf])
        d = np.max(np.abs(tb[c][:, :2 * N, :nf, :] - t))
        assert d < TB_TOL, (c, N, d)
        assert np.all(tb[c][:, 2 * N:, :, :] == -9999.0)


def test_chunked_run_equals_single_run(native):
    # chunks grouped by NUMMU and trimmed to their own sizes give the same
    # bits as one launch over the whole batch
    import torch
    b = wl.uneven_batch(24, seed=12, nfreq_range=(2, 6))
    one = pbatch.run(b, 0)
    torch.cuda.synchronize()
    ch = pbatch.chunk_columns(b, 96 << 20)
    assert len(ch) > 2
    got = pbatch.run_chunked(b, 96 << 20)
    assert np.array_equal(got["tb"], one["tb"].cpu().numpy())
    assert np.array_equal(got["status"], one["status"].cpu().numpy())


def test_ragged_columns(oracle_mod, native):
    # three columns with 30, 24 and 18 layers, padded with -9999 (pyPamtra convention)
    warnings.simplefilter("ignore")
    pam = pb.pyPamtra()
    pam.df.addHydrometeor(wl.CLOUD_C1)
    pam.df.addHydrometeor(wl.RAIN_C1)
    L = 30
    hl = np.full((3, L + 1), -9999.0)
    tl = np.full((3, L + 1), -9999.0)
    pl = np.full((3, L + 1), -9999.0)
    hq = np.zeros((3, L, 2))
    for c, nl in enumerate((30, 24, 18)):
        h = np.linspace(0.0, 9000.0, nl + 1)
        _, p, T = pb.meteoSI.usStandard(h)
        hl[c, :nl + 1], tl[c, :nl + 1], pl[c, :nl + 1] = h, T, p
        hq[c, 3:8, 1] = 8e-4
    hgt = np.where(hl[:, 1:] > -9999, 0.5 * (hl[:, 1:] + hl[:, :-1]), -9999.0)
    pam.createProfile(hgt_lev=hl, hgt=hgt, temp_lev=tl, press_lev=pl, relhum_lev=np.where(hl > -9999, 60.0, -9999.0),
                      hydro_q=hq)
    assert list(pam.p["nlyrs"].ravel()) == [30, 24, 18]
    ref, _ = oracle_mod.run_pamtra(copy.deepcopy(pam), [89.0])
    pam.runPamtra([89.0], checkData=False)
    assert np.max(np.abs(pam.r["tb"] - ref["tb"])) < TB_TOL


def test_norm_failure_is_reported(native):
    # without scattering the phase function no longer integrates to the
    # scattering coefficient; the reference aborts in check_norm4
    pam = _custom_pam(q={(5, 1): 5e-3, (6, 1): 5e-3}, nml={"lhyd_scattering": False})
    with pytest.raises(RuntimeError):
        pam.runPamtra([89.0])
    pam.runPamtra([89.0], failOnError=False)
    assert pam.fortError == 2
    assert np.all(pam.r["status"] & 0x100)


# ----------------------------------------------------------------- batched form
def test_batched_equals_plain_bitwise(native):
    import torch
    dev = torch.device("cuda", 0)
    big = pbatch.pack_pam(wl.c2_pam(16, seed=5), wl.C2_FREQS)
    out = pbatch.run(big, 0)
    torch.cuda.synchronize()
    tb = out["tb"].cpu().numpy()
    pam_all = wl.c2_pam(16, seed=5)
    for c in range(16):
        pam1 = copy.deepcopy(pam_all)
        sel = np.zeros((16, 1), dtype=bool)
        sel[c, 0] = True
        for k in ("hgt_lev", "temp_lev", "press_lev", "relhum_lev", "hgt", "hydro_q", "hydro_n", "hydro_reff",
                  "obs_height", "groundtemp", "nlyrs", "sfc_refl", "sfc_type"):
            pam1.p[k] = pam1.p[k][c:c + 1]
        pam1.p["ngridx"] = 1
        one = pbatch.pack_pam(pam1, wl.C2_FREQS)
        o1 = pbatch.run(one, 0)
        torch.cuda.synchronize()
        assert np.array_equal(o1["tb"].cpu().numpy()[0], tb[c])


def test_host_path_equals_device_path(native):
    import torch
    b = pbatch.pack_pam(wl.c2_pam(32, seed=6), wl.C2_FREQS)
    dv = pbatch.run(b, 0)
    torch.cuda.synchronize()
    hv = pbatch.run_host(b, 0)
    assert np.array_equal(dv["tb"].cpu().numpy(), hv["tb"])
    assert np.array_equal(dv["status"].cpu().numpy(), hv["status"])


def test_c2_full_size_properties(oracle_mod, native):
    import torch
    b = pbatch.pack_pam(wl.c2_pam(4096), wl.C2_FREQS)
    out = pbatch.run(b, 0)
    torch.cuda.synchronize()
    tb = out["tb"].cpu().numpy()
    assert int((out["status"] != 0).sum()) == 0
    assert np.all((tb > 2.7) & (tb < 330.0))
    # sampled columns against the oracle
    for c in (0, 1234, 4095):
        err, t, _, _, _ = oracle_mod.run_column(oracle_mod.settings(b.settings), b.species, b.host, c, wl.C2_FREQS)
        assert err == 0
        assert np.max(np.abs(tb[c] - t)) < TB_TOL
    # a second run is bit-identical (deterministic scheduling independence)
    out2 = pbatch.run(b, 0)
    torch.cuda.synchronize()
    assert np.array_equal(out2["tb"].cpu().numpy(), tb)


# ----------------------------------------------------------------- tensor-core products
def test_mmult_3xtf32_kernel(native):
    # 3xTF32 tcgen05 products: FP32-level accuracy (a single TF32 product
    # would be off by ~1e-3 relative)
    import torch
    rng = np.random.default_rng(17)
    cnt = 300
    a = rng.normal(size=(cnt, 32, 32))
    b = rng.normal(size=(cnt, 32, 32))
    dev = torch.device("cuda", 0)
    at = torch.from_numpy(np.ascontiguousarray(a.transpose(0, 2, 1))).to(dev)
    bt = torch.from_numpy(np.ascontiguousarray(b.transpose(0, 2, 1))).to(dev)
    ct = torch.zeros_like(at)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    rc = native.load().pamtra_b200_mmult_3xtf32_batched(at.data_ptr(), bt.data_ptr(), ct.data_ptr(), 32, cnt,
                                                        err.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    c = ct.cpu().numpy().transpose(0, 2, 1)
    ref = a @ b
    rel = np.max(np.abs(c - ref)) / np.max(np.abs(ref))
    assert rel < 2e-6, rel


# ----------------------------------------------------------------- split-precision batched form
SPLIT_TB_TOL = 0.05  # K: every TB of the 3xTF32 batched form against FP64


def _run_prec(b, prec):
    import torch
    out = pbatch.run(b, 0, precision=prec)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def test_split_precision_c2(oracle_mod, native):
    from pamtra_b200._native import PREC_3XTF32, PREC_FP64
    b = pbatch.pack_pam(wl.c2_pam(96, seed=8), wl.C2_FREQS)
    f64 = _run_prec(b, PREC_FP64)
    s = _run_prec(b, PREC_3XTF32)
    assert int(np.count_nonzero(s["status"])) == 0
    d = np.abs(s["tb"] - f64["tb"])
    assert np.max(d) <= SPLIT_TB_TOL, np.max(d)
    assert np.max(d) > 0.0  # the products really ran in split precision
    for c in (0, 47, 95):
        err, t, _, _, _ = oracle_mod.run_column(oracle_mod.settings(b.settings), b.species, b.host, c, wl.C2_FREQS)
        assert err == 0
        assert np.max(np.abs(s["tb"][c] - t)) <= SPLIT_TB_TOL


def test_split_precision_target_shape(native):
    from pamtra_b200._native import PREC_3XTF32, PREC_FP64
    b = wl.target_batch(48, seed=9)
    f64 = _run_prec(b, PREC_FP64)
    s = _run_prec(b, PREC_3XTF32)
    assert int(np.count_nonzero(s["status"])) == 0
    assert np.max(np.abs(s["tb"] - f64["tb"])) <= SPLIT_TB_TOL


def test_split_precision_uneven(native):
    # NUMMU 16 and 32 columns take the tensor-core doubling, NUMMU 8 the FP64
    # one; NUMMU 16 columns also the tensor-core adding, NUMMU 8 and 32 the
    # one-inverse FP64 adding of the batched FP64 form.  The split form
    # stores the Legendre coefficients in FP32, so its NUMMU 8 columns differ
    # from the batched FP64 form only by that rounding (micro-kelvin).
    from pamtra_b200._native import PREC_3XTF32, PREC_FP64, PREC_FP64_BATCHED
    b = wl.uneven_batch(24, seed=13, nfreq_range=(2, 5))
    f64 = _run_prec(b, PREC_FP64)
    f64b = _run_prec(b, PREC_FP64_BATCHED)
    s = _run_prec(b, PREC_3XTF32)
    assert np.array_equal(s["status"], f64["status"])
    nmu = b.host["nummu"]
    d = np.abs(s["tb"] - f64["tb"])
    assert np.max(d) <= SPLIT_TB_TOL
    assert np.max(d[nmu == 32]) > 0.0  # NUMMU 32 ran in split precision
    d8 = np.abs(s["tb"][nmu == 8] - f64b["tb"][nmu == 8])
    assert np.max(d8) < 1e-4


def test_split_precision_nummu_32(oracle_mod, native):
    # the n = 64 split-precision kernel (one item per CTA, K = 64 operand tiles)
    # against the oracle and the FP64 form, and run-to-run reproducible
    from pamtra_b200._native import PREC_3XTF32, PREC_FP64
    b = wl.uneven_batch(12, seed=47, nummu_choices=(32,), nfreq_range=(2, 3))
    f64 = _run_prec(b, PREC_FP64)
    s = _run_prec(b, PREC_3XTF32)
    assert int(np.count_nonzero(s["status"])) == 0
    assert np.max(np.abs(s["tb"] - f64["tb"])) <= SPLIT_TB_TOL
    again = _run_prec(b, PREC_3XTF32)
    assert np.array_equal(again["tb"], s["tb"])
    for c in (0, 11):
        err, t, N, nf = _oracle_packed_column(oracle_mod, b, c)
        assert err == 0 and N == 32
        assert np.max(np.abs(s["tb"][c][:, :2 * N, :nf, :] - t)) <= SPLIT_TB_TOL


def test_split_precision_pairing_independent(native):
    # The split-precision layer and adding kernels carry two items (units)
    # per tensor-core MMA; each one's result depends on its own operands
    # only, so a column gives bit-identical TBs when the items around it (and
    # hence the pairs) change.  Three frequencies make the per-column item
    # count odd, so dropping the first column re-pairs every later item.
    from pamtra_b200._native import PREC_3XTF32
    freqs = [23.8, 31.4, 89.0]
    b = pbatch.pack_pam(wl.c2_pam(9, seed=21), freqs)
    full = _run_prec(b, PREC_3XTF32)
    assert int(np.count_nonzero(full["status"])) == 0
    sub = _run_prec(pbatch.subset(b, list(range(1, 9))), PREC_3XTF32)
    assert np.array_equal(sub["tb"], full["tb"][1:])
    again = _run_prec(b, PREC_3XTF32)
    assert np.array_equal(again["tb"], full["tb"])


# ----------------------------------------------------------------- batched FP64 form (one-inverse adding)
def test_fp64_batched_form_matches_plain_order(oracle_mod, native):
    # The batched FP64 form derives each combine's minus-side inverse from
    # the plus-side one; it stays within 1e-10 K of the reference operation
    # order, is run-to-run reproducible and matches the oracle.
    from pamtra_b200._native import PREC_FP64, PREC_FP64_BATCHED
    b = pbatch.pack_pam(wl.c2_pam(48, seed=41), wl.C2_FREQS)
    ref = _run_prec(b, PREC_FP64)
    got = _run_prec(b, PREC_FP64_BATCHED)
    assert np.array_equal(got["status"], ref["status"])
    assert np.max(np.abs(got["tb"] - ref["tb"])) < 1e-10
    again = _run_prec(b, PREC_FP64_BATCHED)
    assert np.array_equal(again["tb"], got["tb"])
    for c in (0, 47):
        err, t, _, _, _ = oracle_mod.run_column(oracle_mod.settings(b.settings), b.species, b.host, c, wl.C2_FREQS)
        assert err == 0
        assert np.max(np.abs(got["tb"][c] - t)) < TB_TOL


def test_fp64_batched_form_uneven(native):
    # every NUMMU and surface path through the one-inverse combine
    from pamtra_b200._native import PREC_FP64, PREC_FP64_BATCHED
    b = wl.uneven_batch(24, seed=43, nfreq_range=(2, 5))
    ref = _run_prec(b, PREC_FP64)
    got = _run_prec(b, PREC_FP64_BATCHED)
    assert np.array_equal(got["status"], ref["status"])
    ok = ref["status"] == 0
    d = np.abs(got["tb"] - ref["tb"])
    assert np.max(d) < 1e-10, np.max(d)


# ----------------------------------------------------------------- simple radar (active, radar_mode 'simple')
def test_simple_radar_golden_fixture(oracle_mod, native):
    # Ze and Att_hydro of the reference's golden scenario (its nmlSet has
    # active=True, radar_mode='simple'), through the pyPamtra facade
    pam = wl.golden_pam()
    pam.runPamtra(wl.GOLDEN_FREQS)
    gold = np.load(GOLDEN)
    np.testing.assert_allclose(pam.r["Ze"], gold["Ze"], rtol=1e-5)
    np.testing.assert_allclose(pam.r["Att_hydro"], gold["Att_hydro"], rtol=1e-5)
    ref, err = oracle_mod.run_pamtra(wl.golden_pam(), wl.GOLDEN_FREQS)
    assert err == 0
    np.testing.assert_allclose(pam.r["Ze"], ref["Ze"], rtol=REL_TOL, atol=1e-12)
    np.testing.assert_allclose(pam.r["Att_hydro"], ref["Att_hydro"], rtol=REL_TOL, atol=1e-15)
    np.testing.assert_allclose(pam.r["Att_atmo"], ref["Att_atmo"], rtol=REL_TOL, atol=1e-15)


@pytest.mark.parametrize("attenuation", ["bottom-up", "top-down"])
def test_simple_radar_path_integrated_attenuation(oracle_mod, native, attenuation):
    # two-way path-integrated attenuation from the surface or from the top
    # (src/radar_simulator.f90:130-156), over columns with clouds and rain
    pam = wl.c1_pam()
    pam.nmlSet["radar_attenuation"] = attenuation
    pam.nmlSet["radar_polarisation"] = "NN,HV"
    pam.runPamtra(wl.C1_FREQS)
    p2 = wl.c1_pam()
    p2.nmlSet["radar_attenuation"] = attenuation
    ref, err = oracle_mod.run_pamtra(p2, wl.C1_FREQS)
    assert err == 0
    ze = pam.r["Ze"]
    assert ze.shape[-2:] == (2, 1)
    np.testing.assert_allclose(ze[..., 0:1, :], ref["Ze"], rtol=REL_TOL, atol=1e-12)
    assert np.all(ze[..., 1, :] == -9999.0)  # no cross-polar backscatter from spheres
    np.testing.assert_allclose(pam.r["Att_hydro"], ref["Att_hydro"], rtol=REL_TOL, atol=1e-15)
    np.testing.assert_allclose(pam.r["Att_atmo"], ref["Att_atmo"], rtol=REL_TOL, atol=1e-15)
    # attenuation lowers the reflectivity where hydrometeors lie beyond
    p3 = wl.c1_pam()
    p3.runPamtra(wl.C1_FREQS)
    has = ze[..., 0, 0] > -9999
    assert np.all(ze[..., 0, 0][has] <= p3.r["Ze"][..., 0, 0][has] + 1e-12)
