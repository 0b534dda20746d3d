"""Single-scattering parity where the CUDA Mie departs most from the
reference's arithmetic: large size parameters and long Mie series.

The Mie-heavy slice has four species of 200 bins up to 10 mm (rain, snow,
graupel, cloud ice) at 89, 157, 176.31 and 190.31 GHz (size parameter up to
about 20, about 35 Mie terms) over temperatures of 240-300 K.  Extinction,
single-scattering albedo, the quadrature phase matrices of every
hydrometeor-bearing layer and frequency, and the per-bin backscattering
cross sections (save_psd) must match the oracle within 1e-9 relative, and
brightness temperatures within 0.01 K (held here to 1e-6 K).  The same is
checked for the NUMMU 8 and 32 phase matrices of the single-column workload.

Reference routines: src/mie_spheres.f90:14-345, src/mie_scat_utilities.f90:
8-160, src/scatcnv.f90:103-192, src/scatProperties.f90:914-949.
"""
import copy

import numpy as np
import pytest

from pamtra_b200 import batch as pbatch
from pamtra_b200 import packing
from pamtra_b200 import workloads as wl

pytestmark = pytest.mark.gpu
REL_TOL = 1e-9
TB_TOL = 1e-6  # K
PSD_NBIN = 200


def _c4_slice(ncol=2, nlay=24, seed=31):
    rng = np.random.default_rng(seed)
    st = wl._settings(16)
    kinds = ["rwc", "swc", "gwc", "iwc"]
    sp = np.empty(4, dtype=packing.SPECIES_DTYPE)
    for j, k in enumerate(kinds):
        sp[j] = wl._species_row(k, np.random.default_rng(200 + j), nbin=200, gamma=(k != "rwc"), rho=400.0)
    nly = np.full(ncol, nlay)
    top = np.full(ncol, 12000.0)
    qs = [[10 ** rng.uniform(-4.0, np.log10(2e-3)) for _ in kinds] for _ in range(ncol)]
    b = wl._packed(st, sp, 0, nly, [wl.MIE_HEAVY_FREQS], None, [kinds] * ncol, qs, top, rng, nlay, 4, False)
    for c in range(ncol):  # 300 K at the ground to 240 K at the top
        b.host["temp_lev"][c, :nlay + 1] = np.linspace(300.0, 240.0, nlay + 1) + rng.uniform(-1.0, 1.0, nlay + 1)
    return b


def _outputs(b, dev):
    import torch
    out = b.alloc_outputs(dev, ssp=True)
    C, F, L = b.ncol, int(b.host["max_nfreq"]), int(b.host["max_nlyrs"])
    H, n = int(b.host["nhydro"]), 2 * b.max_nummu
    out["scatter_matrix"] = torch.zeros((C, F, L, 4, n, n), dtype=torch.float64, device=dev)
    if H:
        for k in ("psd_d", "psd_deltad", "psd_n", "psd_mass", "psd_area", "psd_bscat"):
            out[k] = torch.zeros((C, L, H, PSD_NBIN), dtype=torch.float64, device=dev)
    return out


def _oracle(oracle_mod, b, c, nummu, psd=True):
    h = b.host
    st = copy.copy(b.settings)
    st.nummu = nummu
    freqs = list(h["freqs"])
    err, tb, _, _, d = oracle_mod.run_column(oracle_mod.settings(st), b.species, h, c, freqs, debug=True,
                                             psd_nbin=PSD_NBIN if psd else 0)
    assert err == 0
    return tb, d


def _compare(b, out, oracle_mod, nummu, psd=True):
    tb = out["tb"].cpu().numpy()
    st = out["status"].cpu().numpy()
    kt, sa = out["kexttot"].cpu().numpy(), out["salbedo"].cpu().numpy()
    sm = out["scatter_matrix"].cpu().numpy()
    nchecked = 0
    for c in range(b.ncol):
        assert not np.any(st[c])
        tr, d = _oracle(oracle_mod, b, c, nummu, psd)
        L = int(b.host["nlyrs"][c])
        assert np.max(np.abs(tb[c] - tr)) < TB_TOL
        pres = d["present"].astype(bool)
        np.testing.assert_allclose(kt[c][:, :L][:, pres], d["kexttot"][:, pres], rtol=REL_TOL)
        np.testing.assert_allclose(sa[c][:, :L][:, pres], d["salbedo"][:, pres], rtol=REL_TOL)
        for f in range(d["kexttot"].shape[0]):
            for z in np.nonzero(pres)[0]:
                ref = d["scatter_matrix"][f, z]
                scale = np.max(np.abs(ref))
                assert np.max(np.abs(sm[c, f, z] - ref)) <= REL_TOL * scale, (c, f, z)
                nchecked += 1
        if psd:
            gb = out["psd_bscat"].cpu().numpy()[c, :L]
            rb = d["psd_bscat"]
            ok = np.isfinite(rb) & (rb != -9999.0)
            assert ok.any()
            assert np.array_equal(np.isfinite(gb), np.isfinite(rb))
            np.testing.assert_allclose(gb[ok], rb[ok], rtol=REL_TOL)
    return nchecked


def test_mie_heavy_slice_single_scattering(oracle_mod, native):
    import torch
    dev = torch.device("cuda", 0)
    b = _c4_slice()
    out = _outputs(b, dev)
    pbatch.run(b, 0, out)
    torch.cuda.synchronize()
    assert _compare(b, out, oracle_mod, 16) > 100


@pytest.mark.parametrize("nummu", [8, 32])
def test_phase_matrices_nummu(oracle_mod, native, nummu):
    import torch
    dev = torch.device("cuda", 0)
    b = pbatch.pack_pam(wl.c1_pam(), wl.C1_FREQS, nummu=nummu)
    out = _outputs(b, dev)
    pbatch.run(b, 0, out)
    torch.cuda.synchronize()
    assert _compare(b, out, oracle_mod, nummu) > 20


def test_mie_heavy_slice_split_form(oracle_mod, native):
    """The batched split-precision form (3xTF32 doubling, Legendre
    coefficients stored in FP32) on the Mie-heavy slice: every TB within
    0.05 K of the FP64 oracle."""
    import torch
    from pamtra_b200._native import PREC_3XTF32
    dev = torch.device("cuda", 0)
    b = _c4_slice()
    out = b.alloc_outputs(dev)
    pbatch.run(b, 0, out, precision=PREC_3XTF32)
    torch.cuda.synchronize()
    tb = out["tb"].cpu().numpy()
    assert not np.any(out["status"].cpu().numpy())
    for c in range(b.ncol):
        tr, _ = _oracle(oracle_mod, b, c, 16, psd=False)
        assert np.max(np.abs(tb[c] - tr)) < 0.05


def _large_particles(ncol=1, nlay=12, seed=37):
    """Ice spheres of 900 kg/m3 up to 3 cm and rain up to 8 mm at 89 and
    190.31 GHz: size parameters up to about 60 (about 80 Mie terms, 160
    Legendre orders, 161 quadrature angles), so the coefficient slab takes
    fewer than 32 bins per pass and the Legendre projection runs in several
    chunks of quadrature points."""
    rng = np.random.default_rng(seed)
    st = wl._settings(16)
    sp = np.empty(2, dtype=packing.SPECIES_DTYPE)
    for j, k in enumerate(("gwc", "rwc")):
        sp[j] = wl._species_row(k, np.random.default_rng(300 + j), nbin=100, gamma=False, rho=900.0)
    sp[0]["d_1"], sp[0]["d_2"], sp[0]["p_2"] = 1.0e-4, 3.0e-2, 5.0e-3
    sp[1]["d_1"], sp[1]["d_2"] = 1.0e-4, 8.0e-3
    nly = np.full(ncol, nlay)
    top = np.full(ncol, 6000.0)
    qs = [[10 ** rng.uniform(-3.5, -2.7) for _ in range(2)] for _ in range(ncol)]
    return wl._packed(st, sp, 0, nly, [[89.0, 190.31]], None, [["gwc", "rwc"]] * ncol, qs, top, rng, nlay, 2, False)


def test_long_mie_series(oracle_mod, native):
    import torch
    dev = torch.device("cuda", 0)
    b = _large_particles()
    out = _outputs(b, dev)
    pbatch.run(b, 0, out)
    torch.cuda.synchronize()
    _, d = _oracle(oracle_mod, b, 0, 16, psd=False)
    # about 77 Mie terms: the projection runs over 2 x 77 orders (past the
    # 128-entry Mie-term table) and 155 quadrature points (three chunks)
    assert int(np.max(d["nlegen"])) > 100
    assert _compare(b, out, oracle_mod, 16) > 10
