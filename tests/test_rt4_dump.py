"""RT4 input files (``pyPamtra.dumpForRT4``, core.py:2595-2697 of the
reference): the run file lists the levels from the top down, and each
scattering file holds the per-km phase matrices, extinction matrices and
emission vectors in RT4's Lobatto block order.  CPU: a run dict with known
values is written and read back position by position.  GPU: the files of a
real ``save_ssp`` run carry that run's single-scattering arrays.
"""
import numpy as np
import pytest

from pamtra_b200 import workloads as wl

N = 16


def _fake_results(pam, rng):
    L = pam._shape3D[2]
    return {"angles_deg": np.concatenate([180.0 - np.linspace(5, 85, N)[::-1], np.linspace(5, 85, N)]),
            "kextatmo": rng.uniform(1e-6, 1e-4, L),
            "scatter_matrix": rng.normal(size=(L, 2, N, 2, N, 4)),
            "extinct_matrix": rng.normal(size=(L, 2, 2, N, 2)),
            "emis_vector": rng.normal(size=(L, 2, N, 2))}


def _nums(line):
    return [float(x) for x in line.split()]


def test_dump_for_rt4_layout(tmp_path):
    pam = wl.golden_pam()   # 3 layers; hydrometeors in layers 1 and 2
    r = _fake_results(pam, np.random.default_rng(1))
    pam.r = r
    run = tmp_path / "run.txt"
    pam.dumpForRT4(str(run), str(tmp_path / "sca"))
    lines = run.read_text().splitlines()
    L = pam._shape3D[2]
    assert len(lines) == L + 1
    # top level first: height km, temperature, gas extinction of the layer below (1/km), file
    top = lines[0].split()
    assert float(top[0]) == pytest.approx(pam.p["hgt_lev"][0, 0, L] / 1e3, abs=5e-3)
    assert float(top[2]) == pytest.approx(r["kextatmo"][L - 1] * 1e3, abs=5e-7)  # %3.6f
    assert lines[0].endswith("'sca_%03d.txt'" % (L - 1))
    assert lines[1].endswith("'sca_001.txt'")
    assert lines[2].endswith("'" + " " * 12 + "'")   # layer 0 carries no hydrometeors
    assert float(lines[-1].split()[2]) == 0.0
    mu = np.cos(np.deg2rad(r["angles_deg"][N:]))
    sm, em, ev = r["scatter_matrix"] * 1e3, r["extinct_matrix"] * 1e3, r["emis_vector"] * 1e3
    lay = 2
    f = (tmp_path / "sca" / ("sca_%03d.txt" % lay)).read_text().splitlines()
    assert f[0].split()[:2] == ["16", "0"] and f[1] == ""
    half = N * 2 * N * 5
    for (si, q, i, j, sj) in ((0, 0, 0, 0, 1), (0, 2, 3, 5, -1), (1, 1, 7, 2, 1), (1, 3, 15, 15, -1)):
        start = 2 + si * half + (i * 2 * N + (N if sj < 0 else 0) + j) * 5
        a = _nums(f[start])
        assert a[0] == pytest.approx((1 - 2 * si) * mu[i], abs=1e-9) and a[1] == pytest.approx(sj * mu[j], abs=1e-9)
        for k in range(2):
            np.testing.assert_allclose(_nums(f[start + 1 + k])[:2], [sm[lay, k, j, 0, i, q], sm[lay, k, j, 1, i, q]],
                                       rtol=1e-12)
        assert _nums(f[start + 3]) == [0.0] * 4
    ext0 = 2 + 2 * half + 1
    assert f[ext0 - 1] == ""
    for h in range(2):
        for i in (0, 9):
            s = ext0 + (h * N + i) * 5
            assert _nums(f[s])[0] == pytest.approx((1 - 2 * h) * mu[i], abs=1e-9)
            np.testing.assert_allclose(_nums(f[s + 2])[:2], [em[lay, 1, 0, i, h], em[lay, 1, 1, i, h]], rtol=1e-12)
    emi0 = ext0 + 2 * N * 5 + 1
    assert f[emi0 - 1] == ""
    for h in range(2):
        v = _nums(f[emi0 + h * N + 4])
        np.testing.assert_allclose(v[:3], [(1 - 2 * h) * mu[4], ev[lay, 0, 4, h], ev[lay, 1, 4, h]], rtol=1e-9)
    assert len(f) == emi0 + 2 * N


@pytest.mark.gpu
def test_dump_for_rt4_after_save_ssp_run(native, tmp_path):
    pam = wl.golden_pam()
    pam.nmlSet["save_ssp"] = True
    pam.runPamtra([35.5])
    pam.dumpForRT4(str(tmp_path / "run.txt"), str(tmp_path / "sca"))
    f = (tmp_path / "sca" / "sca_001.txt").read_text().splitlines()
    np.testing.assert_allclose(_nums(f[3])[:2], pam.r["scatter_matrix"][1, 0, 0, :, 0, 0] * 1e3, rtol=1e-12)
    assert len((tmp_path / "run.txt").read_text().splitlines()) == 4
