"""The split-precision adding (k_adding_tc + k_adding_finish, PREC_3XTF32 for
NUMMU 16): COMBINE_LAYERS4 (src/radintg4.f90:447-513) with its products as
3xTF32 tensor-core MMAs over FP32 stacks, the (I - R R)^-1 of every combine,
the surface coupling and the radiances in FP64.

Held to the batched form with the FP64 adding (PREC_3XTF32_FP64ADD, the same
split-precision doubling) within 0.02 K and to the FP64 oracle within the
split-precision bound of 0.05 K, on the headline and target shapes and on
columns whose layer structure walks every state of the adding stack: empty,
clear only, a scattering layer first (top), after clear layers (bottom),
alone in the middle, adjacent to another, alternating with clear layers, and
a dense cloud.  Three frequencies make the units of a CTA pair straddle
columns.
"""
import warnings

import numpy as np
import pytest

import pamtra_b200 as pb
from pamtra_b200 import batch as pbatch
from pamtra_b200 import workloads as wl
from pamtra_b200._native import PREC_3XTF32, PREC_3XTF32_FP64ADD

pytestmark = pytest.mark.gpu
TOL_VS_FP64_ADDING = 0.02  # K
SPLIT_TB_TOL = 0.05        # K, against the FP64 oracle
FREQS = [23.8, 89.0, 150.0]

STRUCTURES = {
    "clear_sky": {},
    "top_layer": {(29, 1): 1e-3},
    "bottom_layer": {(0, 1): 1e-3},
    "middle_layer": {(14, 1): 1e-3, (14, 0): 3e-4},
    "adjacent_pair": {(10, 1): 8e-4, (11, 1): 8e-4},
    "alternating": {(5, 1): 5e-4, (7, 1): 5e-4, (9, 0): 3e-4, (11, 1): 5e-4, (13, 0): 3e-4},
    "dense": {**{(z, 1): 6e-4 for z in range(3, 26)}, **{(z, 0): 2e-4 for z in range(8, 20)}},
}


def _pam(q):
    warnings.simplefilter("ignore")
    pam = pb.pyPamtra()
    pam.df.addHydrometeor(wl.CLOUD_C1)
    pam.df.addHydrometeor(wl.RAIN_C1)
    nlay = 30
    hl = np.linspace(0.0, 10000.0, nlay + 1)
    _, p, T = pb.meteoSI.usStandard(hl)
    hq = np.zeros((nlay, 2))
    for (z, h), v in q.items():
        hq[z, h] = v
    pam.createProfile(hgt_lev=hl, temp_lev=T, press_lev=p, relhum_lev=np.full(nlay + 1, 70.0), hydro_q=hq)
    return pam


def _run(b, prec):
    import torch
    out = pbatch.run(b, 0, precision=prec)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


def _check(b, oracle_mod, cols, freqs):
    s = _run(b, PREC_3XTF32)
    f = _run(b, PREC_3XTF32_FP64ADD)
    assert int(np.count_nonzero(s["status"])) == 0
    assert int(np.count_nonzero(f["status"])) == 0
    d = np.abs(s["tb"] - f["tb"])
    assert np.max(d) <= TOL_VS_FP64_ADDING, np.max(d)
    h = b.host
    H = int(h["nhydro"])
    for c in cols:
        sp = b.species[c * H:(c + 1) * H] if b.species_stride else b.species
        err, t, _, _, _ = oracle_mod.run_column(oracle_mod.settings(b.settings), sp, h, c, freqs)
        assert err == 0
        nf = len(freqs)
        assert np.max(np.abs(s["tb"][c][:, :, :nf, :] - t)) <= SPLIT_TB_TOL, c
    return s, f, d


def test_split_adding_c2(oracle_mod, native):
    b = pbatch.pack_pam(wl.c2_pam(64, seed=30), wl.C2_FREQS)
    s, f, d = _check(b, oracle_mod, (0, 31, 63), wl.C2_FREQS)
    assert np.max(d) > 0.0  # the adding products really ran in split precision
    again = _run(b, PREC_3XTF32)
    assert np.array_equal(again["tb"], s["tb"])  # run to run reproducible


def test_split_adding_target_shape(native):
    b = wl.target_batch(24, seed=31)
    s = _run(b, PREC_3XTF32)
    f = _run(b, PREC_3XTF32_FP64ADD)
    assert int(np.count_nonzero(s["status"])) == 0
    assert np.max(np.abs(s["tb"] - f["tb"])) <= TOL_VS_FP64_ADDING


def test_split_adding_layer_structures(oracle_mod, native):
    parts = [pbatch.pack_pam(_pam(q), FREQS) for q in STRUCTURES.values()]
    b, _ = pbatch.concat(parts)
    assert b.ncol == len(STRUCTURES)
    s, f, d = _check(b, oracle_mod, range(b.ncol), FREQS)
    # a clear column has no combine: both adding forms reduce to the same
    # FP64 vector recursion up to the FP32 stack
    assert np.max(d[0]) < 1e-3


def test_split_adding_partner_independent(native):
    # each unit's TB depends on its own layers only: dropping the first
    # structure re-pairs every later unit (three frequencies per column)
    parts = [pbatch.pack_pam(_pam(q), FREQS) for q in STRUCTURES.values()]
    b, _ = pbatch.concat(parts)
    full = _run(b, PREC_3XTF32)
    sub = _run(pbatch.subset(b, list(range(1, b.ncol))), PREC_3XTF32)
    assert np.array_equal(sub["tb"], full["tb"][1:])
