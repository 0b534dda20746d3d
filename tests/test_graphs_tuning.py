"""CUDA-graph replay and launch-shape tuning of the batched form.

A captured batch replays bit-identically to a direct run and picks up new
input values written into the same device buffers; every launch shape the
autotuner may choose gives bit-identical results; the tuner's cache keys and
file round trip need no GPU.
"""
import json

import numpy as np
import pytest

from pamtra_b200 import autotune
from pamtra_b200 import batch as pbatch
from pamtra_b200 import workloads as wl


def _np(out):
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_graph_replay_matches_direct_run(native, precision):
    import torch
    from pamtra_b200._native import Engine
    eng = Engine(0)
    b = pbatch.pack_pam(wl.c2_pam(64, seed=31), wl.C2_FREQS)
    direct = _np(pbatch.run(b, 0, precision=precision, eng=eng))
    stream = torch.cuda.Stream()
    g, out = pbatch.capture(b, 0, precision=precision, stream=stream, eng=eng)
    out["tb"].zero_()
    g.launch(stream)
    stream.synchronize()
    assert np.array_equal(out["tb"].cpu().numpy(), direct["tb"])
    assert np.array_equal(out["status"].cpu().numpy(), direct["status"])
    # new values in the captured input buffers give the new results
    dev = b.device_arrays(torch.device("cuda", 0))
    dev["hydro_q"].mul_(0.5)
    g.launch(stream)
    stream.synchronize()
    b2 = pbatch.pack_pam(wl.c2_pam(64, seed=31), wl.C2_FREQS)
    b2.host["hydro_q"] = b2.host["hydro_q"] * 0.5
    ref2 = _np(pbatch.run(b2, 0, precision=precision, eng=eng))
    assert np.array_equal(out["tb"].cpu().numpy(), ref2["tb"])
    assert not np.array_equal(ref2["tb"], direct["tb"])
    g.close()
    eng.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_launch_shapes_give_identical_results(native, precision):
    from pamtra_b200._native import Engine
    eng = Engine(0)
    b = wl.uneven_batch(24, seed=33, nfreq_range=(2, 4))
    ref = _np(pbatch.run(b, 0, precision=precision, eng=eng))
    for shape in autotune.CANDIDATES[1:]:
        eng.set_launch(shape)
        assert eng.get_launch() == shape
        got = _np(pbatch.run(b, 0, precision=precision, eng=eng))
        assert np.array_equal(got["tb"], ref["tb"]), shape
        assert np.array_equal(got["status"], ref["status"]), shape
    with pytest.raises(ValueError):
        eng.set_launch((3, 0, 0, 0))
    eng.close()


@pytest.mark.gpu
def test_autotune_selects_and_caches(native, tmp_path, monkeypatch):
    from pamtra_b200._native import Engine
    monkeypatch.setenv("PAMTRA_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    monkeypatch.setattr(autotune, "_cache", {})
    eng = Engine(0)
    b = pbatch.pack_pam(wl.c2_pam(32, seed=34), wl.C2_FREQS)
    shape, report = autotune.tune(b, 0, eng=eng, reps=1)
    assert eng.get_launch() == shape
    for stage, knobs in autotune.STAGE_KNOBS.items():
        assert len(report[stage]) == len(autotune.CANDIDATES)
        i = int(np.argmin(report[stage]))
        assert all(shape[k] == autotune.CANDIDATES[i][k] for k in knobs)
    assert autotune.lookup(b) == shape
    assert json.load(open(tmp_path / "tune.json"))[autotune.signature(b)] == list(shape)
    eng.close()


def test_tune_cache_signature_and_file(tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("PAMTRA_B200_TUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "_cache", {})
    b = pbatch.pack_pam(wl.c2_pam(48, seed=35), wl.C2_FREQS)
    sig = autotune.signature(b)
    assert sig == "m2_p0_c64_l64_f4_h2"
    assert autotune.signature(b, 1) != sig
    autotune._cache[sig] = (8, 0, 1, 1)
    autotune._save_file()
    monkeypatch.setattr(autotune, "_cache", {})
    assert autotune.lookup(b) == (8, 0, 1, 1)
