"""The allocation-free entry point (pamtra_b200_run_noalloc).

It serves callers that cannot call cudaMalloc -- hosts whose own device
memory manager owns every allocation, and latency-critical callers that
cannot accept an allocation's device-wide synchronisation.  It runs the plain
form of one column with its scratch in a fixed static device array, so this
test calls it through the C ABI twice in a row and compares both results with
the context-based entry point pamtra_b200_run.
"""
import ctypes

import numpy as np
import pytest

from pamtra_b200 import batch as pbatch
from pamtra_b200 import workloads as wl

pytestmark = pytest.mark.gpu
TB_TOL = 1e-6  # K, the tolerance of the other GPU parity tests


def _device_inputs():
    import torch
    dev = torch.device("cuda", 0)
    b = pbatch.pack_pam(wl.c1_pam(), wl.C1_FREQS)
    arrs = b.device_arrays(dev)
    sp_dev = torch.from_numpy(np.frombuffer(b.species.tobytes(), dtype=np.uint8).copy()).to(dev)
    return b, arrs, sp_dev, dev


def test_noalloc_matches_context_entry_point(native):
    import torch
    b, arrs, sp_dev, dev = _device_inputs()
    eng = native.engine(0)
    ref = b.alloc_outputs(dev)
    eng.run(b.settings, b.columns(arrs), eng.make_outputs(ref))
    torch.cuda.synchronize()
    tb_ref = ref["tb"].cpu().numpy()
    assert int(ref["status"].abs().sum()) == 0

    lib = native.load()
    cols = b.columns(arrs)
    cols.species = sp_dev.data_ptr()  # device pointer on this entry point
    for _ in range(2):
        out = b.alloc_outputs(dev)
        rc = lib.pamtra_b200_run_noalloc(ctypes.byref(b.settings), ctypes.byref(cols),
                                         ctypes.byref(eng.make_outputs(out)), None)
        assert rc == 0
        torch.cuda.synchronize()
        tb = out["tb"].cpu().numpy()
        assert int(out["status"].abs().sum()) == 0
        assert np.max(np.abs(tb - tb_ref)) <= TB_TOL
        np.testing.assert_allclose(out["angles_deg"].cpu().numpy(), ref["angles_deg"].cpu().numpy(), rtol=1e-12)


def test_noalloc_rejects_oversized_requests(native):
    import torch
    b, arrs, sp_dev, dev = _device_inputs()
    lib = native.load()
    cols = b.columns(arrs)
    cols.species = sp_dev.data_ptr()
    out = b.alloc_outputs(dev)
    o = native.Engine.make_outputs(out)
    cols.max_nfreq = 5  # above PAMTRA_B200_NOALLOC_MAX_NFREQ
    assert lib.pamtra_b200_run_noalloc(ctypes.byref(b.settings), ctypes.byref(cols), ctypes.byref(o), None) == \
        (2 | native.ST_SIZE)
    cols.max_nfreq = 3
    cols.ncol = 2
    assert lib.pamtra_b200_run_noalloc(ctypes.byref(b.settings), ctypes.byref(cols), ctypes.byref(o), None) == \
        (2 | native.ST_SIZE)
    torch.cuda.synchronize()
