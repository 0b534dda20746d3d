"""The allocation-free entry point (pamtra_b200_run_noalloc).

It serves callers that cannot call cudaMalloc -- hosts whose own device
memory manager owns every allocation, and latency-critical callers that
cannot accept an allocation's device-wide synchronisation.  It runs the plain
form of one column with its scratch in a fixed static device array, so this
test calls it through the C ABI twice in a row and compares both results with
the context-based entry point pamtra_b200_run.
"""
import copy
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
    """Two calls in a row agree with pamtra_b200_run.  The allocation-free
    calls come first, so in a fresh process they run before any library
    context exists on the device: the entry point needs none.  The second
    call must leave both torch's allocator and the device's free memory
    unchanged (the first call is the per-device set-up)."""
    import torch
    b, arrs, sp_dev, dev = _device_inputs()
    lib = native.load()
    cols = b.columns(arrs)
    cols.species = sp_dev.data_ptr()  # device pointer on this entry point
    outs = [b.alloc_outputs(dev) for _ in range(2)]
    torch.cuda.synchronize()
    for i, out in enumerate(outs):
        o = native.Engine.make_outputs(out)
        if i == 1:
            alloc0, resv0 = torch.cuda.memory_allocated(dev), torch.cuda.memory_reserved(dev)
            free0, _ = torch.cuda.mem_get_info(dev)
        rc = lib.pamtra_b200_run_noalloc(ctypes.byref(b.settings), ctypes.byref(cols), ctypes.byref(o), None)
        assert rc == 0
        torch.cuda.synchronize()
        if i == 1:
            assert torch.cuda.memory_allocated(dev) == alloc0
            assert torch.cuda.memory_reserved(dev) == resv0
            assert torch.cuda.mem_get_info(dev)[0] == free0

    eng = native.engine(0)
    ref = b.alloc_outputs(dev)
    eng.run(b.settings, b.columns(arrs), eng.make_outputs(ref))
    torch.cuda.synchronize()
    tb_ref = ref["tb"].cpu().numpy()
    assert int(ref["status"].abs().sum()) == 0
    for out in outs:
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
    # a quadrature wider than the output rows (max_nummu) would write past
    # the caller's buffers: rejected before anything is launched
    cols.ncol = 1
    cols.max_nummu = 8
    assert b.settings.nummu == 16
    assert lib.pamtra_b200_run_noalloc(ctypes.byref(b.settings), ctypes.byref(cols), ctypes.byref(o), None) == \
        (2 | native.ST_SIZE)
    st8 = copy.copy(b.settings)
    st8.nummu = 8
    cols.nummu_mask = 2  # N = 16 launched with 8-angle output rows
    assert lib.pamtra_b200_run_noalloc(ctypes.byref(st8), ctypes.byref(cols), ctypes.byref(o), None) == \
        (2 | native.ST_SIZE)
    cols.nummu_mask = 4  # N = 32 is beyond this entry point
    cols.max_nummu = 32
    assert lib.pamtra_b200_run_noalloc(ctypes.byref(st8), ctypes.byref(cols), ctypes.byref(o), None) == \
        (2 | native.ST_SIZE)
    torch.cuda.synchronize()
