"""Serving loop on the GPU: every request's result is the same served alone
and served in a mix of concurrent requests (merged batches, chunked
requests, overlapping slots).  Tolerance: 0 K (bit-identical), since a
(column, frequency) solve never reads another column's data."""
import numpy as np
import pytest

from pamtra_b200 import batch as pbatch
from pamtra_b200 import serve

pytestmark = pytest.mark.gpu


def _alone(b, precision=0):
    import torch
    out = pbatch.run(b, 0, precision=precision)
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


# the reference-order FP64 form and the split-precision form, whose kernels
# pair items and units of different columns inside one CTA (the pairs change
# with the mix)
@pytest.mark.parametrize("precision", [0, 1])
def test_results_same_alone_and_in_mix(native, precision):
    reqs = serve.request_stream(7, seed=50, max_cols=24, nfreq_range=(1, 6))
    alone = [_alone(b, precision) for b in reqs]
    # small arenas force chunking of the larger requests and merging of the small ones
    srv = serve.Server(0, slots=3, arena_bytes=192 << 20, max_cols=48, precision=precision)
    try:
        served = [srv.submit(b) for b in reqs]
        assert srv.drain(timeout=300)
    finally:
        srv.close()
    chunked = sum(1 for r in served if r._parts is not None)
    assert chunked >= 1
    for r, a in zip(served, alone):
        assert r.error is None, r.error
        assert np.array_equal(r.result["tb"], a["tb"])
        assert np.array_equal(r.result["status"], a["status"])
        assert r.latency > 0


def test_plain_server_matches(native):
    reqs = serve.request_stream(2, seed=51, max_cols=4, nfreq_range=(1, 3))
    alone = [_alone(b) for b in reqs]
    srv = serve.Server(0, slots=1, arena_bytes=256 << 20, max_cols=1)
    try:
        served = [srv.submit(b) for b in reqs]
        assert srv.drain(timeout=300)
    finally:
        srv.close()
    assert srv.batches_launched == sum(b.ncol for b in reqs)
    for r, a in zip(served, alone):
        assert np.array_equal(r.result["tb"], a["tb"])


def test_slots_overlap_on_device(native):
    """Batches of different slots are in flight on the device at the same
    time: their CUDA-event intervals (recorded on each slot's stream around
    the library call, measured from one common origin event) overlap."""
    reqs = serve.request_stream(6, seed=52, max_cols=96, nfreq_range=(12, 16))
    srv = serve.Server(0, slots=3, arena_bytes=512 << 20, max_cols=96)
    try:
        served = [srv.submit(b) for b in reqs]
        assert srv.drain(timeout=300)
    finally:
        srv.close()
    assert all(r.error is None for r in served)
    assert len({iv[0] for iv in srv.intervals}) >= 2  # more than one slot took work
    pairs = serve.overlapping_pairs(srv.intervals)
    assert pairs, srv.intervals
    assert max(ov for _, _, ov in pairs) > 0.1  # ms


def test_staging_buffers_are_reused(native):
    # the second batch on a slot writes into the same device buffers
    reqs = serve.request_stream(2, seed=53, max_cols=8, nfreq_range=(1, 3))
    srv = serve.Server(0, slots=1, arena_bytes=256 << 20, max_cols=8)
    try:
        d_in, d_out = srv.slots[0].d_in.data_ptr(), srv.slots[0].d_out.data_ptr()
        a = srv.submit(reqs[0])
        assert srv.drain(timeout=300)
        b = srv.submit(reqs[1])
        assert srv.drain(timeout=300)
        assert srv.slots[0].d_in.data_ptr() == d_in and srv.slots[0].d_out.data_ptr() == d_out
    finally:
        srv.close()
    for r, bt in ((a, reqs[0]), (b, reqs[1])):
        assert np.array_equal(r.result["tb"], _alone(bt)["tb"])
