"""Host-side logic of the request loop (no GPU): staging-buffer bounds,
overlap detection of device intervals, the seeded request stream."""
import numpy as np

from pamtra_b200 import batch as pbatch
from pamtra_b200 import serve


def _bytes(b):
    """Input and output bytes of a batch as the server lays them out."""
    ins = [(k, v.nbytes) for k, v in b.host.items() if isinstance(v, np.ndarray)]
    outs = [(k, int(np.prod(s)) * np.dtype(dt).itemsize) for k, (s, dt) in b.output_shapes().items()]
    return serve._layout(ins)[1], serve._layout(outs)[1]


def test_staging_bound_covers_merged_batches():
    reqs = serve.request_stream(6, seed=60, max_cols=12, nfreq_range=(1, 32))
    for r in reqs:
        b_in, b_out = _bytes(r)
        cap_in, cap_out = serve.batch_bytes_bound(r.ncol)
        assert b_in <= cap_in and b_out <= cap_out
    merged, _ = pbatch.concat([r for r in reqs if r.max_nummu == reqs[0].max_nummu])
    b_in, b_out = _bytes(merged)
    cap_in, cap_out = serve.batch_bytes_bound(merged.ncol)
    assert b_in <= cap_in and b_out <= cap_out


def test_layout_alignment():
    offs, total = serve._layout([("a", 3), ("b", 300), ("c", 1)])
    assert offs == {"a": 0, "b": 256, "c": 768} and total == 769


def test_overlapping_pairs():
    iv = [(0, 0.0, 10.0, 5), (1, 5.0, 12.0, 5), (0, 11.0, 20.0, 5), (2, 30.0, 31.0, 1)]
    pairs = serve.overlapping_pairs(iv)
    # same-slot intervals never count; (0,1) overlap 5 ms, (1,2) overlap 1 ms
    assert [(i, j) for i, j, _ in pairs] == [(0, 1), (1, 2)]
    assert [round(o, 6) for _, _, o in pairs] == [5.0, 1.0]


def test_loguniform_request_sizes():
    reqs = serve.request_stream(40, seed=61, max_cols=512, nfreq_range=(1, 2), sizes="loguniform")
    cols = np.array([r.ncol for r in reqs])
    assert cols.min() >= 1 and cols.max() <= 512
    assert np.median(cols) < 128  # many small requests
    for r in reqs:
        assert len(set(np.asarray(r.host["nummu"]).tolist())) == 1  # one NUMMU per request
