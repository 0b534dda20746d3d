"""Host-side logic of the batched form and the serving loop (no GPU):
packing of per-column batches, merging and splitting, chunking by scratch
size, and the scheduler's packing policy."""
import collections
import warnings

import numpy as np
import pytest

from pamtra_b200 import batch as pbatch
from pamtra_b200 import libWrapper, packing, serve
from pamtra_b200 import workloads as wl
from pamtra_b200._native import workspace_bytes

pytestmark = pytest.mark.usefixtures("native")  # workspace sizes come from the library (no device needed)


def _need(b):
    return workspace_bytes(b.columns(b.host))


def test_present_bound_matches_facade_helper():
    warnings.simplefilter("ignore")
    pam = wl.c2_pam(16, seed=9)
    b = pbatch.pack_pam(pam, wl.C2_FREQS)
    cols = packing.profile_columns(pam.p, 2)
    assert b.max_present == libWrapper.present_bound(cols, pam.df.data)
    assert pbatch.present_layers(b.host, b.species, 0) == int(np.sum(pbatch.present_per_column(b.host, b.species, 0)))


def test_uneven_batch_shapes():
    b = wl.uneven_batch(40, seed=21)
    h = b.host
    assert b.species_stride == 5 and len(b.species) == 40 * 5
    assert np.all((h["nlyrs"] >= 40) & (h["nlyrs"] <= 150))
    assert np.all((h["nfreq"] >= 8) & (h["nfreq"] <= 32))
    assert set(np.unique(h["nummu"])) <= {8, 16, 32}
    for c in range(40):
        nf = h["nfreq"][c]
        f = h["freqs"][c, :nf]
        assert np.all(np.diff(f) > 0) and f[0] >= 10.0 and f[-1] <= 183.0
        sp = b.species[c * 5:(c + 1) * 5]
        on = sp["dist"] != packing.DIST_CODES["disabled"]
        assert 1 <= on.sum() <= 5
        assert np.all((sp["nbin"][on] >= 20) & (sp["nbin"][on] <= 80))
        ice = on & (sp["liq_ice"] == -1)
        assert np.all((sp["rho_ms"][ice] >= 100.0) & (sp["rho_ms"][ice] <= 900.0))
        # no hydrometeor input in disabled slots
        assert np.all(h["hydro_q"][c, :, ~on] == 0.0)


def test_subset_keeps_columns():
    b = wl.uneven_batch(12, seed=22)
    idx = [7, 2, 9]
    s = pbatch.subset(b, idx)
    assert s.ncol == 3
    L = int(s.host["max_nlyrs"])
    F = int(s.host["max_nfreq"])
    assert L == max(b.host["nlyrs"][idx]) and F == max(b.host["nfreq"][idx])
    for j, c in enumerate(idx):
        nl = b.host["nlyrs"][c]
        assert np.array_equal(s.host["temp_lev"][j, :nl + 1], b.host["temp_lev"][c, :nl + 1])
        assert np.array_equal(s.host["hydro_q"][j], b.host["hydro_q"][c, :L])
        assert np.array_equal(s.host["freqs"][j], b.host["freqs"][c, :F])
        assert s.species[j * 5:(j + 1) * 5].tobytes() == b.species[c * 5:(c + 1) * 5].tobytes()
    assert s.max_present == int(np.sum(pbatch.present_per_column(b.host, b.species, 5)[idx]))


def test_chunks_cover_once_and_fit():
    b = wl.uneven_batch(48, seed=23)
    budget = 600 << 20
    chunks = pbatch.chunk_columns(b, budget)
    allc = np.concatenate(chunks)
    assert sorted(allc.tolist()) == list(range(48))
    for ch in chunks:
        s = pbatch.subset(b, ch)
        assert _need(s) <= budget
        assert len(np.unique(b.host["nummu"][ch])) == 1  # one NUMMU per chunk
    with pytest.raises(MemoryError):
        pbatch.chunk_columns(b, 1 << 20)


def test_concat_and_split_roundtrip():
    a = wl.uneven_batch(3, seed=24, nummu_choices=(8,), nfreq_range=(2, 3))
    b = pbatch.pack_pam(wl.c2_pam(2, seed=25), wl.C2_FREQS)
    c = wl.uneven_batch(4, seed=26, nummu_choices=(32,), nfreq_range=(5, 6))
    m, starts = pbatch.concat([a, b, c])
    assert starts == [0, 3, 5] and m.ncol == 9
    assert m.max_nummu == 32 and m.nummu_mask == 1 | 2 | 4
    assert list(m.host["nummu"]) == [8] * 3 + [16] * 2 + [32] * 4
    # b had 2 species shared by all columns: padded to 5 with disabled slots
    sp = m.species.reshape(9, 5)
    assert sp[3, 0].tobytes() == b.species[0].tobytes() and sp[4, 1].tobytes() == b.species[1].tobytes()
    assert np.all(sp[3:5, 2:]["dist"] == packing.DIST_CODES["disabled"])
    assert np.array_equal(m.host["freqs"][3, :4], wl.C2_FREQS)
    assert m.max_present == a.max_present + b.max_present + c.max_present
    # fake merged outputs tagged by column / angle / frequency
    shp = m.output_shapes()
    outs = {k: np.zeros(s_, dtype=dt) for k, (s_, dt) in shp.items()}
    C, NO, NA, F, _ = shp["tb"][0]
    outs["tb"][:] = (np.arange(C)[:, None, None, None, None] * 1e4 + np.arange(NA)[None, None, :, None, None] * 100
                     + np.arange(F)[None, None, None, :, None])
    parts = pbatch.split_outputs(outs, [a, b, c], starts)
    for part, bb, c0 in zip(parts, [a, b, c], starts):
        assert part["tb"].shape == bb.output_shapes()["tb"][0]
        assert part["tb"][0, 0, 1, 1, 0] == c0 * 1e4 + 100 + 1


def test_pack_units_policy():
    warnings.simplefilter("ignore")
    reqs = [wl.uneven_batch(n, seed=30 + i, nummu_choices=(N,), nfreq_range=(2, 4))
            for i, (n, N) in enumerate([(3, 16), (2, 8), (4, 16), (2, 16), (5, 8)])]
    units = collections.deque(serve._Unit(serve.Request(i, b, 0.0), b) for i, b in enumerate(reqs))
    big = 1 << 40
    take = serve.pack_units(units, big, 100, _need)
    # oldest first; same NUMMU joins, NUMMU 8 units stay queued in order
    assert [u.req.id for u in take] == [0, 2, 3]
    assert [u.req.id for u in units] == [1, 4]
    # column cap
    units = collections.deque(serve._Unit(serve.Request(i, b, 0.0), b) for i, b in enumerate(reqs))
    take = serve.pack_units(units, big, 6, _need)
    assert [u.req.id for u in take] == [0, 3]
    # arena: a merged batch that does not fit leaves the candidate queued
    units = collections.deque(serve._Unit(serve.Request(i, b, 0.0), b) for i, b in enumerate(reqs))
    arena = _need(reqs[0]) + 1
    take = serve.pack_units(units, arena, 100, _need)
    assert [u.req.id for u in take] == [0]
    assert [u.req.id for u in units] == [1, 2, 3, 4]


def test_split_request_and_assemble():
    b = wl.uneven_batch(10, seed=40, nfreq_range=(2, 3))
    r = serve.Request(0, b, 0.0)
    units = serve.split_request(r, 200 << 20, 4, _need)
    assert len(units) >= 3 and r._left == len(units)
    assert sorted(np.concatenate([u.cols for u in units]).tolist()) == list(range(10))
    parts = []
    for u in units:
        shp = u.batch.output_shapes()
        o = {k: np.zeros(s_, dtype=dt) for k, (s_, dt) in shp.items()}
        o["tb"][:] = u.cols[:, None, None, None, None]
        parts.append((u.cols, u.batch, o))
    full = serve._assemble(b, parts)
    for c in range(10):
        N, nf = b.host["nummu"][c], b.host["nfreq"][c]
        assert np.all(full["tb"][c, :, :2 * N, :nf] == c)


def test_latency_stats_and_arrivals():
    t = serve.poisson_arrivals(2000, 200.0, seed=1)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 200.0) < 20.0

    class R(object):
        def __init__(self, lat):
            self.latency = lat
    st = serve.latency_stats([R(x / 1000.0) for x in range(1, 101)])
    assert abs(st["p50_ms"] - 50.5) < 1e-9 and abs(st["p99_ms"] - 99.01) < 1e-9


def test_bench_oracle_sample_prefers_cheap_columns():
    import bench
    b = wl.uneven_batch(64, seed=62, nfreq_range=(2, 9))
    idxs = bench.oracle_sample(b, 8)
    assert len(idxs) == 8 and idxs == sorted(set(idxs))
    nmu = np.asarray(b.host["nummu"])
    assert {8, 16, 32} & set(nmu[idxs].tolist()) == set(np.unique(nmu).tolist()) & {8, 16, 32}


def test_split_adding_workspace():
    # the split adding (PREC_3XTF32, NUMMU 16) adds one FP32 stack record of
    # 4224 floats per (column, frequency) unit to the plan; the split
    # doubling with the FP64 adding and the FP64 forms need none
    from pamtra_b200._native import PREC_3XTF32, PREC_3XTF32_FP64ADD, PREC_FP64_BATCHED
    b = pbatch.pack_pam(wl.c2_pam(16, seed=5), wl.C2_FREQS)
    cols = b.columns(b.host)
    w1 = workspace_bytes(cols, precision=PREC_3XTF32)
    w3 = workspace_bytes(cols, precision=PREC_3XTF32_FP64ADD)
    w2 = workspace_bytes(cols, precision=PREC_FP64_BATCHED)
    assert w1 - w3 == 16 * len(wl.C2_FREQS) * 4224 * 4
    assert w3 < w2  # FP32 Legendre coefficients in the split forms
