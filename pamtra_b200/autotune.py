"""Launch-shape autotuner of the batched form.

The persistent kernels take their work from device counters, so any launch
shape gives the same results; only the speed differs with the batch's mix of
layers, species, bins and frequencies.  For a batch signature (NUMMU set,
precision, and power-of-two buckets of columns, layers, frequencies and
species) the tuner times candidate shapes with the library's per-stage CUDA
events and keeps, stage by stage, the fastest:

* Mie: warps per CTA (2, 4, 8), CTAs per SM, and the tile of its
  phase-function sums (size bins per work item: 4 or 8, two compiled
  instantiations of the kernel),
* layer doubling: CTAs per SM (FP64 teams, or item pairs of the
  split-precision kernel),
* adding: CTAs per SM,

The stages are separate kernels, so one timed run per candidate row measures
one option of every stage at once.  Choices are cached per signature in
memory and, when ``PAMTRA_B200_TUNE_CACHE`` names a file, in JSON there.

:func:`tune_columns` picks the serving batch size: the smallest column count
whose throughput reaches ``frac`` of the best measured.

The reference has no counterpart (its Fortran runs on CPU processes,
python/pyPamtra/core.py:1570-1676).
"""

import json
import os

import numpy as np

from ._native import PREC_FP64, engine

# candidate rows: (mie warps, mie CTAs/SM, layer CTAs/SM, adding CTAs/SM, mie bins per work
# item); 0 = as many as fit (CTAs) or the default (warps, bins)
CANDIDATES = [
    (4, 0, 0, 0, 4),
    (8, 0, 1, 1, 8),
    (2, 0, 2, 0, 4),
    (4, 2, 3, 1, 8),
    (8, 1, 0, 0, 4),
    (4, 0, 0, 2, 8),
]
STAGE_KNOBS = {"mie": (0, 1, 4), "layer": (2,), "adding": (3,)}
DEFAULT = (4, 0, 0, 0, 4)

_cache = {}


def _bucket(v):
    v = max(int(v), 1)
    return 1 << (v - 1).bit_length()


def signature(batch, precision=PREC_FP64):
    h = batch.host
    return "m%d_p%d_c%d_l%d_f%d_h%d" % (batch.nummu_mask, int(precision), _bucket(batch.ncol),
                                          _bucket(int(h["max_nlyrs"])), _bucket(int(h["max_nfreq"])),
                                          int(h["nhydro"]))


def _load_file():
    path = os.environ.get("PAMTRA_B200_TUNE_CACHE")
    if path and os.path.exists(path):
        try:
            with open(path) as f:
                for k, v in json.load(f).items():
                    _cache.setdefault(k, tuple(v))
        except (OSError, ValueError):
            pass


def _save_file():
    path = os.environ.get("PAMTRA_B200_TUNE_CACHE")
    if path:
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump({k: list(v) for k, v in _cache.items()}, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def lookup(batch, precision=PREC_FP64):
    """Cached launch shape for the batch's signature, or None."""
    if not _cache:
        _load_file()
    return _cache.get(signature(batch, precision))


def tune(batch, device=0, precision=PREC_FP64, stream=None, eng=None, reps=2, candidates=None, outputs=None):
    """Time the candidate launch shapes on ``batch`` (inputs resident on the
    device), set the fastest on the engine and return (shape, report), where
    report maps each stage to its per-candidate milliseconds."""
    import torch
    from . import batch as pbatch
    eng = eng or engine(device)
    cands = list(candidates or CANDIDATES)
    out = outputs if outputs is not None else batch.alloc_outputs(torch.device("cuda", device))
    old = eng.get_launch()
    eng.set_launch(DEFAULT)
    pbatch.run(batch, device, out, precision=precision, stream=stream, eng=eng)  # warm-up: arena, tables
    times = np.zeros((len(cands), len(STAGE_KNOBS)))
    eng.set_timing(True)
    try:
        for i, c in enumerate(cands):
            eng.set_launch(c)
            acc = {}
            for _ in range(reps):
                pbatch.run(batch, device, out, precision=precision, stream=stream, eng=eng)
                for k, v in eng.stage_ms().items():
                    acc[k] = acc.get(k, 0.0) + v / reps
            times[i] = [acc.get(k, 0.0) for k in STAGE_KNOBS]
    finally:
        eng.set_timing(False)
        eng.set_launch(old)
    best = list(DEFAULT)
    for j, (stage, knobs) in enumerate(STAGE_KNOBS.items()):
        i = int(np.argmin(times[:, j]))
        for kn in knobs:
            best[kn] = cands[i][kn]
    best = tuple(best)
    _cache[signature(batch, precision)] = best
    _save_file()
    eng.set_launch(best)
    report = {stage: [float(times[i, j]) for i in range(len(cands))] for j, stage in enumerate(STAGE_KNOBS)}
    return best, report


def apply(batch, device=0, precision=PREC_FP64, eng=None, **kw):
    """Set the cached shape for this batch's signature, tuning it first if
    there is none."""
    eng = eng or engine(device)
    shape = lookup(batch, precision)
    if shape is None:
        shape, _ = tune(batch, device, precision, eng=eng, **kw)
    else:
        eng.set_launch(shape)
    return shape


def tune_columns(make_batch, sizes, device=0, precision=PREC_FP64, eng=None, frac=0.9, reps=2):
    """Serving batch size: time ``make_batch(ncol)`` for each size and return
    (chosen size, {size: solves/s}), the smallest size within ``frac`` of the
    best throughput (larger batches add latency for little gain)."""
    import torch
    from . import batch as pbatch
    eng = eng or engine(device)
    rate = {}
    for n in sizes:
        b = make_batch(n)
        out = b.alloc_outputs(torch.device("cuda", device))
        pbatch.run(b, device, out, precision=precision, eng=eng)
        torch.cuda.synchronize(device)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            pbatch.run(b, device, out, precision=precision, eng=eng)
        e.record()
        e.synchronize()
        rate[n] = b.n_solves() * reps / (s.elapsed_time(e) * 1e-3)
        del out
    top = max(rate.values())
    chosen = min(n for n, r in rate.items() if r >= frac * top)
    return chosen, rate
