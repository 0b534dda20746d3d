"""Failure reporting without a GPU fault.

* Bounded waits on the tensor core: with a wait limit of 0 polls every wait
  of the split-precision layer kernels on an MMA gives up at once.  The run
  must return normally, every (column, frequency) whose layers needed an MMA
  must carry ST_TIMEOUT, and the next run on the same context with the
  default limit must give the batched FP64 result within the split-precision
  tolerance (the timed-out CTAs drained their last MMA and freed their tensor
  memory).  The reference has no device waits; its errors are the status
  codes of src/report_module.f90:11-14.
* A column whose quadrature no kernel of the run solves (per-column NUMMU
  not among the launched ones) reports FATAL | ST_SIZE instead of a silent
  -9999.
"""
import copy

import numpy as np
import pytest

from pamtra_b200 import batch as pbatch
from pamtra_b200 import workloads as wl
from pamtra_b200._native import (PREC_3XTF32, PREC_FP64_BATCHED, ST_SIZE, ST_TIMEOUT, WAIT_LIMIT_DEFAULT)

pytestmark = pytest.mark.gpu
SPLIT_TOL = 0.05  # K, split precision against FP64


def test_zero_wait_limit_reports_timeouts_and_context_recovers(native):
    import torch
    dev = torch.device("cuda", 0)
    b = wl.uneven_batch(12, seed=21, nummu_choices=(16, 32), nfreq_range=(2, 3))
    eng = native.Engine(0)  # a context of its own
    ref = b.alloc_outputs(dev, ssp=True)
    pbatch.run(b, 0, ref, precision=PREC_FP64_BATCHED, eng=eng)
    torch.cuda.synchronize()
    assert int(ref["status"].abs().sum()) == 0
    nd = ref["num_doubles"].cpu().numpy()          # [C][F][L], -1 = no hydrometeors
    needs_mma = np.any(nd > 0, axis=2)             # (column, frequency) with a doubled layer

    eng.set_wait_limit(0)
    out = b.alloc_outputs(dev)
    pbatch.run(b, 0, out, precision=PREC_3XTF32, eng=eng)  # raises if the call itself failed
    torch.cuda.synchronize()
    st = out["status"].cpu().numpy()
    assert needs_mma.any()
    assert np.all(st[needs_mma] & ST_TIMEOUT)
    assert np.all(st[needs_mma] & 2)

    eng.set_wait_limit(WAIT_LIMIT_DEFAULT)
    again = b.alloc_outputs(dev)
    pbatch.run(b, 0, again, precision=PREC_3XTF32, eng=eng)
    torch.cuda.synchronize()
    assert int(again["status"].abs().sum()) == 0
    tb, tr = again["tb"].cpu().numpy(), ref["tb"].cpu().numpy()
    ok = tr > -9000
    assert np.array_equal(tb > -9000, ok)
    assert np.max(np.abs(tb[ok] - tr[ok])) < SPLIT_TOL
    eng.close()


def test_unlaunched_quadrature_is_reported(native):
    # every column asks for NUMMU 32, the run launches NUMMU 16 only
    import torch
    dev = torch.device("cuda", 0)
    b = wl.uneven_batch(3, seed=22, nummu_choices=(32,), nfreq_range=(2, 3))
    assert b.nummu_mask == 4 and b.max_nummu == 32
    eng = native.engine(0)
    arrs = b.device_arrays(dev)
    cols = b.columns(arrs)
    cols.nummu_mask = 0  # = settings.nummu only
    st = copy.copy(b.settings)
    st.nummu = 16
    out = b.alloc_outputs(dev)
    eng.run(st, cols, eng.make_outputs(out), PREC_FP64_BATCHED)
    torch.cuda.synchronize()
    status = out["status"].cpu().numpy()
    nf = b.host["nfreq"]
    for c in range(b.ncol):
        assert np.all(status[c, :nf[c]] == (2 | ST_SIZE))
        assert np.all(out["tb"].cpu().numpy()[c] == -9999.0)
