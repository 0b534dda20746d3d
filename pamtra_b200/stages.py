"""Per-stage device times of the batched forward path on the seeded workloads.

``python -m pamtra_b200.stages [--workload c2|target|uneven|mieheavy] [--ncol N]
[--precision fp64|fp64b|3xtf32|3xtf32d|both|all] [--reps K]`` runs one untimed and
K timed batches per precision (fp64: the reference operation order, fp64b:
the batched FP64 form, 3xtf32: the split-precision form, 3xtf32d: its
doubling with the FP64 adding) through
:func:`pamtra_b200.batch.run` and prints one JSON line per precision:
milliseconds per stage (CUDA events the library records between its kernels
on the run's stream), the number of (layer, frequency) items and their mean
doubling count, and the largest TB difference from the first precision.  It is the command the kernel profiles
are taken with (under ``ncu -k <kernel> -s 1 -c 1``: launch 0 of each
kernel is the untimed batch, launch 1 the first timed one).
"""

import argparse
import json
import warnings


def _batch(name, ncol, nummu=None):
    from . import batch as pbatch
    from . import workloads as wl
    if name == "c2":
        return pbatch.pack_pam(wl.c2_pam(ncol, seed=2), wl.C2_FREQS)
    if name == "target":
        return wl.target_batch(ncol, seed=4)
    if name == "uneven":
        return wl.uneven_batch(ncol, seed=3, nummu_choices=(nummu,) if nummu else (8, 16, 32))
    if name == "mieheavy":
        return wl.mie_heavy_batch(ncol, seed=6)
    raise ValueError("unknown workload %r" % name)


def run(name, ncol, precisions, reps, device=0, nummu=None):
    import numpy as np
    import torch

    from . import batch as pbatch
    from ._native import Engine
    eng = Engine(device)
    b = _batch(name, ncol, nummu)
    stream = torch.cuda.Stream(torch.device("cuda", device))
    lines, tbs = [], []
    for prec in precisions:
        out = b.alloc_outputs(torch.device("cuda", device), ssp=True)
        with torch.cuda.stream(stream):
            pbatch.run(b, device, out, precision=prec, stream=stream, eng=eng)
        stream.synchronize()
        eng.set_timing(True)
        tot = {}
        for _ in range(reps):
            with torch.cuda.stream(stream):
                pbatch.run(b, device, out, precision=prec, stream=stream, eng=eng)
            for k, v in eng.stage_ms().items():
                tot[k] = tot.get(k, 0.0) + v / reps
        eng.set_timing(False)
        nd = out["num_doubles"].cpu().numpy()
        d = nd[nd > 0]
        tbs.append(out["tb"].cpu().numpy())
        lines.append({"workload": name, "columns": b.ncol, "precision": ["fp64", "3xtf32", "fp64_batched", "3xtf32_fp64add"][prec],
                      "stage_ms": tot, "items": int(np.count_nonzero(nd >= 0)),
                      "doublings_mean": float(d.mean()) if d.size else 0.0,
                      "status_nonzero": int((out["status"] != 0).sum())})
    for ln, tb in zip(lines[1:], tbs[1:]):
        ln["tb_max_diff_vs_%s_K" % lines[0]["precision"]] = float(np.max(np.abs(tb - tbs[0])))
    eng.close()
    return lines


def main(argv=None):
    warnings.simplefilter("ignore")
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--workload", default="c2", choices=["c2", "target", "uneven", "mieheavy"])
    ap.add_argument("--ncol", type=int, default=256)
    ap.add_argument("--precision", default="both", choices=["fp64", "3xtf32", "fp64b", "3xtf32d", "both", "all"])
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--nummu", type=int, default=0, choices=[0, 8, 16, 32], help="uneven workload: one NUMMU only")
    a = ap.parse_args(argv)
    precs = {"fp64": [0], "3xtf32": [1], "fp64b": [2], "3xtf32d": [3], "both": [0, 1], "all": [0, 2, 1, 3]}[a.precision]
    for ln in run(a.workload, a.ncol, precs, a.reps, nummu=a.nummu or None):
        print(json.dumps(ln))


if __name__ == "__main__":
    main()
