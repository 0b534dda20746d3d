#!/usr/bin/env python
"""Benchmark of the B200 passive forward path.

Metric: column x frequency solves per second (one solve = gas + PSD + Mie +
scatcnv + RT4 + TB for one column at one frequency).

Default workload (the batched FP64 configuration): 4096 seeded columns of 50
layers over 0-12 km, cloud liquid (exp, 40 bins) and rain (Marshall-Palmer,
50 bins) in layers 5-25 with mixing ratios log-uniform over 0.01-2 g/kg,
frequencies 23.8, 31.4, 89 and 150 GHz, NUMMU = 16, FP64.

  value  : batched FP64 form (PREC_FP64_BATCHED: one inverse per adding
           combine) in solves/s with inputs resident in HBM (device-timed,
           CUDA events on the launching stream, L2 flushed between steps),
           launch shapes from the autotuner
  e2e    : same metric through the C ABI with host buffers (pinned), the
           host<->device copies inside the timed region
  plain  : the plain form (one column per call, the reference operation
           order PREC_FP64) on a sample of columns
  split_3xtf32 / target_shape / serving / graph_replay: the split-precision
           form, the 150-layer 4-species shape, the request loop and the
           CUDA-graph replay of the same step

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Under torchrun each rank runs its own columns (weak scaling, no collective on
the data path); rank 0 prints one JSON line.
"""

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FREQS = [23.8, 31.4, 89.0, 150.0]
METRIC = "column*freq solves/s"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ncol", type=int, default=4096)
    ap.add_argument("--cpu-sample", type=int, default=0, help="columns for the CPU baseline (0 = 2 per core)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=200, help="requests in the serving replay (0 = skip)")
    ap.add_argument("--serve-plain", type=int, default=30, help="requests of the stream served by the plain form")
    ap.add_argument("--target-cols", type=int, default=1024, help="columns of the 150-layer target batch (0 = skip)")
    ap.add_argument("--uneven-cols", type=int, default=16384, help="columns of the uneven batch (0 = skip)")
    ap.add_argument("--mieheavy-cols", type=int, default=2048, help="columns of the Mie-heavy batch (0 = skip)")
    ap.add_argument("--tmatrix-items", type=int, default=128,
                    help="(layer, frequency) items of 32 bins in the T-matrix line (0 = skip)")
    return ap.parse_args()


def _config(ncol):
    return {"workload": "batched FP64: %d columns x 50 layers (0-12 km), 2 Mie species (cloud exp 40 bins, "
                        "rain Marshall-Palmer 50 bins) in layers 5-25, q log-uniform 0.01-2 g/kg, "
                        "f = 23.8/31.4/89/150 GHz, NUMMU=16" % ncol,
            "columns_per_gpu": ncol, "layers": 50, "frequencies": FREQS, "nummu": 16,
            "l2": "flushed between timed steps (256 MiB write)"}


# ---------------------------------------------------------------- CPU baseline
def _oracle_chunk(task):
    st_fields, species, cols, idxs, freqs = task
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    st = oracle.OrcSettings(**st_fields)
    out = []
    t0 = time.perf_counter()
    for c in idxs:
        err, tb, _, _, _ = oracle.run_column(st, species, cols, c, freqs)
        out.append((c, err, tb))
    return out, time.perf_counter() - t0


def _oracle_packed(task):
    """Oracle TB of columns of a small packed batch with per-column NUMMU,
    frequency lists and species (the worker side of oracle_tb_errors)."""
    st_fields, species, stride, host, cols = task
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    out = []
    H = int(host["nhydro"])
    for c in cols:
        st = oracle.OrcSettings(**st_fields)
        if host.get("nummu") is not None:
            st.nummu = int(host["nummu"][c])
        sp = species[c * H:(c + 1) * H] if stride else species
        freqs = list(host["freqs"][c, :int(host["nfreq"][c])]) if host.get("nfreq") is not None \
            else list(host["freqs"])
        err, tb, _, _, _ = oracle.run_column(st, sp, host, c, freqs)
        out.append((c, err, tb, int(st.nummu), len(freqs)))
    return out


def oracle_sample(b, k=8):
    """Columns of ``b`` for the oracle check: the cheapest ones of each NUMMU
    (CPU cost ~ N^3 x layers x frequencies), up to ``k`` in all."""
    h = b.host
    C = b.ncol
    nmu = np.asarray(h["nummu"]) if h.get("nummu") is not None else np.full(C, b.max_nummu)
    nf = np.asarray(h["nfreq"]) if h.get("nfreq") is not None else np.full(C, int(h["max_nfreq"]))
    cost = nmu.astype(np.float64) ** 3 * np.asarray(h["nlyrs"]) * nf
    picks = []
    for N, quota in ((8, k // 2), (16, k // 4 + (k % 4 > 0)), (32, max(1, k // 8))):
        cand = np.nonzero(nmu == N)[0]
        picks += cand[np.argsort(cost[cand])][:quota].tolist()
    if len(picks) < k:
        rest = [int(c) for c in np.argsort(cost) if int(c) not in picks]
        picks += rest[:k - len(picks)]
    return sorted(picks[:k])


def oracle_tb_errors(b, idxs, tbs, pool):
    """Max |TB - oracle TB| (K) over the columns ``idxs`` for each TB array
    in ``tbs`` (name -> [C][nout][2N][F][2]); one oracle task per column."""
    from pamtra_b200 import batch as pbatch
    sub = pbatch.subset(b, idxs)
    st_fields = {k: getattr(b.settings, k) for k, _ in b.settings._fields_}
    tasks = [(st_fields, sub.species, sub.species_stride, sub.host, [j]) for j in range(len(idxs))]
    res = pool.map(_oracle_packed, tasks)
    errs = {name: 0.0 for name in tbs}
    bad = 0
    for out in res:
        for j, err, tb, N, nf in out:
            if err:
                bad += 1
                continue
            c = idxs[j]
            for name, t in tbs.items():
                errs[name] = max(errs[name], float(np.max(np.abs(t[c][:, :2 * N, :nf, :] - tb))))
    return errs, bad


def _tm_oracle_bin(task):
    """One bin of the T-matrix branch on the oracle (quad-precision solve,
    one core): the worker side of tmatrix_cpu_baseline."""
    nummu, freq, ref_re, ref_im, phase, arrs = task
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    t0 = time.perf_counter()
    r = oracle.tmatrix_species(nummu, freq, ref_re, ref_im, phase, *arrs)
    return time.perf_counter() - t0, r is not None


def tmatrix_cpu_baseline(pool, cores, bins, nummu=16, freq=89e9, ref=(1.78, -0.002), phase=-1, min_tasks=0):
    """All-core CPU figure of the T-matrix line: the given bins (dict of
    per-bin arrays dmax, del_d, ndens, density, as_ratio, canting), cycled to
    at least max(8 cores, min_tasks) single-bin tasks, one worker process per
    core (the process model of runParallelPamtra); returns (bins/s, tasks,
    wall seconds, all solved)."""
    keys = ("dmax", "del_d", "ndens", "density", "as_ratio", "canting")
    nb = len(bins["dmax"])
    ntask = max(nb, 8 * cores, min_tasks)
    tasks = [(nummu, freq, ref[0], ref[1], phase, [np.asarray(bins[k][i % nb:i % nb + 1], dtype=np.float64)
                                                   for k in keys]) for i in range(ntask)]
    t0 = time.perf_counter()
    res = pool.map(_tm_oracle_bin, tasks)
    wall = time.perf_counter() - t0
    return ntask / wall, ntask, wall, all(ok for _, ok in res)


def make_pool(cores):
    """Worker processes (spawned, so no CUDA state is inherited), warmed up
    outside any timed region."""
    import multiprocessing as mp
    pool = mp.get_context("spawn").Pool(cores)
    pool.map(_warm, range(cores))
    return pool


def _warm(_):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.lib()
    return 0


def cpu_model():
    """Host CPU model name (from /proc/cpuinfo)."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.lower().startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_single_core(batch, idxs, freqs):
    """The oracle on one host core (one worker, no pool) over ``idxs``:
    solves/s and wall seconds."""
    st_fields = {k: getattr(batch.settings, k) for k, _ in batch.settings._fields_}
    cols = {k: (v[idxs] if isinstance(v, np.ndarray) and v.ndim >= 1 and v.shape[0] == batch.ncol else v)
            for k, v in batch.host.items()}
    _oracle_chunk((st_fields, batch.species, cols, [0], freqs))  # warm-up: library load
    out, wall = _oracle_chunk((st_fields, batch.species, cols, list(range(len(idxs))), freqs))
    return len(idxs) * len(freqs) / wall, wall


def cpu_baseline(batch, idxs, freqs, cores, pool):
    """Time the oracle (C++ restatement of the reference) on host cores,
    one single-threaded worker per core (the reference's runParallelPamtra
    process model)."""
    st_fields = {k: getattr(batch.settings, k) for k, _ in batch.settings._fields_}
    cols = {k: (v[idxs] if isinstance(v, np.ndarray) and v.ndim >= 1 and v.shape[0] == batch.ncol else v)
            for k, v in batch.host.items()}
    local = list(range(len(idxs)))
    chunks = [local[i::cores] for i in range(cores)]
    tasks = [(st_fields, batch.species, cols, ch, freqs) for ch in chunks if ch]
    t0 = time.perf_counter()
    res = pool.map(_oracle_chunk, tasks)
    wall = time.perf_counter() - t0
    tbs = {}
    for out, _ in res:
        for c, err, tb in out:
            tbs[idxs[c]] = tb
    return len(idxs) * len(freqs) / wall, wall, tbs


# ---------------------------------------------------------------- clocks
class ClockSampler(object):
    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def fp64_peak_tflops(dev):
    """Measured FP64 throughput of cuBLAS DGEMM on this GPU (the roofline
    denominator for FP64 kernels; the driver's peak file carries bf16 only)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


# k_layer<16> DRAM traffic per (layer, frequency) item: ncu capture of the
# 256-column run (21,504 items): 17.7 MB read + 348.3 MB written per launch
LAYER_TRAFFIC_PER_ITEM = (17.698560e6 + 348.297472e6) / 21504


def layer_flops(nd, N):
    """Algorithmic FLOPs of the doubling stage: per scattering layer and
    frequency, each doubling is 6 n x n products and one inverse (2 n^3
    each), n = 2N."""
    n = 2 * N
    d = nd[nd > 0].astype(np.float64)
    return float(np.sum(d) * 7 * 2 * n ** 3)


def _timed_steps(b, local, eng, stream, out, prec, steps, warmup, flush):
    """Device-timed batched steps (CUDA events on the launching stream, L2
    flushed before each); returns per-step ms and mean stage ms."""
    import torch
    from pamtra_b200 import batch as pbatch
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            pbatch.run(b, local, out, precision=prec, stream=stream, eng=eng)
    stream.synchronize()
    eng.set_timing(True)
    ms, stages = [], {}
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            pbatch.run(b, local, out, precision=prec, stream=stream, eng=eng)
            e.record(stream)
        e.synchronize()
        ms.append(s.elapsed_time(e))
        for k, v in eng.stage_ms().items():
            stages[k] = stages.get(k, 0.0) + v / steps
    eng.set_timing(False)
    return ms, stages


def _target_shape(args, local, eng, stream):
    """The 150-layer, 16-angle, 4-species shape: batched FP64 over
    ``--target-cols`` columns (device-timed, L2 flushed) against the plain
    form (one column per call) on 16 of them."""
    import torch
    from pamtra_b200 import batch as pbatch
    from pamtra_b200.workloads import target_batch
    dev = torch.device("cuda", local)
    from pamtra_b200 import autotune
    b = target_batch(args.target_cols, seed=4)
    out = b.alloc_outputs(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    from pamtra_b200._native import PREC_FP64_BATCHED as BF
    autotune.tune(b, local, precision=BF, eng=eng, stream=stream, outputs=out)
    with torch.cuda.stream(stream):
        for _ in range(2):
            pbatch.run(b, local, out, precision=BF, stream=stream, eng=eng)
    stream.synchronize()
    ms = []
    for _ in range(3):
        with torch.cuda.stream(stream):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            pbatch.run(b, local, out, precision=BF, stream=stream, eng=eng)
            e.record(stream)
        e.synchronize()
        ms.append(s.elapsed_time(e))
    batched = b.n_solves() / (np.mean(ms) * 1e-3)
    st_bad = int((out["status"] != 0).sum())
    from pamtra_b200._native import PREC_3XTF32
    sout = b.alloc_outputs(dev)
    autotune.tune(b, local, precision=PREC_3XTF32, eng=eng, stream=stream, outputs=sout)
    sms_, sstages = _timed_steps(b, local, eng, stream, sout, PREC_3XTF32, 3, 2, flush)
    eng.set_launch(autotune.DEFAULT)
    split = b.n_solves() / (np.mean(sms_) * 1e-3)
    split_err = float((sout["tb"] - out["tb"]).abs().max().item())
    singles = [pbatch.subset(b, [c]) for c in range(16)]
    souts = [sb.alloc_outputs(dev) for sb in singles]
    with torch.cuda.stream(stream):
        for sb, so in zip(singles, souts):
            pbatch.run(sb, local, so, stream=stream, eng=eng)
    stream.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        s.record(stream)
        for sb, so in zip(singles, souts):
            pbatch.run(sb, local, so, stream=stream, eng=eng)
        e.record(stream)
    e.synchronize()
    plain = sum(sb.n_solves() for sb in singles) / (s.elapsed_time(e) * 1e-3)
    tb = out["tb"].cpu().numpy()
    plain_diff = max(float(np.max(np.abs(so["tb"].cpu().numpy()[0] - tb[c]))) for c, so in enumerate(souts))
    del flush
    return {"workload": "%d columns x 150 layers (0-15 km), NUMMU=16, 4 Mie species (cloud water, cloud ice, "
                        "snow, rain; 40 bins each), f = 23.8/31.4/89/150 GHz" % args.target_cols,
            "batched_fp64": batched, "plain_fp64": plain, "batched_over_plain": batched / plain,
            "batched_3xtf32": split, "batched_3xtf32_over_plain": split / plain,
            "tb_err_3xtf32_vs_fp64_K": split_err, "stage_ms_3xtf32": sstages,
            "unit": "solves/s", "batched_ms_per_step": float(np.mean(ms)), "status_nonzero": st_bad,
            "plain_sample_columns": 16, "plain_vs_batched_fp64_tb_max_diff_K": plain_diff,
            "forms": "batched FP64: one-inverse adding (PREC_FP64_BATCHED); plain: one column per call in the "
                     "reference operation order (PREC_FP64)"}


def _config_line(name, b, local, eng, stream, pool, nplain=8, reps=1, noracle=8):
    """Batched FP64 and split-precision solves/s on one workload at its
    stated size (default launch shapes, device-timed, L2 flushed) against the
    plain form (one column per call, reference order) on its first
    ``nplain`` columns, with the TB error of both batched forms against the
    oracle on ``noracle`` sampled columns.  A batch whose scratch exceeds a
    third of the free device memory runs as NUMMU-grouped chunks
    (batch.chunk_columns), one after another inside each timed step."""
    import torch
    from pamtra_b200 import autotune
    from pamtra_b200 import batch as pbatch
    from pamtra_b200._native import PREC_3XTF32, PREC_FP64_BATCHED
    dev = torch.device("cuda", local)
    eng.set_launch(autotune.DEFAULT)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    free, _ = torch.cuda.mem_get_info(dev)
    idx_chunks = pbatch.chunk_columns(b, free // 3)
    res = {"unit": "solves/s", "columns": b.ncol, "solves_per_step": b.n_solves(), "chunks": len(idx_chunks),
           "launch_shape": list(autotune.DEFAULT)}
    full = {}
    for label, prec in (("batched_fp64", PREC_FP64_BATCHED), ("batched_3xtf32", PREC_3XTF32)):
        # untimed warm-up on the first chunk (arena, tables)
        cb0 = pbatch.subset(b, idx_chunks[0])
        pbatch.run(cb0, local, cb0.alloc_outputs(dev), precision=prec, stream=stream, eng=eng)
        stream.synchronize()
        ms = []
        tb_full = None
        for _ in range(reps):
            with torch.cuda.stream(stream):
                flush.zero_()
            stream.synchronize()
            tot = 0.0
            parts = []
            for idx in idx_chunks:
                cb = pbatch.subset(b, idx)
                o = cb.alloc_outputs(dev)
                arrs = cb.device_arrays(dev)  # inputs resident before the timed launch
                torch.cuda.synchronize(dev)
                s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s0.record(stream)
                pbatch.run(cb, local, o, precision=prec, stream=stream, eng=eng)
                e0.record(stream)
                e0.synchronize()
                tot += s0.elapsed_time(e0)
                parts.append((idx, o["tb"].cpu().numpy(), int((o["status"] != 0).sum())))
                del o, arrs
                cb._dev = None
            ms.append(tot)
            tb_full = parts
        res[label] = b.n_solves() / (np.mean(ms) * 1e-3)
        res[label + "_ms_per_step"] = float(np.mean(ms))
        res[label + "_status_nonzero"] = int(sum(p[2] for p in tb_full))
        C, nout, F, N = b.ncol, int(b.host["noutlevels"]), int(b.host["max_nfreq"]), b.max_nummu
        tb = np.full((C, nout, 2 * N, F, 2), -9999.0)
        for idx, t, _ in tb_full:
            tb[idx, :, :t.shape[2], :t.shape[3], :] = t
        full[label] = tb
    singles = [pbatch.subset(b, [c]) for c in range(nplain)]
    souts = [sb.alloc_outputs(dev) for sb in singles]
    for sb, so in zip(singles, souts):
        pbatch.run(sb, local, so, stream=stream, eng=eng)
    stream.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        s.record(stream)
        for sb, so in zip(singles, souts):
            pbatch.run(sb, local, so, stream=stream, eng=eng)
        e.record(stream)
    e.synchronize()
    res["plain_fp64"] = sum(sb.n_solves() for sb in singles) / (s.elapsed_time(e) * 1e-3)
    res["plain_sample_columns"] = nplain
    res["batched_fp64_over_plain"] = res["batched_fp64"] / res["plain_fp64"]
    res["batched_3xtf32_over_plain"] = res["batched_3xtf32"] / res["plain_fp64"]
    a3, a64 = full["batched_3xtf32"], full["batched_fp64"]
    ok = a64 > -9000
    res["tb_err_3xtf32_vs_fp64_K"] = float(np.max(np.abs(a3 - a64)[ok])) if np.any(ok) else None
    if pool is not None and noracle > 0:
        idxs = oracle_sample(b, noracle)
        errs, bad = oracle_tb_errors(b, idxs, {"fp64": a64, "3xtf32": a3}, pool)
        res["tb_err_vs_oracle_K"] = {"batched_fp64": errs["fp64"], "batched_3xtf32": errs["3xtf32"],
                                     "columns": idxs, "oracle_errors": bad,
                                     "sample": "the cheapest columns of each NUMMU for the CPU oracle"}
    res["workload"] = name
    del flush
    return res


def _serving(args, local):
    """Replay one seeded stream of uneven requests through the
    continuous-batching server: the batched split-precision form at 200
    requests/s (far above capacity: latency is queueing) and at half of the
    capacity that run measured (latency is service), the batched FP64 form at
    200 requests/s, and the plain form (one column per call) on the first
    requests of the same stream at 200 requests/s."""
    from pamtra_b200 import serve
    from pamtra_b200._native import PREC_3XTF32, PREC_FP64, PREC_FP64_BATCHED
    n = args.serve_requests
    reqs = serve.request_stream(n, seed=5, max_cols=512, nfreq_range=(1, 32), sizes="loguniform")
    warm = serve.request_stream(3, seed=7, max_cols=16, nfreq_range=(1, 4))
    res = {"stream": "%d requests (seed 5): each 1-512 columns (log-uniform) of 40-150 layers, 1-5 species, "
                     "1-32 frequencies in 10-183 GHz, NUMMU in {8,16,32}; %d columns, %d solves in all"
                     % (n, sum(b.ncol for b in reqs), sum(b.n_solves() for b in reqs))}

    def one(prec, slots, cols, rate, nreq):
        arr = serve.poisson_arrivals(nreq, rate, seed=6)
        srv = serve.Server(local, slots=slots, hbm_fraction=0.5 if slots > 1 else 0.2, max_cols=cols,
                           precision=prec)
        for b in warm:
            srv.submit(b)
        srv.drain()
        nb0, ni0 = srv.batches_launched, len(srv.intervals)
        done, wall = serve.replay(srv, reqs[:nreq], arr)
        nb = srv.batches_launched - nb0
        iv = srv.intervals[ni0:]
        srv.close()
        solves = sum(r.n_solves() for r in done)
        ov = serve.overlapping_pairs(iv)
        return dict(serve.latency_stats(done), rate_req_s=rate, requests=nreq, solves=solves,
                    solves_per_s=solves / wall, wall_s=wall, batches=nb, slots=slots,
                    requests_with_error=sum(1 for r in done if r.error),
                    overlapping_batch_pairs=len(ov), overlap_ms=float(sum(o for _, _, o in ov)))

    hi = one(PREC_3XTF32, 3, 2048, 200.0, n)
    low_rate = 0.5 * n / hi["wall_s"]
    res["batched_3xtf32"] = {"rate_200": hi, "rate_half_capacity": one(PREC_3XTF32, 3, 2048, low_rate, n)}
    res["batched_fp64"] = {"rate_200": one(PREC_FP64_BATCHED, 3, 2048, 200.0, n)}
    nplain = min(n, args.serve_plain)
    res["plain_fp64"] = {"rate_200": one(PREC_FP64, 1, 1, 200.0, nplain)}
    res["note"] = ("rate_200 offers far more work than any form can serve, so its latencies are queueing "
                   "delay; rate_half_capacity offers half of the requests/s the batched split-precision form "
                   "completed at rate_200, so its latencies are service time. The plain form serves the "
                   "first %d requests of the same stream." % nplain)
    return res


# ---------------------------------------------------------------- reference arm
def _tmatrix_line(args, eng, dev, cpu_leg, pool=None, cores=1):
    """The T-matrix branch (scat_name 'tmatrix', src/tmatrix.f90:14) on a
    snow-like batch: soft ice spheroids (300 kg/m3, aspect ratio 0.6) in 32
    bins of 0.2-4 mm at 89 GHz, NUMMU 16, upright, per (layer, frequency)
    item; device-resident inputs for ``value``, host arrays through the C-ABI
    for ``e2e``; canted particles (beta 20 deg, the full amplitude path) on
    a smaller batch; the oracle (quad-precision restatement, one core) on the
    first item as the CPU baseline and the parity check."""
    import torch
    from pamtra_b200 import tmatrix as ptm
    ni, nb = args.tmatrix_items, 32

    def arrays(n, beta):
        d = np.linspace(0.2e-3, 4e-3, nb)[None, :].repeat(n, 0)
        return dict(dmax=d, del_d=np.full_like(d, 1.2e-4), ndens=np.full_like(d, 1e6),
                    density=np.full_like(d, 300.0), as_ratio=np.full_like(d, 0.6), canting=np.full_like(d, beta))

    def timed(n, beta, steps):
        a = arrays(n, beta)
        t = {k: torch.tensor(v, dtype=torch.float64, device=dev) for k, v in a.items()}
        fr = torch.full((n,), 89e9, dtype=torch.float64, device=dev)
        ri = torch.full((n,), 1.78 - 0.002j, dtype=torch.complex128, device=dev)
        ph = torch.full((n,), -1, dtype=torch.int32, device=dev)

        def run():
            return ptm.calc_tmatrix_batch(fr, ri, ph, t["dmax"], t["del_d"], t["ndens"], t["density"], t["as_ratio"],
                                          t["canting"], eng=eng)
        o = run()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            o = run()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, o, a

    ms, o, a = timed(ni, 0.0, 3)
    nm = o["nmax"].cpu().numpy()
    # e2e: numpy arrays through the host path of the C-ABI (copies in the call)
    h = arrays(ni, 0.0)
    fr, ri, ph = np.full(ni, 89e9), np.full(ni, 1.78 - 0.002j), np.full(ni, -1, dtype=np.int32)
    ptm.calc_tmatrix_batch(fr, ri, ph, h["dmax"], h["del_d"], h["ndens"], h["density"], h["as_ratio"], h["canting"],
                           eng=eng)
    t0 = time.perf_counter()
    for _ in range(3):
        oh = ptm.calc_tmatrix_batch(fr, ri, ph, h["dmax"], h["del_d"], h["ndens"], h["density"], h["as_ratio"],
                                    h["canting"], eng=eng)
    e2e_s = (time.perf_counter() - t0) / 3
    h2d = sum(v.nbytes for v in h.values()) + fr.nbytes + ri.nbytes + ph.nbytes
    d2h = sum(oh[k].nbytes for k in ("scatter_matrix", "extinct_matrix", "emis_vector", "sback", "back_spec", "status"))
    nc = max(1, ni // 16)
    ms_c, oc, _ = timed(nc, 20.0, 1)
    line = {"value": ni * nb / (ms * 1e-3), "unit": "bins/s", "ms_per_step": ms,
            "workload": "%d items x %d bins, soft ice spheroids 300 kg/m3, aspect ratio 0.6, 0.2-4 mm, 89 GHz, "
                        "NUMMU 16, upright" % (ni, nb),
            "nmax_range": [int(nm.min()), int(nm.max())], "status_nonzero": int(np.count_nonzero(o["status"].cpu().numpy())),
            "e2e": {"value": ni * nb / e2e_s, "unit": "bins/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "gpu_launches_per_step": 3,
            "canted": {"value": nc * nb / (ms_c * 1e-3), "unit": "bins/s", "items": nc, "beta_deg": 20.0,
                       "form": "full AMPL per (incident angle, scattered angle, azimuth)"},
            "bound": "latency: one FP64 CTA chain per bin (solves of order 2 (NMAX - m + 1) with a CTA barrier "
                     "per pivot, then the angular sums); no tensor-core or HBM bound applies"}
    if cpu_leg:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        t0 = time.perf_counter()
        r = oracle.tmatrix_species(16, 89e9, 1.78, -0.002, -1, *[a[k][0] for k in ("dmax", "del_d", "ndens", "density",
                                                                                  "as_ratio", "canting")])
        cpu_s = time.perf_counter() - t0
        err = 0.0
        g = {"scatter_matrix": o["scatter_matrix"][0].cpu().numpy().reshape((2, 16, 2, 16, 2), order="F"),
             "extinct_matrix": o["extinct_matrix"][0].cpu().numpy().reshape((2, 2, 16), order="F"),
             "emis_vector": o["emis_vector"][0].cpu().numpy().reshape((2, 16), order="F"),
             "back_spec": o["back_spec"][0].cpu().numpy()}
        for k, v in g.items():
            err = max(err, float(np.max(np.abs(v - r[k])) / np.max(np.abs(r[k]))))
        line["cpu_baseline"] = {"value": nb / cpu_s, "unit": "bins/s", "cores": 1, "kind": "port",
                                "sample": "the first item's %d bins, quad-precision T-matrix solve like the "
                                          "reference's REAL*16 tmatrix_amplq" % nb}
        if pool is not None:
            v, ntask, wall, ok = tmatrix_cpu_baseline(pool, cores, {k: a[k][0] for k in a})
            line["cpu_baseline"]["all_cores"] = {"value": v, "unit": "bins/s", "cores": cores, "tasks": ntask,
                                                 "wall_s": wall, "all_solved": ok,
                                                 "sample": "the first item's bins cycled to %d one-bin tasks, "
                                                           "one worker process per core" % ntask}
        line["max_rel_err_vs_oracle"] = err
    return line


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import warnings
    warnings.simplefilter("ignore")
    from pamtra_b200 import batch as pbatch
    from pamtra_b200.workloads import c2_pam
    cores = os.cpu_count() or 1
    ncol = min(args.ncol, 512)
    b = pbatch.pack_pam(c2_pam(ncol), FREQS)
    per_step = max(1, 4 * cores) if not args.cpu_sample else args.cpu_sample
    rng = np.random.default_rng(0)
    vals = []
    pool = make_pool(cores)
    for step in range(args.warmup + args.steps):
        idxs = sorted(rng.choice(ncol, size=min(per_step, ncol), replace=False).tolist())
        v, wall, _ = cpu_baseline(b, idxs, FREQS, cores, pool)
        if step >= args.warmup:
            vals.append((len(idxs) * len(FREQS), wall))
    pool.close()
    solves = sum(s for s, _ in vals)
    wall = sum(w for _, w in vals)
    value = solves / wall
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / len(vals),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": _config(args.ncol),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": "%d random columns x %d frequencies per step of the same workload; "
                                       "C++ FP64 restatement of the reference Fortran (no Fortran compiler "
                                       "on this image)" % (per_step, len(FREQS))},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- our arm
def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
        return
    import warnings
    warnings.simplefilter("ignore")
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from pamtra_b200 import batch as pbatch
    from pamtra_b200 import build as pbuild
    from pamtra_b200._native import Engine
    from pamtra_b200.workloads import c2_pam
    from pamtra_b200 import autotune
    from pamtra_b200 import replicas
    pbuild.build()
    eng = Engine(local)
    b = pbatch.pack_pam(c2_pam(args.ncol, seed=2 + rank), FREQS)
    stream = torch.cuda.Stream(dev)
    out = b.alloc_outputs(dev, ssp=True)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # launch shapes of the persistent kernels, tuned on this batch (untimed)
    from pamtra_b200._native import PREC_FP64_BATCHED as BF
    shape64, tune64 = autotune.tune(b, local, precision=BF, eng=eng, stream=stream, outputs=out)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            pbatch.run(b, local, out, precision=BF, stream=stream, eng=eng)
    stream.synchronize()
    status = out["status"].cpu().numpy()
    nd = out["num_doubles"].cpu().numpy()
    nlaunch = eng.last_launch_count()
    # ---- device-timed batched steps
    eng.set_timing(True)
    stage_tot = {}
    times = []
    sampler = ClockSampler(local)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            pbatch.run(b, local, out, precision=BF, stream=stream, eng=eng)
            e.record(stream)
        e.synchronize()
        times.append(s.elapsed_time(e))
        for k, v in eng.stage_ms().items():
            stage_tot[k] = stage_tot.get(k, 0.0) + v
    torch.cuda.synchronize()
    clocks = sampler.stop()
    eng.set_timing(False)
    layer_products = eng.layer_products(stream)
    t_total = sum(times) * 1e-3
    t_total = replicas.max_over_ranks(t_total)
    solves_step = b.n_solves()
    value = world * solves_step * args.steps / t_total
    # ---- the same step replayed from a captured CUDA graph
    graph, gout = pbatch.capture(b, local, precision=BF, stream=stream, eng=eng)
    for _ in range(args.warmup):
        graph.launch(stream)
    stream.synchronize()
    g_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            graph.launch(stream)
            e.record(stream)
        e.synchronize()
        g_ms.append(s.elapsed_time(e))
    graph_same = bool(np.array_equal(gout["tb"].cpu().numpy(), out["tb"].cpu().numpy()))
    graph.close()
    del gout
    graph_value = world * solves_step / (np.mean(g_ms) * 1e-3)
    # ---- end-to-end through the C ABI with host buffers
    hout = b.alloc_outputs(None, pinned=True)
    pbatch.run_host(b, local, hout, precision=BF, eng=eng)
    e2e_t = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        pbatch.run_host(b, local, hout, precision=BF, eng=eng)
        e2e_t.append(time.perf_counter() - t0)
    e2e_total = sum(e2e_t)
    e2e_total = replicas.max_over_ranks(e2e_total)
    h2d = sum(v.nbytes for v in b.host.values() if isinstance(v, np.ndarray))
    d2h = sum(v.nbytes for v in hout.values())
    # ---- split-precision batched form (3xTF32 tcgen05 doubling and adding) on the same columns
    from pamtra_b200._native import PREC_3XTF32, PREC_3XTF32_FP64ADD
    sout = b.alloc_outputs(dev)
    shape_s, _ = autotune.tune(b, local, precision=PREC_3XTF32, eng=eng, stream=stream, outputs=sout)
    sms_, sstages = _timed_steps(b, local, eng, stream, sout, PREC_3XTF32, args.steps, args.warmup, flush)
    split_value = world * solves_step / (np.mean(sms_) * 1e-3)
    tb_split = sout["tb"].cpu().numpy()
    split_err_f64 = float(np.max(np.abs(tb_split - out["tb"].cpu().numpy())))
    # the same with the FP64 adding (split-precision doubling only), for comparison; its adding
    # stage runs the FP64 kernel, so it takes the FP64 shape's adding CTAs per SM
    fout = b.alloc_outputs(dev)
    shape_fa = list(shape_s)
    shape_fa[3] = shape64[3]
    eng.set_launch(shape_fa)
    fms_, fstages = _timed_steps(b, local, eng, stream, fout, PREC_3XTF32_FP64ADD, args.steps, args.warmup, flush)
    eng.set_launch(shape64)
    split_fa = {"value": world * solves_step / (np.mean(fms_) * 1e-3), "unit": "solves/s",
                "ms_per_step": float(np.mean(fms_)), "stage_ms": fstages,
                "tb_err_vs_fp64_batched_K": float(np.max(np.abs(fout["tb"].cpu().numpy() - out["tb"].cpu().numpy()))),
                "launch_shape": shape_fa,
                "form": "PREC_3XTF32_FP64ADD: the 3xTF32 doubling with the one-inverse FP64 adding"}
    del fout
    # ---- plain form: one column per call
    nplain = 32
    plain_batches = [pbatch.pack_pam(c2_pam(1, seed=1000 + i), FREQS) for i in range(nplain)]
    pouts = [pb_.alloc_outputs(dev) for pb_ in plain_batches]
    with torch.cuda.stream(stream):
        for pb_, po in zip(plain_batches, pouts):
            pbatch.run(pb_, local, po, stream=stream, eng=eng)
    stream.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        s.record(stream)
        for pb_, po in zip(plain_batches, pouts):
            pbatch.run(pb_, local, po, stream=stream, eng=eng)
        e.record(stream)
    e.synchronize()
    plain_value = nplain * len(FREQS) / (s.elapsed_time(e) * 1e-3)
    # the plain form on the first columns of the batch: agreement with the batched form
    tb_b = out["tb"].cpu().numpy()
    plain_diff = 0.0
    for c in range(4):
        po = pbatch.run(pbatch.subset(b, [c]), local, eng=eng)
        plain_diff = max(plain_diff, float(np.max(np.abs(po["tb"].cpu().numpy()[0] - tb_b[c]))))

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    # one spawned pool of oracle workers for the CPU baseline and the oracle checks
    cores = os.cpu_count() or 1
    pool = make_pool(cores) if not args.no_cpu else None
    target = _target_shape(args, local, eng, stream) if args.target_cols > 0 else None
    from pamtra_b200 import workloads as wl
    uneven = _config_line("%d columns, layers uniform 40-150, 1-5 species (cloud water, cloud ice, snow, graupel, "
                          "rain; exp or mgamma with mu 0-4; 20-80 bins; ice 100-900 kg/m3), 8-32 frequencies in "
                          "10-183 GHz, NUMMU 8/16/32 per column" % args.uneven_cols,
                          wl.uneven_batch(args.uneven_cols, seed=3), local, eng, stream, pool) \
        if args.uneven_cols > 0 else None
    mieheavy = _config_line("%d columns x 100 layers, 4 species x 200 bins up to 10 mm (rain, snow, graupel, "
                            "cloud ice), f = 89/157/176.31/190.31 GHz, NUMMU 16" % args.mieheavy_cols,
                            wl.mie_heavy_batch(args.mieheavy_cols, seed=6), local, eng, stream, pool) \
        if args.mieheavy_cols > 0 else None
    serving = _serving(args, local) if args.serve_requests > 0 else None
    tmat = _tmatrix_line(args, eng, dev, not args.no_cpu, pool, cores) if args.tmatrix_items > 0 else None
    # ---- roofline of the dominant kernel (doubling stage)
    peak = fp64_peak_tflops(dev)
    t_layer = stage_tot.get("layer", 0.0) / args.steps * 1e-3
    flops = layer_flops(nd, 16)
    achieved = flops / t_layer / 1e12 if t_layer > 0 else 0.0
    items = int(np.count_nonzero(nd >= 0))
    roofline = {"bound": "tensor", "pipe": "FP64 tensor (DMMA)", "kernel": "k_layer<16> (scatcnv + init + doubling)",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                "traffic": LAYER_TRAFFIC_PER_ITEM * items,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch at 256 columns "
                                  "(21,504 items), scaled by the %d items of this launch" % items,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor pipe); "
                               "MEASURED_PEAKS.json carries bf16 and HBM only",
                "flops_per_launch": flops, "kernel_ms": t_layer * 1e3,
                "achieved_executed": 2.0 * 32 ** 3 * layer_products / t_layer / 1e12 if t_layer > 0 else None,
                "executed_products_per_launch": layer_products,
                "executed_note": "n x n products the kernel issued (5 per doubling plus the Neumann/Horner "
                                 "series, Gauss-Jordan counted as one), 2 n^3 FLOP each, n = 32; the algorithmic "
                                 "figure counts 6 products and one inverse per doubling"}
    roofline["frac_executed"] = roofline["achieved_executed"] / peak if peak and roofline["achieved_executed"] \
        else None
    # ---- CPU baseline + TB error vs the oracle on the same columns
    cpu = None
    tb_err = None
    split_err_oracle = None
    if pool is not None:
        nsamp = args.cpu_sample or min(b.ncol, 8 * cores)
        idxs = sorted(np.random.default_rng(7).choice(b.ncol, size=nsamp, replace=False).tolist())
        cval, wall, tbs = cpu_baseline(b, idxs, FREQS, cores, pool)
        pool.close()
        one_val, one_wall = cpu_single_core(b, idxs[:max(2, nsamp // (2 * cores))], FREQS)
        tb_gpu = out["tb"].cpu().numpy()
        tb_err = max(float(np.max(np.abs(tb_gpu[c] - tbs[c]))) for c in idxs)
        split_err_oracle = max(float(np.max(np.abs(tb_split[c] - tbs[c]))) for c in idxs)
        cpu = {"value": cval, "unit": "solves/s", "cores": cores, "kind": "port",
               "sample": "%d random columns x %d frequencies of the same workload, one worker process per core; "
                         "C++ FP64 restatement of the reference Fortran (no Fortran compiler on this image)"
                         % (nsamp, len(FREQS)),
               "single_core": {"value": one_val, "unit": "solves/s", "cores": 1,
                               "sample": "%d of those columns x %d frequencies in one process"
                                         % (max(2, nsamp // (2 * cores)), len(FREQS)), "wall_s": one_wall},
               "cpu_model": cpu_model(), "wall_s": wall}
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": _config(args.ncol),
        "e2e": {"value": world * solves_step * args.steps / e2e_total, "unit": "solves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(nlaunch * args.steps),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks,
        "plain_fp64": {"value": plain_value, "unit": "solves/s",
                       "form": "one column per call, FP64 in the reference operation order (PREC_FP64)",
                       "tb_max_diff_vs_batched_K": plain_diff},
        "batched_form": "FP64, one-inverse adding combine (PREC_FP64_BATCHED)",
        "graph_replay": {"value": graph_value, "unit": "solves/s", "ms_per_step": float(np.mean(g_ms)),
                         "tb_equals_direct": graph_same,
                         "form": "the batched FP64 step captured once as a CUDA graph and replayed"},
        "launch_shape": {"fp64": list(shape64), "split_3xtf32": list(shape_s),
                         "fields": "mie warps/CTA, mie CTAs/SM, layer CTAs/SM, adding CTAs/SM (0 = as many as fit)",
                         "stage_ms_per_candidate_fp64": tune64,
                         "candidates": [list(c) for c in autotune.CANDIDATES]},
        "batched_over_plain": value / world / plain_value,
        "tb_err_vs_oracle_K": tb_err,
        "split_3xtf32": {"value": split_value, "unit": "solves/s", "ms_per_step": float(np.mean(sms_)),
                         "over_plain": split_value / world / plain_value,
                         "tb_err_vs_fp64_batched_K": split_err_f64,
                         "tb_err_vs_oracle_K": split_err_oracle, "stage_ms": sstages,
                         "form": "doubling and adding products as 3xTF32 tcgen05 MMAs (FP32 accumulation in "
                                 "TMEM); thin-layer init, the (I - R R)^-1 of each combine, sources of the "
                                 "doubling setup, surface and radiances in FP64",
                         "with_fp64_adding": split_fa},
        "stage_ms": {k: v / args.steps for k, v in stage_tot.items()},
        "serving": serving,
        "target_shape": target,
        "uneven": uneven,
        "mie_heavy": mieheavy,
        "tmatrix": tmat,
        "status_nonzero": int(np.count_nonzero(status)),
    }

    def g(d, *ks):
        for k in ks:
            if d is None:
                return None
            d = d.get(k)
        return d
    # the figures that matter, last on the line
    line["summary"] = {
        "c2_batched_fp64": value, "c2_batched_3xtf32": split_value, "c2_plain_fp64": plain_value,
        "c2_fp64_over_plain": value / world / plain_value, "c2_3xtf32_over_fp64": split_value / value,
        "c2_3xtf32_fp64_adding": split_fa["value"],
        "c2_adding_ms": {"fp64": stage_tot.get("adding", 0.0) / args.steps, "3xtf32": sstages.get("adding"),
                         "3xtf32_fp64_adding": fstages.get("adding")},
        "c2_tb_err_vs_oracle_K": {"fp64": tb_err, "3xtf32": split_err_oracle},
        "target_fp64_over_plain": g(target, "batched_over_plain"),
        "target_3xtf32_over_plain": g(target, "batched_3xtf32_over_plain"),
        "target_3xtf32_over_fp64": (target["batched_3xtf32"] / target["batched_fp64"]) if target else None,
        "uneven_cols": g(uneven, "columns"), "uneven_fp64": g(uneven, "batched_fp64"),
        "uneven_3xtf32": g(uneven, "batched_3xtf32"), "uneven_3xtf32_over_plain": g(uneven, "batched_3xtf32_over_plain"),
        "uneven_tb_err_vs_oracle_K": g(uneven, "tb_err_vs_oracle_K"),
        "mieheavy_cols": g(mieheavy, "columns"), "mieheavy_fp64": g(mieheavy, "batched_fp64"),
        "mieheavy_3xtf32": g(mieheavy, "batched_3xtf32"),
        "mieheavy_3xtf32_over_plain": g(mieheavy, "batched_3xtf32_over_plain"),
        "mieheavy_tb_err_vs_oracle_K": g(mieheavy, "tb_err_vs_oracle_K"),
        "serving_3xtf32_rate200_p50_p99_ms": [g(serving, "batched_3xtf32", "rate_200", "p50_ms"),
                                              g(serving, "batched_3xtf32", "rate_200", "p99_ms")],
        "serving_3xtf32_halfcap_p50_p99_ms": [g(serving, "batched_3xtf32", "rate_half_capacity", "p50_ms"),
                                              g(serving, "batched_3xtf32", "rate_half_capacity", "p99_ms")],
        "tmatrix_bins_per_s": {"gpu": g(tmat, "value"), "e2e": g(tmat, "e2e", "value"),
                               "cpu_1core": g(tmat, "cpu_baseline", "value"),
                               "cpu_all_cores": g(tmat, "cpu_baseline", "all_cores", "value"),
                               "max_rel_err_vs_oracle": g(tmat, "max_rel_err_vs_oracle")},
        "serving_solves_per_s": {"3xtf32": g(serving, "batched_3xtf32", "rate_200", "solves_per_s"),
                                 "fp64": g(serving, "batched_fp64", "rate_200", "solves_per_s"),
                                 "plain": g(serving, "plain_fp64", "rate_200", "solves_per_s")},
    }
    print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
