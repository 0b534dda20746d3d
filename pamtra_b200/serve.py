"""Continuous-batching request loop for column solves.

The reference has no server: pyPamtra runs one profile per call and farms
chunks to CPU processes (python/pyPamtra/core.py:1570-1676).  Here a single
scheduler thread owns ``slots`` execution slots on one GPU, each a native
context (its own scratch arena, reserved once from free HBM), a CUDA stream
and a set of device buffers.  Requests (packed batches of any size) arrive
through :meth:`Server.submit` from any thread.  Whenever a slot is free the
scheduler packs the waiting requests, oldest first, into one batch whose
scratch fits the slot's arena (pamtra_b200_workspace_bytes), copies it to the
device, launches the passive path and queues the copy of the results back,
all on the slot's stream, and goes on admitting into the other slots, so
work of several batches overlaps on the device.  A request larger than an
arena is split into chunks (grouped by NUMMU) that run as separate batches.
Inputs and scratch stay on the device until the batch's completion event
fires; the results of every request are then cut out of the merged outputs
in the request's own layout.

Latency of a request = completion seen by the scheduler - submit time.
"""

import collections
import threading
import time

import numpy as np

from . import batch as pbatch
from ._native import PREC_FP64, Engine, workspace_bytes


class Request(object):
    """One column-solve request: a packed batch plus its timing."""

    def __init__(self, rid, batch, t_submit):
        self.id = rid
        self.batch = batch
        self.t_submit = t_submit
        self.t_start = None    # first launch of any of its work
        self.t_done = None
        self.result = None     # dict of numpy arrays in the request's layout
        self.error = None
        self._parts = None     # chunked requests: [(col idx, sub batch, result)]
        self._left = 0
        self.done = threading.Event()

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_submit

    def n_solves(self):
        return self.batch.n_solves()


class _Unit(object):
    """A schedulable piece of work: a whole request or one chunk of it."""

    def __init__(self, req, batch, cols=None):
        self.req = req
        self.batch = batch
        self.cols = cols  # column indices in the request for chunks, else None


class _Slot(object):
    def __init__(self, device, arena_bytes):
        import torch
        self.eng = Engine(device)
        self.eng.reserve(arena_bytes)
        self.arena = arena_bytes
        self.stream = torch.cuda.Stream(device)
        self.busy = False
        self.units = None
        self.event = None
        self.keep = None
        self.host_out = None
        self.merged = None
        self.starts = None


class Server(object):
    """Continuous-batching server on one GPU.

    ``hbm_fraction`` of the free device memory at start-up is split evenly
    into the slots' scratch arenas; batches are packed to fit them.
    ``max_cols`` caps the columns of one merged batch (1 gives the plain
    form: one column per call)."""

    def __init__(self, device=0, slots=3, hbm_fraction=0.5, max_cols=2048, precision=PREC_FP64,
                 arena_bytes=None):
        import torch
        self.device = device
        self.dev = torch.device("cuda", device)
        torch.cuda.set_device(self.dev)
        if arena_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            arena_bytes = int(free * hbm_fraction / max(1, slots))
        self.slots = [_Slot(device, arena_bytes) for _ in range(slots)]
        self.max_cols = max_cols
        self.precision = precision
        self._queue = collections.deque()
        self._lock = threading.Lock()
        self._wake = threading.Condition(self._lock)
        self._stop = False
        self._next_id = 0
        self._all = []
        self.completed = []
        self.batches_launched = 0
        self.busy_time = 0.0
        self._thread = threading.Thread(target=self._loop, name="pamtra-b200-serve", daemon=True)
        self._thread.start()

    # ------------------------------------------------------------------ client side
    def submit(self, batch):
        """Queue a packed batch; returns its :class:`Request`."""
        with self._lock:
            r = Request(self._next_id, batch, time.perf_counter())
            self._next_id += 1
            self._queue.append(r)
            self._all.append(r)
            self._wake.notify()
        return r

    def close(self, wait=True):
        with self._lock:
            self._stop = True
            self._wake.notify()
        if wait:
            self._thread.join()

    def drain(self, timeout=None):
        """Wait until every request submitted so far is done."""
        with self._lock:
            reqs = list(self._all)
        t_end = None if timeout is None else time.perf_counter() + timeout
        for r in reqs:
            left = None if t_end is None else max(0.0, t_end - time.perf_counter())
            if not r.done.wait(left):
                return False
        return True

    # ------------------------------------------------------------------ scheduler
    def _split(self, req, arena):
        return split_request(req, arena, self.max_cols, self._need)

    def _need(self, b):
        return workspace_bytes(b.columns(b.host), precision=self.precision)

    def _loop(self):
        import torch
        torch.cuda.set_device(self.dev)
        waiting = collections.deque()  # units ready to be packed
        arena = min(s.arena for s in self.slots)
        while True:
            with self._lock:
                while self._queue:
                    waiting.extend(self._split(self._queue.popleft(), arena))
                if self._stop and not waiting and not any(s.busy for s in self.slots):
                    return
            progressed = False
            # completions
            for s in self.slots:
                if s.busy and s.event.query():
                    self._complete(s)
                    progressed = True
            # admissions
            for s in self.slots:
                if not waiting:
                    break
                if not s.busy:
                    try:
                        self._launch(s, waiting)
                    except Exception as exc:  # a failed launch ends its requests, not the loop
                        self._fail(s, exc)
                    progressed = True
            if not progressed:
                with self._lock:
                    if not self._queue and not self._stop:
                        self._wake.wait(timeout=0.0005)

    def _pack(self, s, waiting):
        return pack_units(waiting, s.arena, self.max_cols, self._need)

    def _launch(self, s, waiting):
        import torch
        units = self._pack(s, waiting)
        s.units = units
        if len(units) == 1:
            merged, starts = units[0].batch, [0]
        else:
            merged, starts = pbatch.concat([u.batch for u in units])
        now = time.perf_counter()
        for u in units:
            if u.req.t_start is None:
                u.req.t_start = now
        with torch.cuda.stream(s.stream):
            pinned = merged.pinned_arrays()
            arrs = dict()
            for k, v in pinned.items():
                if isinstance(v, np.ndarray):
                    arrs[k] = torch.from_numpy(v).to(self.dev, non_blocking=True)
                else:
                    arrs[k] = v
            dout = merged.alloc_outputs(self.dev)
            s.eng.run(merged.settings, merged.columns(arrs), s.eng.make_outputs(dout), self.precision, s.stream)
            hout = dict()
            for k, v in dout.items():
                h = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                h.copy_(v, non_blocking=True)
                hout[k] = h
            ev = torch.cuda.Event()
            ev.record(s.stream)
        s.busy = True
        s.units, s.merged, s.starts = units, merged, starts
        s.event, s.host_out = ev, hout
        s.keep = (pinned, arrs, dout)
        s.t_launch = now
        self.batches_launched += 1

    def _fail(self, s, exc):
        now = time.perf_counter()
        for u in (s.units or []):
            if not u.req.done.is_set():
                u.req.error = "launch failed: %s" % exc
                u.req.t_done = now
                u.req.done.set()
        s.busy = False
        s.units = s.merged = s.starts = s.event = s.host_out = s.keep = None

    def _complete(self, s):
        now = time.perf_counter()
        outs = {k: v.numpy() for k, v in s.host_out.items()}
        parts = pbatch.split_outputs(outs, [u.batch for u in s.units], s.starts)
        for u, r in zip(s.units, parts):
            req = u.req
            if u.cols is None:
                req.result = {k: np.array(v) for k, v in r.items()}
                self._finish(req, now)
            else:
                req._parts.append((u.cols, u.batch, {k: np.array(v) for k, v in r.items()}))
                req._left -= 1
                if req._left == 0:
                    req.result = _assemble(req.batch, req._parts)
                    self._finish(req, now)
        s.busy = False
        s.units = s.merged = s.starts = s.event = s.host_out = s.keep = None

    def _finish(self, req, now):
        req.t_done = now
        if np.any(req.result["status"] & 2):
            req.error = "fatal status in %d column-frequency solves" % int(np.sum((req.result["status"] & 2) != 0))
        self.completed.append(req)
        req.done.set()


def split_request(req, arena, max_cols, need):
    """Units of a request: the request itself if its scratch fits ``arena``
    and it has at most ``max_cols`` columns, else its chunks
    (batch.chunk_columns)."""
    if need(req.batch) <= arena and req.batch.ncol <= max_cols:
        return [_Unit(req, req.batch)]
    chunks = pbatch.chunk_columns(req.batch, arena, max_cols=max_cols)
    req._parts = []
    req._left = len(chunks)
    return [_Unit(req, pbatch.subset(req.batch, idx), idx) for idx in chunks]


LOOKAHEAD = 64  # waiting units further back are not pulled past older ones


def pack_units(waiting, arena, max_cols, need, lookahead=LOOKAHEAD):
    """Greedy packing, oldest first: the oldest waiting unit opens the batch;
    younger units with the same settings, output levels and NUMMU (a batch's
    layer matrices are strided for its largest NUMMU) join while the merged
    batch's scratch ``need(batch)`` fits ``arena`` and the column cap holds.
    Takes the chosen units off ``waiting`` (a deque) and returns them;
    skipped units keep their order."""
    head = waiting.popleft()
    take = [head]
    cols = head.batch.ncol
    key = (bytes(head.batch.settings), int(head.batch.host["noutlevels"]), head.batch.max_nummu)
    skipped = []
    looked = 0
    while waiting and looked < lookahead and cols < max_cols:
        cand = waiting.popleft()
        looked += 1
        ck = (bytes(cand.batch.settings), int(cand.batch.host["noutlevels"]), cand.batch.max_nummu)
        if ck != key or cols + cand.batch.ncol > max_cols:
            skipped.append(cand)
            continue
        merged, _ = pbatch.concat([u.batch for u in take] + [cand.batch])
        if need(merged) > arena:
            skipped.append(cand)
            continue
        take.append(cand)
        cols += cand.batch.ncol
    waiting.extendleft(reversed(skipped))
    return take


def _assemble(b, parts):
    """Results of a chunked request in the request's own layout."""
    C, F, N = b.ncol, int(b.host["max_nfreq"]), b.max_nummu
    shapes = b.output_shapes()
    out = dict()
    for k, (shape, dt) in shapes.items():
        out[k] = np.zeros(shape, dtype=dt)
    out["tb"][:] = -9999.0
    for cols, sub, r in parts:
        n2, Fs, Ns = 2 * sub.max_nummu, int(sub.host["max_nfreq"]), sub.max_nummu
        out["tb"][cols, :, :n2, :Fs, :] = r["tb"]
        out["emissivity"][cols, :, :Fs, :Ns] = r["emissivity"]
        out["status"][cols, :Fs] = r["status"]
        if Ns == N:
            out["angles_deg"][:] = r["angles_deg"]
    del F, C
    return out


def latency_stats(requests):
    """p50 / p99 / mean latency in ms over completed requests."""
    lat = np.array([r.latency for r in requests if r.latency is not None]) * 1e3
    if len(lat) == 0:
        return dict(p50_ms=None, p99_ms=None, mean_ms=None, n=0)
    return dict(p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                mean_ms=float(lat.mean()), max_ms=float(lat.max()), n=int(len(lat)))


def poisson_arrivals(n, rate, seed=0):
    """Seeded arrival offsets [s] of a Poisson stream of ``rate`` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, n))


def request_stream(n, seed=5, max_cols=512, nfreq_range=(1, 32)):
    """Seeded requests shaped like the serving workload: 1-``max_cols``
    columns each, 40-150 layers, 1-5 species, 1-32 frequencies in 10-183 GHz
    and NUMMU in {8, 16, 32}, one NUMMU per request."""
    from . import workloads
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ncol = int(rng.integers(1, max_cols + 1))
        N = int(rng.choice([8, 16, 32]))
        out.append(workloads.uneven_batch(ncol, seed=int(rng.integers(1 << 30)), nummu_choices=(N,),
                                          nfreq_range=nfreq_range))
    return out


def replay(server, batches, arrivals):
    """Submit ``batches`` at the seeded ``arrivals`` offsets (seconds after
    the call) and wait for all of them; returns the requests and the wall
    time from the first arrival to the last completion."""
    t0 = time.perf_counter()
    reqs = []
    for b, ta in zip(batches, arrivals):
        dt = t0 + ta - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        reqs.append(server.submit(b))
    for r in reqs:
        r.done.wait()
    t_first = min(r.t_submit for r in reqs)
    t_last = max(r.t_done for r in reqs)
    return reqs, t_last - t_first
