"""Continuous-batching request loop for column solves.

The reference has no server: pyPamtra runs one profile per call and farms
chunks to CPU processes (python/pyPamtra/core.py:1570-1676).  Here a single
scheduler thread owns ``slots`` execution slots on one GPU.  Each slot is a
native context (its own scratch arena, reserved once from free HBM), a CUDA
stream and a pair of resident staging buffers (device memory and page-locked
host memory, sized at start-up for the largest batch the server packs and
reused by every batch).  Requests (packed batches of any size) arrive
through :meth:`Server.submit` from any thread.  Whenever a slot is free the
scheduler packs the waiting requests, oldest first, into one batch whose
scratch fits the slot's arena (pamtra_b200_workspace_bytes), writes its
inputs into the slot's host buffer, and queues on the slot's stream one
host-to-device copy, the passive path and one device-to-host copy of the
results; then it goes on admitting into the other slots, so the work of
several batches overlaps on the device.  A request larger than an arena is
split into chunks (grouped by NUMMU) that run as separate batches.

Each slot has a waiter thread that blocks on the batch's completion event,
cuts every request's results out of the merged outputs in the request's
own layout, frees the slot and wakes the scheduler; nothing polls.  The
species tables and the scatcnv azimuth weight tables stay resident in each
slot's context between batches.

Latency of a request = completion seen by the waiter - submit time.
"""

import collections
import queue
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


_ALIGN = 256


def _layout(items):
    """Offsets (256-byte aligned) of (name, nbytes) items in one buffer."""
    offs, off = {}, 0
    for k, nb in items:
        off = (off + _ALIGN - 1) // _ALIGN * _ALIGN
        offs[k] = off
        off += nb
    return offs, off


def batch_bytes_bound(max_cols, max_layers=150, max_freqs=32, max_nummu=32, max_species=5, noutlevels=2):
    """Upper bounds on the input and output bytes of a batch of ``max_cols``
    columns (the sizes of a slot's staging buffers)."""
    L, F, N, H = max_layers, max_freqs, max_nummu, max_species
    per_in = 8 * (4 * (L + 1) + 4 * L + 3 * L * H + F + 2 + noutlevels) + 3 * 4 + 1
    per_out = 8 * (noutlevels * 2 * N * F * 2 + 2 * F * N) + 4 * F
    n_arrays = 24
    return max_cols * per_in + n_arrays * _ALIGN, max_cols * per_out + 8 * 2 * N + 8 * _ALIGN


class _Slot(object):
    def __init__(self, index, device, arena_bytes, in_bytes, out_bytes):
        import torch
        self.index = index
        self.device = device
        self.eng = Engine(device)
        self.eng.reserve(arena_bytes)
        self.arena = arena_bytes
        self.stream = torch.cuda.Stream(device)
        self.h_in = self.d_in = self.h_out = self.d_out = None
        self._ensure(in_bytes, out_bytes)
        self.busy = False
        self.units = self.merged = self.starts = self.outs = None
        self.ev_start = self.ev_end = self.t_launch = None
        self.jobs = queue.Queue()

    def _ensure(self, in_bytes, out_bytes):
        """Grow the staging buffers (only when a batch exceeds them; the
        server sizes them at start-up so that this does not happen)."""
        import torch
        dev = torch.device("cuda", self.device)
        if self.h_in is None or self.h_in.numel() < in_bytes:
            self.h_in = torch.empty(int(in_bytes), dtype=torch.uint8).pin_memory()
            self.d_in = torch.empty(int(in_bytes), dtype=torch.uint8, device=dev)
        if self.h_out is None or self.h_out.numel() < out_bytes:
            self.h_out = torch.empty(int(out_bytes), dtype=torch.uint8).pin_memory()
            self.d_out = torch.empty(int(out_bytes), dtype=torch.uint8, device=dev)


_TORCH_DT = None


def _tdt(np_dtype):
    import torch
    global _TORCH_DT
    if _TORCH_DT is None:
        _TORCH_DT = {np.dtype(np.float64): torch.float64, np.dtype(np.int32): torch.int32,
                     np.dtype(np.int8): torch.int8}
    return _TORCH_DT[np.dtype(np_dtype)]


class Server(object):
    """Continuous-batching server on one GPU.

    ``hbm_fraction`` of the free device memory at start-up is split evenly
    into the slots' scratch arenas; batches are packed to fit them.
    ``max_cols`` caps the columns of one merged batch (1 gives the plain
    form: one column per call); the staging buffers are sized for it and
    the largest column shape (``max_layers``, ``max_freqs``, ``max_nummu``,
    ``max_species``)."""

    def __init__(self, device=0, slots=3, hbm_fraction=0.5, max_cols=2048, precision=PREC_FP64,
                 arena_bytes=None, max_layers=150, max_freqs=32, max_nummu=32, max_species=5):
        import torch
        self.device = device
        self.dev = torch.device("cuda", device)
        torch.cuda.set_device(self.dev)
        in_b, out_b = batch_bytes_bound(max_cols, max_layers, max_freqs, max_nummu, max_species)
        if arena_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            arena_bytes = int((free * hbm_fraction - slots * (in_b + out_b)) / max(1, slots))
        self.slots = [_Slot(i, device, arena_bytes, in_b, out_b) for i in range(slots)]
        self.max_cols = max_cols
        self.precision = precision
        self._queue = collections.deque()
        self._lock = threading.Lock()
        self._cv = threading.Condition(self._lock)
        self._stop = False
        self._next_id = 0
        self._all = []
        self.completed = []
        self.batches_launched = 0
        self.intervals = []  # per batch: (slot, device start ms, device end ms, columns), from a common origin
        torch.cuda.synchronize(self.dev)
        self._t0 = torch.cuda.Event(enable_timing=True)
        self._t0.record(torch.cuda.current_stream(self.dev))
        self._t0.synchronize()
        self._waiters = [threading.Thread(target=self._wait_loop, args=(s,), name="pamtra-b200-wait%d" % s.index,
                                          daemon=True) for s in self.slots]
        for t in self._waiters:
            t.start()
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
            self._cv.notify_all()
        return r

    def close(self, wait=True):
        with self._lock:
            self._stop = True
            self._cv.notify_all()
        if wait:
            self._thread.join()
            for s in self.slots:
                s.jobs.put(None)
            for t in self._waiters:
                t.join()

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
        waiting = collections.deque()  # units ready to be packed (scheduler thread only)
        arena = min(s.arena for s in self.slots)
        while True:
            with self._lock:
                while True:
                    new = list(self._queue)
                    self._queue.clear()
                    free = [s for s in self.slots if not s.busy]
                    if new or (waiting and free):
                        break
                    if self._stop and not waiting and len(free) == len(self.slots):
                        return
                    self._cv.wait()  # woken by a submission, a completion or close()
                if not new and free:
                    free[0].busy = True  # claimed under the lock; released by its waiter
            for r in new:
                waiting.extend(self._split(r, arena))
            if new:
                continue  # re-check the free slots with the new units in place
            s = free[0]
            try:
                self._launch(s, waiting)
            except Exception as exc:  # a failed launch ends its requests, not the loop
                self._fail(s, exc)

    def _launch(self, s, waiting):
        import torch
        units = pack_units(waiting, s.arena, self.max_cols, self._need)
        s.units = units
        if len(units) == 1:
            merged, starts = units[0].batch, [0]
        else:
            merged, starts = pbatch.concat([u.batch for u in units])
        now = time.perf_counter()
        for u in units:
            if u.req.t_start is None:
                u.req.t_start = now
        h = merged.host
        in_items = [(k, v.nbytes) for k, v in h.items() if isinstance(v, np.ndarray)]
        in_off, in_bytes = _layout(in_items)
        shapes = merged.output_shapes()
        out_items = [(k, int(np.prod(shp)) * np.dtype(dt).itemsize) for k, (shp, dt) in shapes.items()]
        out_off, out_bytes = _layout(out_items)
        s._ensure(in_bytes, out_bytes)
        # inputs: host arrays -> the slot's page-locked buffer -> one copy to the device
        hb = s.h_in.numpy()
        for k, nb in in_items:
            v = np.ascontiguousarray(h[k])
            hb[in_off[k]:in_off[k] + nb] = v.view(np.uint8).reshape(-1)
        arrs = dict()
        for k, v in h.items():
            if isinstance(v, np.ndarray):
                o = in_off[k]
                arrs[k] = s.d_in[o:o + v.nbytes].view(_tdt(v.dtype)).view(v.shape)
            else:
                arrs[k] = v
        dout = dict()
        for k, (shp, dt) in shapes.items():
            o = out_off[k]
            n = int(np.prod(shp)) * np.dtype(dt).itemsize
            dout[k] = s.d_out[o:o + n].view(_tdt(dt)).view(shp)
        s.ev_start = torch.cuda.Event(enable_timing=True)
        s.ev_end = torch.cuda.Event(enable_timing=True, blocking=True)
        with torch.cuda.stream(s.stream):
            s.d_in[:in_bytes].copy_(s.h_in[:in_bytes], non_blocking=True)
            s.d_out[:out_bytes].zero_()
            s.ev_start.record(s.stream)
            s.eng.run(merged.settings, merged.columns(arrs), s.eng.make_outputs(dout), self.precision, s.stream)
            s.ev_end.record(s.stream)
            s.h_out[:out_bytes].copy_(s.d_out[:out_bytes], non_blocking=True)
            done = torch.cuda.Event(blocking=True)
            done.record(s.stream)
        hob = s.h_out.numpy()
        s.outs = {k: hob[out_off[k]:out_off[k] + nb].view(shapes[k][1]).reshape(shapes[k][0])
                  for k, nb in out_items}
        s.merged, s.starts, s.t_launch = merged, starts, now
        self.batches_launched += 1
        s.jobs.put(done)

    def _wait_loop(self, s):
        import torch
        torch.cuda.set_device(self.dev)
        while True:
            done = s.jobs.get()
            if done is None:
                return
            try:
                done.synchronize()
                self._complete(s)
            except Exception as exc:
                self._fail(s, exc)
                continue
            with self._lock:
                s.busy = False
                self._cv.notify_all()

    def _fail(self, s, exc):
        now = time.perf_counter()
        for u in (s.units or []):
            if not u.req.done.is_set():
                u.req.error = "launch failed: %s" % exc
                u.req.t_done = now
                u.req.done.set()
        with self._lock:
            s.busy = False
            s.units = s.merged = s.starts = s.outs = None
            self._cv.notify_all()

    def _complete(self, s):
        now = time.perf_counter()
        self.intervals.append((s.index, self._t0.elapsed_time(s.ev_start), self._t0.elapsed_time(s.ev_end),
                               s.merged.ncol))
        parts = pbatch.split_outputs(s.outs, [u.batch for u in s.units], s.starts)
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
        s.units = s.merged = s.starts = s.outs = None

    def _finish(self, req, now):
        req.t_done = now
        if np.any(req.result["status"] & 2):
            req.error = "fatal status in %d column-frequency solves" % int(np.sum((req.result["status"] & 2) != 0))
        self.completed.append(req)
        req.done.set()


def overlapping_pairs(intervals):
    """Pairs of batches of different slots whose device intervals overlap,
    with the overlap in ms: [(i, j, ms)]."""
    out = []
    for i in range(len(intervals)):
        for j in range(i + 1, len(intervals)):
            si, a0, a1, _ = intervals[i]
            sj, b0, b1, _ = intervals[j]
            ov = min(a1, b1) - max(a0, b0)
            if si != sj and ov > 0:
                out.append((i, j, ov))
    return out


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


def request_stream(n, seed=5, max_cols=512, nfreq_range=(1, 32), sizes="uniform"):
    """Seeded requests shaped like the serving workload: 1-``max_cols``
    columns each (uniform, or log-uniform with ``sizes="loguniform"``: many
    small requests and few large ones), 40-150 layers, 1-5 species, 1-32
    frequencies in 10-183 GHz and NUMMU in {8, 16, 32}, one NUMMU per
    request."""
    from . import workloads
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        if sizes == "loguniform":
            ncol = min(max_cols, int(np.exp(rng.uniform(0.0, np.log(max_cols + 1.0)))))
        else:
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
