"""Batched form: packs many columns (each with its own layer count,
hydrometeor set, frequency list and NUMMU) into one set of padded arrays,
keeps them resident on the device and runs them through one launch
sequence of the native library.

The reference parallelises (column, frequency) chunks over CPU processes
(python/pyPamtra/core.py:1570-1676); here a whole batch is one stream of
persistent kernels.
"""

import numpy as np

from . import libWrapper, packing
from ._native import PREC_FP64, Columns, Engine, engine, workspace_bytes

_MASK = {8: 1, 16: 2, 32: 4}


class PackedBatch(object):
    """Host-side packed batch.  ``host`` holds C-contiguous numpy arrays in the
    layouts of include/pamtra_b200.h."""

    def __init__(self, settings, species, host, nummu_mask, max_nummu, species_stride, max_present):
        self.settings = settings
        self.species = species
        self.host = host
        self.nummu_mask = nummu_mask
        self.max_nummu = max_nummu
        self.species_stride = species_stride
        self.max_present = max_present
        self._dev = None
        self._pinned = None

    @property
    def ncol(self):
        return int(self.host["ncol"])

    def n_solves(self):
        """Number of column x frequency solves in the batch."""
        if self.host.get("nfreq") is not None:
            return int(np.sum(self.host["nfreq"]))
        return self.ncol * int(self.host["max_nfreq"])

    def columns(self, arrs):
        return Engine.make_columns(arrs, self.species, nmu_mask=self.nummu_mask, max_present=self.max_present,
                                   species_stride=self.species_stride, max_nummu=self.max_nummu)

    def device_arrays(self, device):
        """Torch CUDA copies of the inputs (cached)."""
        import torch
        if self._dev is None:
            d = dict()
            for k, v in self.host.items():
                if isinstance(v, np.ndarray):
                    d[k] = torch.from_numpy(np.ascontiguousarray(v)).to(device)
                else:
                    d[k] = v
            self._dev = d
        return self._dev

    def pinned_arrays(self):
        """Page-locked host copies of the inputs (cached), for end-to-end runs."""
        import torch
        if self._pinned is None:
            d = dict()
            for k, v in self.host.items():
                if isinstance(v, np.ndarray):
                    t = torch.from_numpy(np.ascontiguousarray(v)).pin_memory()
                    d[k] = t.numpy()
                else:
                    d[k] = v
            self._pinned = (d, None)
        return self._pinned[0]

    def output_shapes(self, ssp=False):
        C, nout = self.ncol, int(self.host["noutlevels"])
        F, N, L = int(self.host["max_nfreq"]), self.max_nummu, int(self.host["max_nlyrs"])
        s = dict(tb=((C, nout, 2 * N, F, 2), np.float64), emissivity=((C, 2, F, N), np.float64),
                 angles_deg=((2 * N,), np.float64), status=((C, F), np.int32))
        if ssp:
            s.update(kextatmo=((C, F, L), np.float64), kexttot=((C, F, L), np.float64),
                     salbedo=((C, F, L), np.float64), num_doubles=((C, F, L), np.int32))
        return s

    def alloc_outputs(self, device=None, ssp=False, pinned=False):
        """Output buffers: torch CUDA tensors (device given) or numpy arrays."""
        out = dict()
        for k, (shape, dt) in self.output_shapes(ssp).items():
            if device is None:
                if pinned:
                    import torch
                    t = torch.empty(shape, dtype=torch.float64 if dt == np.float64 else torch.int32).pin_memory()
                    out[k] = t.numpy()
                else:
                    out[k] = np.zeros(shape, dtype=dt)
            else:
                import torch
                out[k] = torch.zeros(shape, dtype=torch.float64 if dt == np.float64 else torch.int32, device=device)
        return out


def present_per_column(host, species, species_stride):
    """Per column, an upper bound on the layers that can carry hydrometeors
    (presence test of src/hydrometeor_extinction.f90:276-283): every layer of
    a column with a moment_in = 0 species, else the layers with a nonzero or
    NaN hydrometeor input."""
    C, L = int(host["ncol"]), int(host["max_nlyrs"])
    H = int(host["nhydro"])
    if H == 0:
        return np.zeros(C, dtype=np.int64)
    valid = np.arange(L)[None, :] < np.asarray(host["nlyrs"])[:, None]
    sp = np.asarray(species).reshape(C if species_stride else 1, H)
    any_q = np.zeros((C, L), dtype=bool)
    for k in ("hydro_q", "hydro_n", "hydro_reff"):
        a = np.asarray(host[k]).reshape(C, L, H)
        any_q |= np.any((a != 0) | np.isnan(a), axis=-1)
    mom0 = np.any(sp["moment_in"] == 0, axis=1)
    if species_stride:
        any_q |= mom0[:, None]
    elif mom0[0]:
        any_q[:] = True
    return np.sum(any_q & valid, axis=1).astype(np.int64)


def present_layers(host, species, species_stride):
    """Upper bound on the (column, layer) pairs that can carry hydrometeors."""
    return int(np.sum(present_per_column(host, species, species_stride)))


def pack_columns(settings, species, host, species_stride=0):
    """Packed batch from host arrays in the layouts of include/pamtra_b200.h.
    ``host`` may carry per-column ``nummu`` [C] and ``nfreq`` [C] (with
    ``freqs`` [C][max_nfreq]); ``species`` is [H] (shared) or [C*H]
    (``species_stride`` = H)."""
    if host.get("nummu") is not None:
        nmu = np.asarray(host["nummu"])
        mask = int(np.bitwise_or.reduce([_MASK[int(v)] for v in np.unique(nmu)]))
        max_nummu = int(nmu.max())
    else:
        mask, max_nummu = _MASK[int(settings.nummu)], int(settings.nummu)
    mp = present_layers(host, species, species_stride)
    return PackedBatch(settings, species, host, mask, max_nummu, species_stride, mp)


def subset(batch, idxs):
    """A new packed batch holding the columns ``idxs`` of ``batch``, trimmed
    to their own largest layer count and frequency count."""
    idxs = np.asarray(idxs, dtype=np.int64)
    h = batch.host
    C = batch.ncol
    L = int(np.max(np.asarray(h["nlyrs"])[idxs]))
    per_f = h.get("nfreq") is not None
    F = int(np.max(np.asarray(h["nfreq"])[idxs])) if per_f else int(h["max_nfreq"])
    out = dict()
    for k, v in h.items():
        if not isinstance(v, np.ndarray):
            out[k] = v
            continue
        if v.ndim >= 1 and v.shape[0] == C and not (k == "freqs" and not per_f):
            a = v[idxs]
            if k in ("hgt_lev", "temp_lev", "press_lev", "relhum_lev"):
                a = a[:, :L + 1]
            elif k in ("hgt", "temp", "press", "relhum", "hydro_q", "hydro_n", "hydro_reff"):
                a = a[:, :L]
            elif k == "freqs":
                a = a[:, :F]
            out[k] = np.ascontiguousarray(a)
        else:
            out[k] = v
    out["ncol"] = len(idxs)
    out["max_nlyrs"] = L
    out["max_nfreq"] = F
    sp = batch.species
    if batch.species_stride:
        H = batch.species_stride
        sp = np.ascontiguousarray(sp.reshape(C, H)[idxs].reshape(-1))
    return pack_columns(batch.settings, sp, out, batch.species_stride)


def chunk_columns(batch, budget_bytes, max_cols=None):
    """Split the columns of ``batch`` into index groups whose scratch
    (pamtra_b200_workspace_bytes) fits ``budget_bytes``.  Columns are grouped
    by NUMMU first (a batch's layer matrices are strided for its largest
    NUMMU) and ordered by decreasing layer count inside a group, so every
    chunk packs columns of similar size."""
    h = batch.host
    C = batch.ncol
    H = int(h["nhydro"])
    nmu = np.asarray(h["nummu"]) if h.get("nummu") is not None else np.full(C, batch.max_nummu)
    nly = np.asarray(h["nlyrs"]).astype(np.int64)
    nfr = np.asarray(h["nfreq"]).astype(np.int64) if h.get("nfreq") is not None else \
        np.full(C, int(h["max_nfreq"]), dtype=np.int64)
    pres = present_per_column(h, batch.species, batch.species_stride)
    sp_all = batch.species.reshape(C, H) if batch.species_stride else None
    order = np.lexsort((-nly, nmu))

    def need(sel):
        c = Columns()
        c.ncol = len(sel)
        c.max_nlyrs = int(nly[sel].max())
        c.nhydro = H
        c.max_nfreq = int(nfr[sel].max())
        c.noutlevels = int(h["noutlevels"])
        c.max_nummu = int(nmu[sel].max())
        c.max_present = max(1, int(pres[sel].sum()))
        c.nummu_mask = int(np.bitwise_or.reduce([_MASK[int(v)] for v in np.unique(nmu[sel])]))
        if sp_all is not None:
            sp = np.ascontiguousarray(sp_all[sel].reshape(-1))
            c.species_stride = H
        else:
            sp = batch.species
            c.species_stride = 0
        c.species = sp.ctypes.data if len(sp) else None
        return workspace_bytes(c, sp)

    chunks = []
    i = 0
    while i < C:
        group_end = i + int(np.sum(nmu[order[i:]] == nmu[order[i]]))
        cap = group_end - i if max_cols is None else min(group_end - i, max_cols)
        if need(order[i:i + 1]) > budget_bytes:
            raise MemoryError("one column needs more scratch than the budget of %d bytes" % budget_bytes)
        ok, bad = 1, None
        step = 1
        while ok < cap:  # grow geometrically, then bisect
            n_try = min(cap, ok + step)
            if need(order[i:i + n_try]) <= budget_bytes:
                ok = n_try
                step *= 2
            else:
                bad = n_try
                break
        if bad is not None:
            while bad - ok > 1:
                mid = (ok + bad) // 2
                if need(order[i:i + mid]) <= budget_bytes:
                    ok = mid
                else:
                    bad = mid
        chunks.append(np.sort(order[i:i + ok]))
        i += ok
    return chunks


def _per_column(batch):
    """Host arrays of ``batch`` with every per-column field explicit: nummu
    [C], nfreq [C], freqs [C][F] and species [C*H] (stride H)."""
    h = dict(batch.host)
    C, H, F = batch.ncol, int(h["nhydro"]), int(h["max_nfreq"])
    if h.get("nummu") is None:
        h["nummu"] = np.full(C, int(batch.settings.nummu), dtype=np.int32)
    if h.get("nfreq") is None:
        h["nfreq"] = np.full(C, F, dtype=np.int32)
        h["freqs"] = np.tile(np.asarray(h["freqs"], dtype=np.float64)[None, :], (C, 1))
    sp = batch.species
    if not batch.species_stride:
        sp = np.tile(sp, C) if H else sp
    return h, sp


def concat(batches):
    """One packed batch holding the columns of ``batches`` (same settings and
    number of output levels), padded to the largest layer, frequency and
    species counts; missing species slots are disabled.  Returns the batch
    and the first column of each part."""
    parts = [_per_column(b) for b in batches]
    C = sum(b.ncol for b in batches)
    L = max(int(b.host["max_nlyrs"]) for b in batches)
    F = max(int(b.host["max_nfreq"]) for b in batches)
    H = max(int(b.host["nhydro"]) for b in batches)
    nout = int(batches[0].host["noutlevels"])
    if any(int(b.host["noutlevels"]) != nout for b in batches):
        raise ValueError("batches with different numbers of output levels cannot be merged")
    out = dict(ncol=C, max_nlyrs=L, max_nfreq=F, nhydro=H, noutlevels=nout)
    lev = ("hgt_lev", "temp_lev", "press_lev", "relhum_lev")
    lay = ("hgt", "temp", "press", "relhum")
    hyd = ("hydro_q", "hydro_n", "hydro_reff")
    for k in lev:
        out[k] = np.full((C, L + 1), np.nan)
    for k in lay:
        out[k] = np.full((C, L), np.nan)
    for k in hyd:
        out[k] = np.zeros((C, L, H))
    out["freqs"] = np.zeros((C, F))
    for k, dt in (("nlyrs", np.int32), ("nummu", np.int32), ("nfreq", np.int32)):
        out[k] = np.zeros(C, dtype=dt)
    out["groundtemp"] = np.zeros(C)
    out["obs_height"] = np.zeros((C, nout))
    out["sfc_refl"] = np.zeros(C, dtype=np.int8)
    sp = np.empty(C * H, dtype=packing.SPECIES_DTYPE)
    starts = []
    c0 = 0
    dis = packing.disabled_species()
    for b, (h, spb) in zip(batches, parts):
        n, Lb, Fb, Hb = b.ncol, int(h["max_nlyrs"]), int(h["max_nfreq"]), int(h["nhydro"])
        sl = slice(c0, c0 + n)
        for k in lev:
            out[k][sl, :Lb + 1] = h[k]
        for k in lay:
            out[k][sl, :Lb] = h[k]
        for k in hyd:
            out[k][sl, :Lb, :Hb] = np.asarray(h[k]).reshape(n, Lb, Hb)
        out["freqs"][sl, :Fb] = h["freqs"]
        for k in ("nlyrs", "nummu", "nfreq", "groundtemp", "sfc_refl"):
            out[k][sl] = h[k]
        out["obs_height"][sl] = h["obs_height"]
        spv = sp.reshape(C, H) if H else sp.reshape(C, 0)
        if H:
            spv[sl, :] = dis
            if Hb:
                spv[sl, :Hb] = spb.reshape(n, Hb)
        starts.append(c0)
        c0 += n
    return pack_columns(batches[0].settings, sp, out, H), starts


def split_outputs(outs, batches, starts):
    """Per-part views of merged outputs (numpy), in each part's own layout."""
    res = []
    for b, c0 in zip(batches, starts):
        n, F, N = b.ncol, int(b.host["max_nfreq"]), b.max_nummu
        r = dict()
        for k, v in outs.items():
            if k == "tb":
                r[k] = v[c0:c0 + n, :, :2 * N, :F, :]
            elif k == "emissivity":
                r[k] = v[c0:c0 + n, :, :F, :N]
            elif k == "angles_deg":
                r[k] = v
            elif k == "status":
                r[k] = v[c0:c0 + n, :F]
            else:
                r[k] = v[c0:c0 + n, :F, :int(b.host["max_nlyrs"])]
        res.append(r)
    return res


def run_chunked(batch, budget_bytes, device=0, precision=PREC_FP64, stream=None, eng=None, ssp=False):
    """Run a batch of any size as chunks whose scratch fits ``budget_bytes``
    (chunk_columns), one after another on ``stream``; returns numpy outputs
    for all columns in the batch's own layout (unused angle / frequency
    slots hold -9999 in tb)."""
    import torch
    eng = eng or engine(device)
    dev = torch.device("cuda", device)
    full = batch.alloc_outputs(None, ssp=ssp)
    full["tb"][:] = -9999.0
    for idx in chunk_columns(batch, budget_bytes):
        sub = subset(batch, idx)
        out = run(sub, device, sub.alloc_outputs(dev, ssp=ssp), precision, stream, eng)
        if stream is not None:
            stream.synchronize()
        else:
            torch.cuda.synchronize(dev)
        n2, F = 2 * sub.max_nummu, int(sub.host["max_nfreq"])
        L = int(sub.host["max_nlyrs"])
        for k, v in out.items():
            a = v.cpu().numpy()
            if k == "tb":
                full[k][idx, :, :n2, :F, :] = a
            elif k == "emissivity":
                full[k][idx, :, :F, :n2 // 2] = a
            elif k == "angles_deg":
                if sub.max_nummu == batch.max_nummu:
                    full[k][:] = a
            elif k == "status":
                full[k][idx, :F] = a
            else:
                full[k][idx, :F, :L] = a
    if not np.any(full["angles_deg"]):
        full["angles_deg"][:] = np.nan
    return full


def pack_pam(pam, freqs, nummu=16):
    """Pack a pyPamtra session (all grid columns, one frequency list)."""
    st = packing.settings_from_nml(pam.nmlSet, nummu)
    sp = packing.species_from_df(pam.df.data)
    cols = packing.profile_columns(pam.p, len(sp))
    host = libWrapper.host_inputs(cols, freqs)
    mp = libWrapper.present_bound(cols, pam.df.data)
    return PackedBatch(st, sp, host, _MASK[nummu], nummu, 0, mp)


def run(batch, device=0, outputs=None, precision=PREC_FP64, stream=None, eng=None):
    """Run a packed batch with inputs resident on ``device``; returns the
    torch output dict."""
    import torch
    eng = eng or engine(device)
    dev = torch.device("cuda", device)
    arrs = batch.device_arrays(dev)
    out = outputs if outputs is not None else batch.alloc_outputs(dev)
    eng.run(batch.settings, batch.columns(arrs), eng.make_outputs(out), precision, stream)
    return out


def run_host(batch, device=0, outputs=None, precision=PREC_FP64, stream=None, eng=None, pinned=True):
    """End-to-end run from host buffers through the C ABI (copies included)."""
    eng = eng or engine(device)
    arrs = batch.pinned_arrays() if pinned else batch.host
    out = outputs if outputs is not None else batch.alloc_outputs(None, pinned=pinned)
    eng.run_host(batch.settings, batch.columns(arrs), eng.make_outputs(out), precision, stream)
    return out


def capture(batch, device=0, outputs=None, precision=PREC_FP64, stream=None, eng=None):
    """CUDA graph of one batched run (inputs resident on ``device``): replay
    with ``graph.launch(stream)``; the kernels re-read the batch's device
    buffers, so values updated in place give new results.  Returns
    (graph, outputs)."""
    import torch
    eng = eng or engine(device)
    dev = torch.device("cuda", device)
    arrs = batch.device_arrays(dev)
    out = outputs if outputs is not None else batch.alloc_outputs(dev)
    g = eng.capture(batch.settings, batch.columns(arrs), eng.make_outputs(out), precision, stream)
    g._keep = g._keep + (batch, out)
    return g, out
