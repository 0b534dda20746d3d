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
from ._native import PREC_FP64, Engine, engine

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
