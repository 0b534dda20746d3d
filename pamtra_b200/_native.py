"""ctypes binding of the C ABI in include/pamtra_b200.h.

The shared library is built in-tree (pamtra_b200/_lib/libpamtra_b200.so) by
:func:`pamtra_b200.build.build`.  There is no fallback: if the library or a
CUDA device is missing, loading raises.
"""

import ctypes
import os

import numpy as np

from .packing import Settings, Species, SPECIES_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpamtra_b200.so")

PREC_FP64 = 0           # reference operation order (plain drop-in)
PREC_3XTF32 = 1         # batched: 3xTF32 tensor-core doubling and (NUMMU 16) adding, FP64 inverses
PREC_FP64_BATCHED = 2   # batched: FP64, one-inverse adding
PREC_3XTF32_FP64ADD = 3  # batched: 3xTF32 doubling, FP64 one-inverse adding

ST_NORM = 0x100
ST_PSD = 0x200
ST_MIE = 0x400
ST_GAS = 0x800
ST_PIVOT = 0x1000
ST_NAN = 0x2000
ST_SIZE = 0x4000
ST_TIMEOUT = 0x8000
ST_RANGE = 0x10000
WAIT_LIMIT_DEFAULT = 1 << 24  # PAMTRA_B200_WAIT_LIMIT_DEFAULT

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32


class Columns(ctypes.Structure):
    """Mirror of ``pamtra_b200_columns``."""
    _fields_ = [("ncol", _i32), ("max_nlyrs", _i32), ("nhydro", _i32), ("max_nfreq", _i32),
                ("noutlevels", _i32), ("max_nummu", _i32), ("species_stride", _i32), ("max_present", _i32),
                ("nummu_mask", _i32), ("species", _vp), ("nlyrs", _vp), ("nummu", _vp), ("nfreq", _vp),
                ("freqs", _vp), ("hgt_lev", _vp), ("temp_lev", _vp), ("press_lev", _vp), ("relhum_lev", _vp),
                ("hgt", _vp), ("temp", _vp), ("press", _vp), ("relhum", _vp), ("hydro_q", _vp),
                ("hydro_n", _vp), ("hydro_reff", _vp), ("groundtemp", _vp), ("obs_height", _vp),
                ("sfc_refl", _vp), ("fs_nbin", _i32), ("fs_d", _vp), ("fs_d_bound", _vp), ("fs_n", _vp),
                ("fs_rho", _vp), ("fs_mass", _vp)]


class Outputs(ctypes.Structure):
    """Mirror of ``pamtra_b200_outputs``."""
    _fields_ = [("tb", _vp), ("emissivity", _vp), ("angles_deg", _vp), ("status", _vp), ("kextatmo", _vp),
                ("kexttot", _vp), ("salbedo", _vp), ("scatter_matrix", _vp), ("num_doubles", _vp),
                ("ze", _vp), ("att_hydro", _vp), ("att_atmo", _vp), ("psd_nbin", _i32), ("psd_d", _vp),
                ("psd_deltad", _vp), ("psd_n", _vp), ("psd_mass", _vp), ("psd_area", _vp), ("psd_bscat", _vp)]


EXPORTS = ["pamtra_b200_create", "pamtra_b200_destroy", "pamtra_b200_workspace_bytes", "pamtra_b200_reserve",
           "pamtra_b200_run", "pamtra_b200_run_host", "pamtra_b200_last_launch_count", "pamtra_b200_gas_r98",
           "pamtra_b200_eps_water_tkc", "pamtra_b200_minvert_batched", "pamtra_b200_set_timing",
           "pamtra_b200_stage_ms", "pamtra_b200_abi_sizes", "pamtra_b200_run_noalloc",
           "pamtra_b200_mmult_3xtf32_batched", "pamtra_b200_set_launch", "pamtra_b200_get_launch",
           "pamtra_b200_graph_capture", "pamtra_b200_graph_launch", "pamtra_b200_graph_destroy",
           "pamtra_b200_get_eps_water", "pamtra_b200_gas_l93", "pamtra_b200_set_wait_limit",
           "pamtra_b200_layer_products", "pamtra_b200_tmatrix"]
NLAUNCH = 5  # PAMTRA_B200_NLAUNCH: mie warps per CTA, mie / layer / adding CTAs per SM, mie bins per item
STAGES = ["prep", "psd", "mie", "layer", "adding"]

_lib = None


class TmatrixIn(ctypes.Structure):
    _fields_ = [("n_items", ctypes.c_int32), ("nbins", ctypes.c_int32), ("nummu", ctypes.c_int32),
                ("on_device", ctypes.c_int32)] + \
        [(k, ctypes.c_void_p) for k in ("freq", "ref_re", "ref_im", "phase", "dmax", "del_d", "ndens", "density",
                                        "as_ratio", "canting")]


class TmatrixOut(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in ("scatter_matrix", "extinct_matrix", "emis_vector", "sback",
                                               "back_spec", "nmax", "status")]


def load():
    """Load the shared library (raises OSError if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("pamtra_b200 native library not built: %s (run pamtra_b200.build.build())" % LIB_PATH)
        l = ctypes.CDLL(LIB_PATH)
        l.pamtra_b200_create.restype = _i32
        l.pamtra_b200_create.argtypes = [_i32, ctypes.POINTER(_vp)]
        l.pamtra_b200_destroy.restype = _i32
        l.pamtra_b200_destroy.argtypes = [_vp]
        l.pamtra_b200_workspace_bytes.restype = ctypes.c_size_t
        l.pamtra_b200_workspace_bytes.argtypes = [ctypes.POINTER(Columns), _i32]
        l.pamtra_b200_reserve.restype = _i32
        l.pamtra_b200_reserve.argtypes = [_vp, ctypes.c_size_t]
        for fn in (l.pamtra_b200_run, l.pamtra_b200_run_host):
            fn.restype = _i32
            fn.argtypes = [_vp, ctypes.POINTER(Settings), ctypes.POINTER(Columns), ctypes.POINTER(Outputs), _i32, _vp]
        l.pamtra_b200_last_launch_count.restype = _i32
        l.pamtra_b200_last_launch_count.argtypes = [_vp]
        l.pamtra_b200_gas_r98.restype = _i32
        l.pamtra_b200_gas_r98.argtypes = [_vp] * 6 + [_i32, _vp]
        l.pamtra_b200_eps_water_tkc.restype = _i32
        l.pamtra_b200_eps_water_tkc.argtypes = [_vp] * 4 + [_i32, _vp]
        l.pamtra_b200_get_eps_water.restype = _i32
        l.pamtra_b200_get_eps_water.argtypes = [_i32] + [_vp] * 6 + [_i32, _vp]
        l.pamtra_b200_gas_l93.restype = _i32
        l.pamtra_b200_gas_l93.argtypes = [_vp] * 5 + [_i32, _vp]
        l.pamtra_b200_minvert_batched.restype = _i32
        l.pamtra_b200_minvert_batched.argtypes = [_vp, _vp, _vp, _i32, _i32, _vp]
        l.pamtra_b200_set_timing.restype = _i32
        l.pamtra_b200_set_timing.argtypes = [_vp, _i32]
        l.pamtra_b200_stage_ms.restype = _i32
        l.pamtra_b200_stage_ms.argtypes = [_vp, ctypes.POINTER(ctypes.c_float), _i32]
        l.pamtra_b200_run_noalloc.restype = _i32
        l.pamtra_b200_run_noalloc.argtypes = [ctypes.POINTER(Settings), ctypes.POINTER(Columns),
                                              ctypes.POINTER(Outputs), _vp]
        l.pamtra_b200_mmult_3xtf32_batched.restype = _i32
        l.pamtra_b200_mmult_3xtf32_batched.argtypes = [_vp, _vp, _vp, _i32, _i32, _vp, _vp]
        l.pamtra_b200_set_launch.restype = _i32
        l.pamtra_b200_set_launch.argtypes = [_vp, ctypes.POINTER(_i32), _i32]
        l.pamtra_b200_get_launch.restype = _i32
        l.pamtra_b200_get_launch.argtypes = [_vp, ctypes.POINTER(_i32), _i32]
        l.pamtra_b200_graph_capture.restype = _i32
        l.pamtra_b200_graph_capture.argtypes = [_vp, ctypes.POINTER(Settings), ctypes.POINTER(Columns),
                                                ctypes.POINTER(Outputs), _i32, _vp, ctypes.POINTER(_vp)]
        l.pamtra_b200_graph_launch.restype = _i32
        l.pamtra_b200_graph_launch.argtypes = [_vp, _vp]
        l.pamtra_b200_graph_destroy.restype = _i32
        l.pamtra_b200_graph_destroy.argtypes = [_vp]
        l.pamtra_b200_set_wait_limit.restype = _i32
        l.pamtra_b200_set_wait_limit.argtypes = [_vp, ctypes.c_uint32]
        l.pamtra_b200_layer_products.restype = _i32
        l.pamtra_b200_layer_products.argtypes = [_vp, ctypes.POINTER(ctypes.c_uint64), _vp]
        l.pamtra_b200_tmatrix.restype = _i32
        l.pamtra_b200_tmatrix.argtypes = [_vp, ctypes.POINTER(TmatrixIn), ctypes.POINTER(TmatrixOut), _vp]
        l.pamtra_b200_abi_sizes.restype = _i32
        l.pamtra_b200_abi_sizes.argtypes = [ctypes.POINTER(ctypes.c_size_t), _i32]
        _lib = l
    return _lib


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


class Engine(object):
    """A native context on one CUDA device."""

    def __init__(self, device=0):
        self.lib = load()
        h = _vp()
        err = self.lib.pamtra_b200_create(int(device), ctypes.byref(h))
        if err != 0:
            raise RuntimeError("pamtra_b200_create failed (%d): no usable CUDA device?" % err)
        self.handle = h
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pamtra_b200_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def make_columns(arrs, species, nmu_mask=0, max_present=0, species_stride=0, max_nummu=16):
        """Columns struct from a dict of arrays (numpy for host runs, torch CUDA
        tensors for device runs).  ``species`` is always a host structured array."""
        c = Columns()
        c.ncol = int(arrs["ncol"])
        c.max_nlyrs = int(arrs["max_nlyrs"])
        c.nhydro = int(arrs["nhydro"])
        c.max_nfreq = int(arrs["max_nfreq"])
        c.noutlevels = int(arrs["noutlevels"])
        c.max_nummu = int(max_nummu)
        c.species_stride = int(species_stride)
        c.max_present = int(max_present)
        c.nummu_mask = int(nmu_mask)
        c.species = species.ctypes.data if len(species) else None
        for k in ("nlyrs", "nummu", "nfreq", "freqs", "hgt_lev", "temp_lev", "press_lev", "relhum_lev", "hgt",
                  "temp", "press", "relhum", "hydro_q", "hydro_n", "hydro_reff", "groundtemp", "obs_height",
                  "sfc_refl", "fs_d", "fs_d_bound", "fs_n", "fs_rho", "fs_mass"):
            setattr(c, k, _ptr(arrs.get(k)))
        c.fs_nbin = int(arrs.get("fs_nbin", 0))
        return c

    @staticmethod
    def make_outputs(outs):
        o = Outputs()
        for k in ("tb", "emissivity", "angles_deg", "status", "kextatmo", "kexttot", "salbedo", "scatter_matrix",
                  "num_doubles", "ze", "att_hydro", "att_atmo", "psd_d", "psd_deltad", "psd_n", "psd_mass",
                  "psd_area", "psd_bscat"):
            setattr(o, k, _ptr(outs.get(k)))
        if outs.get("psd_d") is not None:
            o.psd_nbin = int(outs["psd_d"].shape[-1])
        return o

    def run(self, settings, columns, outputs, precision=PREC_FP64, stream=None):
        """Device-pointer run on ``stream`` (a torch.cuda.Stream or None)."""
        s = None if stream is None else stream.cuda_stream
        err = self.lib.pamtra_b200_run(self.handle, ctypes.byref(settings), ctypes.byref(columns),
                                       ctypes.byref(outputs), int(precision), s)
        if err != 0:
            raise RuntimeError("pamtra_b200_run failed with code %d" % err)

    def run_host(self, settings, columns, outputs, precision=PREC_FP64, stream=None):
        """Host-pointer run: copies in, computes, copies out, synchronises."""
        s = None if stream is None else stream.cuda_stream
        err = self.lib.pamtra_b200_run_host(self.handle, ctypes.byref(settings), ctypes.byref(columns),
                                            ctypes.byref(outputs), int(precision), s)
        if err != 0:
            raise RuntimeError("pamtra_b200_run_host failed with code %d" % err)

    def set_launch(self, params):
        """Launch shapes of the persistent kernels: (mie warps per CTA, mie /
        layer / adding CTAs per SM, mie bins per work item), 0 = default."""
        arr = (_i32 * NLAUNCH)(*[int(v) for v in params])
        if self.lib.pamtra_b200_set_launch(self.handle, arr, len(params)) != 0:
            raise ValueError("invalid launch shape %r" % (tuple(params),))

    def get_launch(self):
        arr = (_i32 * NLAUNCH)()
        self.lib.pamtra_b200_get_launch(self.handle, arr, NLAUNCH)
        return tuple(int(v) for v in arr)

    def capture(self, settings, columns, outputs, precision=PREC_FP64, stream=None):
        """Run once on ``stream`` and capture the same call as a CUDA graph
        (see :class:`Graph`).  The structs' buffers must stay alive and in
        place while the graph is used."""
        s = None if stream is None else stream.cuda_stream
        g = _vp()
        err = self.lib.pamtra_b200_graph_capture(self.handle, ctypes.byref(settings), ctypes.byref(columns),
                                                 ctypes.byref(outputs), int(precision), s, ctypes.byref(g))
        if err != 0 or not g:
            raise RuntimeError("pamtra_b200_graph_capture failed with code %d" % err)
        return Graph(self, g, (settings, columns, outputs))

    def reserve(self, nbytes):
        if self.lib.pamtra_b200_reserve(self.handle, int(nbytes)) != 0:
            raise MemoryError("cannot reserve %d bytes of device scratch" % nbytes)

    def workspace_bytes(self, columns, precision=PREC_FP64):
        return workspace_bytes(columns, precision=precision)

    def last_launch_count(self):
        return int(self.lib.pamtra_b200_last_launch_count(self.handle))

    def set_wait_limit(self, polls=WAIT_LIMIT_DEFAULT):
        """Polls of each wait on a tensor-core MMA before it gives up
        (status ST_TIMEOUT); 0 gives up at once."""
        if self.lib.pamtra_b200_set_wait_limit(self.handle, int(polls)) != 0:
            raise RuntimeError("pamtra_b200_set_wait_limit failed")

    def layer_products(self, stream=None):
        """n x n products the FP64 doubling kernels of the last run issued."""
        v = ctypes.c_uint64(0)
        s = None if stream is None else stream.cuda_stream
        if self.lib.pamtra_b200_layer_products(self.handle, ctypes.byref(v), s) != 0:
            raise RuntimeError("pamtra_b200_layer_products failed")
        return int(v.value)

    def set_timing(self, on):
        self.lib.pamtra_b200_set_timing(self.handle, int(bool(on)))

    def stage_ms(self):
        """Milliseconds per stage of the last run (needs set_timing(True))."""
        buf = (ctypes.c_float * len(STAGES))()
        self.lib.pamtra_b200_stage_ms(self.handle, buf, len(STAGES))
        return dict(zip(STAGES, [float(v) for v in buf]))


class Graph(object):
    """A captured launch sequence of one batch (pamtra_b200_graph_*)."""

    def __init__(self, eng, handle, keep):
        self.eng = eng
        self.handle = handle
        self._keep = keep  # the structs whose pointers the graph holds

    def launch(self, stream=None):
        s = None if stream is None else stream.cuda_stream
        err = self.eng.lib.pamtra_b200_graph_launch(self.handle, s)
        if err != 0:
            raise RuntimeError("pamtra_b200_graph_launch failed with code %d (arena regrown? capture again)" % err)

    def close(self):
        if getattr(self, "handle", None):
            self.eng.lib.pamtra_b200_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def workspace_bytes(columns, species=None, precision=PREC_FP64):
    """Scratch bytes a batch needs (pamtra_b200_workspace_bytes; no device
    work).  ``species`` only keeps the array behind columns.species alive."""
    del species
    return int(load().pamtra_b200_workspace_bytes(ctypes.byref(columns), int(precision)))


def abi_sizes():
    """(settings, species, columns, outputs, tmatrix_in, tmatrix_out) struct
    sizes as compiled."""
    buf = (ctypes.c_size_t * 6)()
    load().pamtra_b200_abi_sizes(buf, 6)
    return tuple(int(v) for v in buf)


_engines = {}


def engine(device=0):
    """Process-wide engine per device."""
    if device not in _engines:
        _engines[device] = Engine(device)
    return _engines[device]
