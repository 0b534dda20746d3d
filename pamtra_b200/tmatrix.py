"""T-matrix scattering of spheroids (scat_name ``'tmatrix'``) on the GPU.

Host-side mirror of the reference's ``calc_tmatrix`` (src/tmatrix.f90:14-433),
the routine ``calc_scatProperties`` calls for a species whose ``scat_name`` is
``tmatrix`` (src/scatProperties.f90:289-306).  The work runs in the native
library (``pamtra_b200_tmatrix``): one CUDA thread block per size bin solves
the spheroid's T-matrix (EBCM, src/tmatrix_amplq.lp.f) in FP64, forms the
amplitude matrices over 30 scattering azimuths at the Lobatto angles, and a
second kernel sums the bins.  There is no CPU path.
"""

import ctypes

import numpy as np

from . import _native

OUT_KEYS = ("scatter_matrix", "extinct_matrix", "emis_vector", "sback", "back_spec", "nmax", "status")


C_LIGHT = 299792458.0


def fp64_envelope(freq, ref_index, phase, dmax, as_ratio):
    """Bins whose T-matrix the FP64 solve reproduces (True), judged by the
    envelope measured against the REAL*16 solve of the reference: every ice
    bin (|m| <= 1.8, all sizes to size parameter 14), and liquid bins of
    equal-volume size parameter x <= 3, or x <= 6 with aspect ratio within
    0.7-1.5.  Arrays [n_items, nbins] for dmax / as_ratio, [n_items] for the
    rest."""
    freq = np.asarray(freq, dtype=np.float64)[:, None]
    m = np.abs(np.asarray(ref_index, dtype=np.complex128))[:, None]
    liquid = (np.asarray(phase)[:, None] == 1)
    dmax = np.asarray(dmax, dtype=np.float64)
    asr = np.asarray(as_ratio, dtype=np.float64)
    axi = np.where(asr <= 1.0, 0.5 * dmax * np.cbrt(asr), 0.5 * dmax / np.maximum(asr, 1e-300) ** (2.0 / 3.0))
    x = 2.0 * np.pi * axi * freq / C_LIGHT
    ok_liquid = (x <= 3.0) | ((x <= 6.0) & (asr >= 0.7) & (asr <= 1.5))
    return ~liquid | (m <= 1.8) | ok_liquid


def _shapes(n_items, nbins, nummu):
    return {"scatter_matrix": (n_items, 2 * nummu * 2 * nummu * 2), "extinct_matrix": (n_items, 4 * nummu),
            "emis_vector": (n_items, 2 * nummu), "sback": (n_items, 4), "back_spec": (n_items, nbins),
            "nmax": (n_items, nbins), "status": (n_items,)}


def calc_tmatrix_batch(freq, ref_index, phase, dmax, del_d, ndens, density, as_ratio, canting, nummu=16,
                       eng=None, stream=None):
    """calc_tmatrix for ``n_items`` (species, layer, frequency) items of
    ``nbins`` bins: ``freq`` (Hz), ``ref_index`` (complex) and ``phase``
    (1 liquid, -1 ice) per item, the bin arrays ``[n_items, nbins]`` (m, m,
    1/m^4, kg/m^3, -, deg).

    numpy inputs run through host buffers (copies in the call); torch CUDA
    tensors stay on the device and the work is queued on ``stream``.
    Returns a dict of flat outputs (see ``_shapes``) with the Fortran element
    order of the reference's arrays inside each item."""
    eng = eng or _native.engine()
    on_dev = not isinstance(dmax, np.ndarray)
    if on_dev:
        import torch
        dev = dmax.device
        f64 = dict(dtype=torch.float64, device=dev)
        n_items, nbins = dmax.shape
        ri = torch.as_tensor(ref_index, device=dev)
        args = {"freq": torch.as_tensor(freq, **f64).contiguous(), "ref_re": ri.real.to(torch.float64).contiguous(),
                "ref_im": ri.imag.to(torch.float64).contiguous(),
                "phase": torch.as_tensor(phase, dtype=torch.int32, device=dev).contiguous()}
        for k, v in (("dmax", dmax), ("del_d", del_d), ("ndens", ndens), ("density", density),
                     ("as_ratio", as_ratio), ("canting", canting)):
            args[k] = torch.as_tensor(v, **f64).reshape(n_items, nbins).contiguous()
        out = {k: torch.zeros(sh, dtype=torch.int32 if k in ("nmax", "status") else torch.float64, device=dev)
               for k, sh in _shapes(n_items, nbins, nummu).items()}
    else:
        dmax = np.asarray(dmax, dtype=np.float64)
        n_items, nbins = dmax.shape
        inside = fp64_envelope(np.asarray(freq).reshape(n_items), np.asarray(ref_index).reshape(n_items),
                               np.asarray(phase).reshape(n_items), dmax,
                               np.asarray(as_ratio, dtype=np.float64).reshape(n_items, nbins))
        occupied = np.asarray(ndens, dtype=np.float64).reshape(n_items, nbins) > 0
        if np.any(~inside & occupied):
            import warnings
            warnings.warn("%d bins lie outside the FP64 envelope of the T-matrix solve (large, aspherical "
                          "liquid drops): their T-matrix departs from the reference's REAL*16 solve"
                          % int(np.count_nonzero(~inside & occupied)), RuntimeWarning)
        ri = np.asarray(ref_index, dtype=np.complex128).reshape(n_items)
        args = {"freq": np.ascontiguousarray(np.asarray(freq, dtype=np.float64).reshape(n_items)),
                "ref_re": np.ascontiguousarray(ri.real), "ref_im": np.ascontiguousarray(ri.imag),
                "phase": np.ascontiguousarray(np.asarray(phase, dtype=np.int32).reshape(n_items))}
        for k, v in (("dmax", dmax), ("del_d", del_d), ("ndens", ndens), ("density", density),
                     ("as_ratio", as_ratio), ("canting", canting)):
            args[k] = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(n_items, nbins))
        out = {k: np.zeros(sh, dtype=np.int32 if k in ("nmax", "status") else np.float64)
               for k, sh in _shapes(n_items, nbins, nummu).items()}
    ti = _native.TmatrixIn()
    ti.n_items, ti.nbins, ti.nummu, ti.on_device = int(n_items), int(nbins), int(nummu), int(on_dev)
    for k, v in args.items():
        setattr(ti, k, _native._ptr(v))
    to = _native.TmatrixOut()
    for k in OUT_KEYS:
        setattr(to, k, _native._ptr(out[k]))
    if stream is None and on_dev:
        import torch
        stream = torch.cuda.current_stream(dmax.device).cuda_stream
    err = eng.lib.pamtra_b200_tmatrix(eng.handle, ctypes.byref(ti), ctypes.byref(to), stream or None)
    if err != 0:
        raise RuntimeError("pamtra_b200_tmatrix failed (%d)" % err)
    out["_keepalive"] = args
    return out


def calc_tmatrix(frequency, ref_index, phase, dmax, del_d, ndens, density, as_ratio, canting, nummu=16, eng=None):
    """calc_tmatrix (src/tmatrix.f90:14) for one species at one frequency, with
    the reference's argument meaning and output shapes: returns
    (scatter_matrix (2, nummu, 2, nummu, 2), extinct_matrix (2, 2, nummu),
    emis_vector (2, nummu), back_spec (nbins,) for radar_pol "NN",
    Sback (2, 2)).  Raises RuntimeError where the reference reports a fatal
    error (invalid bin, NMAX or Gauss-point limit)."""
    o = calc_tmatrix_batch(np.array([frequency]), np.array([ref_index]), np.array([phase]),
                           np.asarray(dmax, dtype=np.float64)[None, :], np.asarray(del_d)[None, :],
                           np.asarray(ndens)[None, :], np.asarray(density)[None, :], np.asarray(as_ratio)[None, :],
                           np.asarray(canting)[None, :], nummu=nummu, eng=eng)
    if int(o["status"][0]) != 0:
        raise RuntimeError("calc_tmatrix: status 0x%x" % int(o["status"][0]))
    return (o["scatter_matrix"][0].reshape((2, nummu, 2, nummu, 2), order="F"),
            o["extinct_matrix"][0].reshape((2, 2, nummu), order="F"),
            o["emis_vector"][0].reshape((2, nummu), order="F"), o["back_spec"][0],
            o["sback"][0].reshape((2, 2), order="F"))


RADAR_POLS = ("NN", "HH", "VV", "HV", "VH")


def back_hydro(sback, radar_pol="NN"):
    """Backscattering of a species per volume (m^-1, before the radar's
    wavelength factors) for one radar polarisation, from its summed Sback
    (2, 2) as the T-matrix branch forms ``back_hydro``
    (src/scatProperties.f90:322-358): "NN" is 4 pi Sback(1,1); "HH", "VV",
    "HV", "VH" take the half sums of Vivekanandan et al. (1991).  ``sback``
    is a (2, 2) array indexed like the Fortran Sback(i, j), or the flat
    four values of the C-ABI in Fortran order."""
    S = np.asarray(sback, dtype=np.float64)
    if S.shape != (2, 2):
        S = S.reshape((2, 2), order="F")
    s11, s12, s21, s22 = S[0, 0], S[0, 1], S[1, 0], S[1, 1]
    if radar_pol == "NN":
        b = s11
    elif radar_pol == "HH":
        b = (s11 - s12 - s21 + s22) * 0.5
    elif radar_pol == "VV":
        b = (s11 + s12 + s21 + s22) * 0.5
    elif radar_pol == "HV":
        b = (s11 - s12 + s21 - s22) * 0.5
    elif radar_pol == "VH":
        b = (s11 + s12 - s21 - s22) * 0.5
    else:
        raise ValueError("do not understand radar_pol: %r" % (radar_pol,))
    return 4 * np.pi * b


def _main(argv=None):
    """``python -m pamtra_b200.tmatrix --items 4 --nbins 32 --reps 2``: soft
    ice spheroids (300 kg/m3, aspect ratio 0.6, 0.2-4 mm, 89 GHz, NUMMU 16)
    from device arrays, ``reps`` calls; prints the status, NMAX range and the
    device time of the last call (a fixed case for profiling)."""
    import argparse
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--items", type=int, default=4)
    ap.add_argument("--nbins", type=int, default=32)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--canting", type=float, default=0.0)
    a = ap.parse_args(argv)
    dev = torch.device("cuda", 0)
    eng = _native.Engine(0)
    d = np.linspace(0.2e-3, 4e-3, a.nbins)[None, :].repeat(a.items, 0)
    t = {k: torch.tensor(v, dtype=torch.float64, device=dev) for k, v in dict(
        dmax=d, del_d=np.full_like(d, 1.2e-4), ndens=np.full_like(d, 1e6), density=np.full_like(d, 300.0),
        as_ratio=np.full_like(d, 0.6), canting=np.full_like(d, a.canting)).items()}
    fr = torch.full((a.items,), 89e9, dtype=torch.float64, device=dev)
    ri = torch.full((a.items,), 1.78 - 0.002j, dtype=torch.complex128, device=dev)
    ph = torch.full((a.items,), -1, dtype=torch.int32, device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(a.reps):
        e0.record()
        o = calc_tmatrix_batch(fr, ri, ph, t["dmax"], t["del_d"], t["ndens"], t["density"], t["as_ratio"],
                               t["canting"], eng=eng)
        e1.record()
    torch.cuda.synchronize()
    nm = o["nmax"].cpu().numpy()
    print("status %d nmax %d-%d ms %.3f" % (int(o["status"].max()), int(nm.min()), int(nm.max()),
                                           e0.elapsed_time(e1)))


if __name__ == "__main__":
    _main()
