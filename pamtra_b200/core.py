"""pyPamtra-compatible user surface for the passive forward path.

Mirrors the reference's ``pyPamtra`` class (python/pyPamtra/core.py:74):
``nmlSet`` defaults (core.py:89-157), ``set``, ``df`` (descriptor file),
``createProfile`` (core.py:756-977), ``_checkData`` (core.py:979-1000),
``runPamtra`` (core.py:1518-1568) and ``runParallelPamtra`` (core.py:1570),
with results in ``r``.  The native seam underneath is
:func:`pamtra_b200.libWrapper.PamtraFortranWrapper`, which runs the B200
kernels; there is no CPU path.
"""

import calendar
import datetime
import os
import pickle
import time
import warnings
from copy import deepcopy

import numpy as np

from .descriptorFile import pamDescriptorFile

missingNumber = -9999.0
missingIntNumber = int(missingNumber)


class pyPamtra(object):
    """Passive-microwave forward model session.  Same attribute names,
    defaults and result keys as the reference class."""

    def __init__(self):
        self.default_p_vars = ["timestamp", "lat", "lon", "wind10u", "wind10v", "hgt", "press", "temp",
                               "relhum", "hgt_lev", "press_lev", "temp_lev", "relhum_lev", "q", "hydro_q",
                               "hydro_n", "hydro_reff", "wind10u", "wind10v", "obs_height", "ngridy",
                               "ngridx", "max_nlyrs", "nlyrs", "model_i", "model_j", "unixtime", "airturb",
                               "radar_prop", "groundtemp", "wind_w", "wind_uv", "turb_edr", "sfc_type",
                               "sfc_model", "sfc_refl", "sfc_salinity", "sfc_slf", "sfc_sif"]
        n = dict()
        n["hydro_threshold"] = 1.e-10
        n["write_nc"] = True
        n["data_path"] = '$PAMTRA_DATADIR'
        n["save_psd"] = False
        n["save_ssp"] = False
        n["add_obs_height_to_layer"] = False
        n["conserve_mass_rescale_dsd"] = True
        n["outpol"] = 'VH'
        n["file_desc"] = ''
        n["creator"] = 'Pamtrauser'
        n["active"] = True
        n["passive"] = True
        n["radar_mode"] = "simple"
        n["randomseed"] = 0
        n["emissivity"] = 0.6
        n["lgas_extinction"] = True
        n["gas_mod"] = 'R98'
        n["lhyd_absorption"] = True
        n["lhyd_scattering"] = True
        n["lhyd_emission"] = True
        n["liq_mod"] = "TKC"
        n["hydro_includehydroinrhoair"] = True
        n["hydro_fullspec"] = False
        n["hydro_limit_density_area"] = True
        n["hydro_softsphere_min_density"] = 10.
        n["hydro_adaptive_grid"] = True
        n["tmatrix_db"] = "none"
        n["tmatrix_db_path"] = "database/"
        n["radar_nfft"] = 256
        n["radar_no_ave"] = 150
        n["radar_max_v"] = 7.885
        n["radar_min_v"] = -7.885
        n["radar_pnoise0"] = -32.23
        n['radar_allow_negative_dD_dU'] = False
        n["radar_airmotion"] = False
        n["radar_airmotion_model"] = "constant"
        n["radar_airmotion_vmin"] = -4.e0
        n["radar_airmotion_vmax"] = +4.e0
        n["radar_airmotion_linear_steps"] = 30
        n["radar_airmotion_step_vmin"] = 0.5e0
        n["radar_peak_min_bins"] = 2
        n["radar_aliasing_nyquist_interv"] = 1
        n["radar_save_noise_corrected_spectra"] = False
        n["radar_use_hildebrand"] = False
        n["radar_peak_snr_definition"] = 'log'
        n["radar_peak_min_snr"] = -10
        n["radar_convolution_fft"] = True
        n["radar_smooth_spectrum"] = True
        n["radar_k2"] = 0.93
        n["radar_npeaks"] = 1
        n["radar_noise_distance_factor"] = 2.0
        n["radar_receiver_uncertainty_std"] = 0.e0
        n["radar_receiver_miscalibration"] = 0.e0
        n["radar_attenuation"] = "disabled"
        n["radar_polarisation"] = "NN"
        n["radar_use_wider_peak"] = False
        n["radar_integration_time"] = 1.4
        n["radar_fwhr_beamwidth_deg"] = 0.31
        n["liblapack"] = True
        self.nmlSet = n

        self.set = dict()
        self.set["pyVerbose"] = 0
        self.set["verbose"] = 0
        self.set["freqs"] = []
        self.set["namelist_file"] = "TMPFILE"
        self._nmlDefaultSet = deepcopy(self.nmlSet)

        self.units = {"hgt_lev": "m", "temp_lev": "K", "p_lev": "Pa", "relhum_lev": "%",
                      "hydro_q": "kg/kg", "hydro_n": "-", "hydro_reff": "m", "tb": "K", "obs_height": "m"}
        self.dimensions = {"tb": ["gridx", "gridy", "outlevels", "angles", "frequency", "passive_npol"],
                           "hydro_q": ["ngridx", "ngridy", "max_nlyrs", "nhydro"],
                           "hgt_lev": ["ngridx", "ngridy", "max_nlyrs+1"]}

        self._nstokes = 2
        self._nangles = 16

        self.p = dict()
        self.r = dict()
        self.p["ngridx"] = 0
        self.p["ngridy"] = 0
        self.p["max_nlyrs"] = 0
        self._shape2D = (0, 0)
        self._shape3D = (0, 0, 0)
        self.df = pamDescriptorFile(self)

    # ------------------------------------------------------------------ profile
    def createProfile(self, **kwargs):
        """Build ``self.p`` from level (``*_lev``) or layer arrays.  Mandatory:
        ``hgt_lev`` (or ``hgt``), ``temp(_lev)``, ``press(_lev)``,
        ``relhum(_lev)`` [%].  Missing optional fields get the reference's
        defaults (core.py:756-977)."""
        for key in list(kwargs.keys()):
            if isinstance(kwargs[key], np.ma.core.MaskedArray):
                kwargs[key] = kwargs[key].filled(np.nan)
            if isinstance(kwargs[key], np.char.chararray):
                continue
            kwargs[key] = np.array(kwargs[key])

        if not self.df.data.shape[0] > 0:
            warnings.warn("No descriptor file defined. Assuming dry profile without hydrometeors")
        for hk in ("hydro_q", "hydro_n", "hydro_reff"):
            if hk in kwargs:
                assert self.df.data.shape[0] > 0
                assert self.df.nhydro == kwargs[hk].shape[-1]
                break

        if 'lfrac' in kwargs:
            if 'sfc_type' in kwargs or 'sfc_refl' in kwargs:
                raise DeprecationWarning('Using lfrac and sfc_type/sfc_refl at the same time is not allowed.')
            kwargs['sfc_type'] = np.around(kwargs['lfrac'])
            kwargs['sfc_refl'] = np.char.chararray(kwargs['sfc_type'].shape)
            kwargs['sfc_refl'][kwargs['sfc_type'] == 0] = 'F'
            kwargs['sfc_refl'][kwargs['sfc_type'] == 1] = 'S'
            kwargs.pop('lfrac')

        for key in kwargs:
            if (key not in self.default_p_vars and key.split("+")[0] not in self.default_p_vars) or \
                    key in ("model_i", "model_j"):
                raise TypeError("Could not parse " + key)

        keys = kwargs.keys()
        if not (("hgt_lev" in keys or "hgt" in keys) and ("temp_lev" in keys or "temp" in keys) and
                ("press_lev" in keys or "press" in keys) and ("relhum_lev" in keys or "relhum" in keys)):
            raise TypeError("I need hgt(_lev) and temp(_lev) and press(_lev) and relhum(_lev)!")

        if "hgt" not in kwargs:
            kwargs["hgt"] = (kwargs["hgt_lev"][..., 1:] + kwargs["hgt_lev"][..., :-1]) / 2.

        noDims = len(np.shape(kwargs["hgt"]))
        if noDims == 1:
            self.p["ngridx"], self.p["ngridy"] = 1, 1
        elif noDims == 2:
            self.p["ngridx"], self.p["ngridy"] = np.shape(kwargs["hgt"])[0], 1
        elif noDims == 3:
            self.p["ngridx"], self.p["ngridy"] = np.shape(kwargs["hgt"])[0], np.shape(kwargs["hgt"])[1]
        else:
            raise IOError("Too many dimensions!")

        self.p["max_nlyrs"] = np.shape(kwargs["hgt"])[-1]
        self.p["nlyrs"] = np.array(np.sum(kwargs["hgt"] != missingNumber, axis=-1))
        try:
            self.p["noutlevels"] = np.shape(kwargs["obs_height"])[-1]
        except (KeyError, IndexError):
            self.p["noutlevels"] = 2

        nx, ny, nl = self.p["ngridx"], self.p["ngridy"], self.p["max_nlyrs"]
        self._shape2D = (nx, ny)
        self._shape3D = (nx, ny, nl)
        self._shape3Dout = (nx, ny, self.p["noutlevels"])
        self._shape3Dplus = (nx, ny, nl + 1)
        self._shape4D = (nx, ny, nl, self.df.nhydro)

        self.p["nlyrs"] = self.p["nlyrs"].reshape(self._shape2D)
        for key in ["hgt_lev", "temp_lev", "press_lev", "relhum_lev"]:
            if key in kwargs:
                self.p[key] = kwargs[key].reshape(self._shape3Dplus).astype(float)
        for key in ["hgt", "temp", "press", "relhum"]:
            if key in kwargs:
                self.p[key] = kwargs[key].reshape(self._shape3D).astype(float)
        if "hgt_lev" not in kwargs:
            h = self.p["hgt"]
            hl = np.empty(self._shape3Dplus)
            hl[..., 0] = h[..., 0] - (h[..., 1] - h[..., 0]) * 0.5
            hl[..., 1:-1] = 0.5 * (h[..., :-1] + h[..., 1:])
            hl[..., -1] = h[..., -1] + (h[..., -1] - h[..., -2]) * 0.5
            self.p["hgt_lev"] = hl

        idx = np.where(np.logical_not(np.isnan(self.p["hgt"][:, :, 0])))
        self.p["model_i"] = np.array(idx[0]).reshape(self._shape2D) + 1
        self.p["model_j"] = np.array(idx[1]).reshape(self._shape2D) + 1

        if "timestamp" not in kwargs:
            self.p["unixtime"] = np.ones(self._shape2D) * int(time.time())
        else:
            ts = kwargs["timestamp"]
            if isinstance(ts, datetime.datetime):
                self.p["unixtime"] = np.ones(self._shape2D, dtype=int) * calendar.timegm(ts.timetuple())
            elif np.ndim(ts) == 0:
                self.p["unixtime"] = np.ones(self._shape2D, dtype=int) * ts
            else:
                self.p["unixtime"] = np.asarray(ts).reshape(self._shape2D)

        for env, preset in [["lat", 50.938056], ["lon", 6.956944], ["wind10u", 0], ["wind10v", 0],
                            ["groundtemp", np.nan], ["sfc_salinity", 33.], ["sfc_slf", 1.], ["sfc_sif", 0.]]:
            if env not in kwargs:
                self.p[env] = np.ones(self._shape2D) * preset
            elif np.ndim(kwargs[env]) == 0:
                self.p[env] = np.ones(self._shape2D) * kwargs[env]
            else:
                self.p[env] = kwargs[env].reshape(self._shape2D)
        for env, preset in [["sfc_type", -9999], ["sfc_model", -9999]]:
            if env not in kwargs:
                self.p[env] = np.ones(self._shape2D, dtype=int) * preset
            elif np.ndim(kwargs[env]) == 0:
                self.p[env] = np.ones(self._shape2D) * kwargs[env]
            else:
                self.p[env] = kwargs[env].reshape(self._shape2D)
        if "sfc_refl" not in kwargs:
            self.p["sfc_refl"] = np.char.chararray(self._shape2D)
            self.p["sfc_refl"][:] = 'S'
        elif isinstance(kwargs["sfc_refl"], str) or np.ndim(kwargs["sfc_refl"]) == 0:
            self.p["sfc_refl"] = np.char.chararray(self._shape2D)
            self.p["sfc_refl"][:] = str(kwargs["sfc_refl"])
        else:
            self.p["sfc_refl"] = np.asarray(kwargs["sfc_refl"]).reshape(self._shape2D)
        if "obs_height" not in kwargs:
            self.p["obs_height"] = np.ones(self._shape3Dout) * np.array([833000., 0.])
        elif np.ndim(kwargs["obs_height"]) == 0:
            self.p["obs_height"] = np.ones(self._shape3Dout) * kwargs["obs_height"]
        else:
            self.p["obs_height"] = kwargs["obs_height"].reshape(self._shape3Dout).astype(float)

        for qValue in ["hydro_q", "hydro_reff", "hydro_n"]:
            if qValue not in kwargs and qValue + "+no000" not in kwargs:
                self.p[qValue] = np.zeros(self._shape4D)
            elif qValue + "+no000" in kwargs:
                self.p[qValue] = np.zeros(self._shape4D)
                for hh in range(self.df.nhydro):
                    self.p[qValue][..., hh] = kwargs[qValue + "+no" + str(hh).zfill(3)].reshape(self._shape3D)
            else:
                self.p[qValue] = kwargs[qValue].reshape(self._shape4D).astype(float)
        for qValue in ["airturb", "wind_w", "wind_uv", "turb_edr"]:
            if qValue not in kwargs:
                self.p[qValue] = np.zeros(self._shape3D) + np.nan
            else:
                self.p[qValue] = kwargs[qValue].reshape(self._shape3D)
        if "radar_prop" in kwargs:
            self.p["radar_prop"] = kwargs["radar_prop"].reshape(self._shape2D + (2,))
        else:
            self.p["radar_prop"] = np.zeros(self._shape2D + (2,)) * np.nan

    def _checkData(self):
        """Range checks on the profile (core.py:979-1000); raises ValueError."""
        maxLimits = {"relhum_lev": 200, "hydro_q": 0.05, "temp_lev": 320, "press_lev": 110000,
                     "relhum": 200, "temp": 320, "press": 110000}
        minLimits = {"relhum_lev": 0, "hydro_q": 0, "temp_lev": 160, "press_lev": 1,
                     "relhum": 0, "temp": 160, "press": 1}
        for key in self.p.keys():
            if type(self.p[key]) != np.ndarray or key in ("sfc_refl",):
                continue
            if not np.issubdtype(self.p[key].dtype, np.number):
                continue
            d = self.p[key][~np.isnan(self.p[key])]
            if key in maxLimits and len(d) > 0 and np.max(d) > maxLimits[key]:
                raise ValueError("unrealistic value for " + key + ": " + str(np.max(d)) +
                                 ", maximum is " + str(maxLimits[key]))
            if key in minLimits and len(d) > 0:
                dd = d[d != missingNumber]
                if len(dd) > 0 and np.min(dd) < minLimits[key]:
                    raise ValueError("unrealistic value for " + key + ": " + str(np.min(d)) +
                                     ", minimum is " + str(minLimits[key]))
        refl = np.asarray(self.p['sfc_refl']).astype(str)
        if np.any(refl[self.p['sfc_type'] == 0] == 'L'):
            raise ValueError("It does not make sense to treat Ocean as Lambertian reflector "
                             "(incompatible sfc_refl and sfc_type).")
        if np.any(refl[self.p['sfc_type'] == 1] == 'F'):
            raise ValueError("It does not make sense to simulate land with Fresnel reflection "
                             "(incompatible sfc_refl and sfc_type).")

    # ------------------------------------------------------------------ run
    def _prepare_freqs(self, freqs):
        if type(freqs) in (int, np.int32, np.int64, float, np.float32, np.float64):
            freqs = [freqs]
        self.set["freqs"] = freqs
        self.set["nfreqs"] = len(freqs)
        self.set["radar_pol"] = self.nmlSet["radar_polarisation"].split(",")
        self.set["radar_npol"] = len(self.set["radar_pol"])
        self.set["att_pol"] = ["N"]
        self.set["att_npol"] = 1
        assert self.set["nfreqs"] > 0
        return freqs

    def runPamtra(self, freqs, checkData=True, failOnError=True):
        """Run the passive forward model for sorted ``freqs`` [GHz] and fill
        ``self.r`` (core.py:1518-1568).  Raises RuntimeError when the native
        run reports an error and ``failOnError`` is set."""
        t0 = time.time()
        freqs = self._prepare_freqs(freqs)
        assert np.array_equal(np.sort(freqs), freqs)
        assert self.p["noutlevels"] > 0
        assert np.prod(self._shape2D) > 0
        if checkData:
            self._checkData()
        if self.nmlSet["add_obs_height_to_layer"]:
            raise NotImplementedError("add_obs_height_to_layer is not supported on the passive path")
        from .libWrapper import PamtraFortranWrapper
        results, self.fortError, fortObject = PamtraFortranWrapper(
            self.set, self.nmlSet, self.df.data, self.df.data4D, self.df.dataFullSpec, self.p)
        if failOnError and (self.fortError != 0):
            raise RuntimeError('Fortran code failed')
        self.r = results
        self.fortObject = fortObject
        self.r["nmlSettings"] = self.nmlSet
        if self.set["pyVerbose"] > 0:
            print("pyPamtra runtime:", time.time() - t0)

    def runParallelPamtra(self, freqs, pp_local_workers="auto", pp_deltaF=1, pp_deltaX=0, pp_deltaY=0,
                          checkData=True, timeout=None):
        """The reference farms (column, frequency) chunks to CPU processes
        (core.py:1570-1676).  Here all columns and frequencies are one batched
        GPU launch sequence; the chunking arguments are accepted for
        compatibility and ignored."""
        self.runPamtra(freqs, checkData=checkData, failOnError=False)

    # ------------------------------------------------------------------ results I/O
    def writeResultsToNumpy(self, fname, seperateFiles=False):
        """Pickle ``r``, ``p`` and settings (core.py:2072)."""
        with open(fname, "wb") as f:
            pickle.dump({"r": self.r, "p": self.p, "nmlSet": self.nmlSet, "set": self.set,
                         "df": self.df.data}, f)

    def loadResultsFromNumpy(self, fname):
        """Inverse of :meth:`writeResultsToNumpy` (core.py:2116)."""
        with open(fname, "rb") as f:
            d = pickle.load(f)
        self.r, self.p, self.nmlSet, self.set = d["r"], d["p"], d["nmlSet"], d["set"]
        self.df.data = d["df"]
        self.df.nhydro = len(d["df"])

    def dumpForRT4(self, runFile, path, prefix="sca_"):
        """Write the input files of Frank Evans' stand-alone RT4 program for
        profile (0, 0) after a run with ``nmlSet['save_ssp']`` at 16 angles
        (core.py:2595-2697): ``runFile`` lists, from the top level down, the
        level height (km), level temperature (K), gas extinction of the layer
        below (1/km) and the name of that layer's scattering file, which
        ``path`` receives (``prefix`` + 3-digit layer index) with the phase
        matrices, extinction matrices and emission vectors in RT4's Lobatto
        layout, all per km.  As in the reference, the level-0 line takes its
        scattering file from index -1 (the top layer) and a layer gets a file
        when any of its hydrometeor mixing ratios is nonzero."""
        os.makedirs(path, exist_ok=True)
        N = 16
        mu = np.cos(np.deg2rad(self.r["angles_deg"][N:]))
        nlev = self._shape3Dplus[2]
        ge = np.zeros(nlev)
        ge[1:nlev] = self.r["kextatmo"] * 1.e3
        sm = self.r["scatter_matrix"] * 1.e3   # (L, 2, N, 2, N, 4)
        em = self.r["extinct_matrix"] * 1.e3   # (L, 2, 2, N, 2)
        ev = self.r["emis_vector"] * 1.e3      # (L, 2, N, 2)
        e = lambda x: "%.12e" % x
        m = lambda x: "%.9f" % x
        zero = e(0.0)
        zrow = " ".join([zero] * 4) + "\n"

        def row4(a, b):
            return e(a) + " " + e(b) + " " + zero + " " + zero + "\n"

        lines = []
        for zz in range(nlev - 1, -1, -1):
            lay = zz - 1   # the layer below level zz (-1 at the bottom level, as the reference indexes)
            if np.all(self.p["hydro_q"][0, 0, lay] == 0.):
                scat_file = " " * 12
            else:
                scat_file = prefix + "%03d" % lay + ".txt"
                out = ["  16   0 'LOBATTO        '\n\n"]
                # phase matrix blocks: (outgoing sign, incoming sign) -> quadrant
                for si, quads in ((1.0, ((1.0, 0), (-1.0, 2))), (-1.0, ((1.0, 1), (-1.0, 3)))):
                    for i in range(N):
                        for sj, q in quads:
                            for j in range(N):
                                out.append(m(si * mu[i]) + "    " + m(sj * mu[j]) + "    0\n")
                                for k in range(2):
                                    out.append(row4(sm[lay, k, j, 0, i, q], sm[lay, k, j, 1, i, q]))
                                out.append(zrow)
                                out.append(zrow)
                out.append("\n")
                for h, sh in ((0, 1.0), (1, -1.0)):
                    for i in range(N):
                        out.append(m(sh * mu[i]) + "\n")
                        for k in range(2):
                            out.append(row4(em[lay, k, 0, i, h], em[lay, k, 1, i, h]))
                        out.append(zrow)
                        out.append(zrow)
                out.append("\n")
                for h, sh in ((0, 1.0), (1, -1.0)):
                    for i in range(N):
                        out.append(m(sh * mu[i]) + "  " + row4(ev[lay, 0, i, h], ev[lay, 1, i, h]))
                with open(os.path.join(path, scat_file), "w") as sf:
                    sf.write("".join(out))
            lines.append("%3.2f" % (self.p["hgt_lev"][0, 0, zz] / 1.e3) + " " + "%3.2f" % self.p["temp_lev"][0, 0, zz] +
                         " " + "%3.6f" % ge[zz] + "  '" + scat_file + "'\n")
        with open(runFile, "w") as f:
            f.write("".join(lines))
