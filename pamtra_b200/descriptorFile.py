"""Hydrometeor descriptor file, same columns and semantics as the reference's
``pamDescriptorFile`` (python/pyPamtra/descriptorFile.py:12-240).

A descriptor row has 20 fields:
hydro_name, as_ratio, liq_ice, rho_ms, a_ms, b_ms, alpha_as, beta_as,
moment_in, nbin, dist_name, p_1, p_2, p_3, p_4, d_1, d_2, scat_name,
vel_size_mod, canting.
"""

import csv

import numpy as np

missingNumber = -9999.0

NAMES = ["hydro_name", "as_ratio", "liq_ice", "rho_ms", "a_ms", "b_ms", "alpha_as", "beta_as",
         "moment_in", "nbin", "dist_name", "p_1", "p_2", "p_3", "p_4", "d_1", "d_2", "scat_name",
         "vel_size_mod", "canting"]
TYPES = ["U15", float, int, float, float, float, float, float, int, int, "U15", float, float, float,
         float, float, float, "U60", "U30", float]


class pamDescriptorFile(object):
    """Descriptor table of the hydrometeor species of a :class:`pyPamtra` run.

    Mirrors python/pyPamtra/descriptorFile.py:12 (``data`` recarray, ``data4D``
    and ``dataFullSpec`` dicts, ``nhydro``).
    """

    def __init__(self, parent):
        self.names = np.array(NAMES)
        self.types = TYPES
        self.data = np.recarray((0,), dtype=list(zip(self.names, self.types)))
        self.data4D = dict()
        self.nhydro = 0
        self.parent = parent
        self.dataFullSpec = dict()
        self.fs_nbin = 0

    def readFile(self, fname):
        """Read an ASCII descriptor file (descriptorFile.py:30-56): space separated,
        lines starting with ``!`` are comments."""
        with open(fname, "r") as f:
            for row in csv.reader(f, delimiter=" ", skipinitialspace=True):
                if not row or row[0][0] == "!":
                    continue
                assert len(row) == len(self.names)
                for ii, item in enumerate(row):
                    if self.types[ii] == float:
                        row[ii] = item.replace("d", "e")
                    if self.types[ii] in ("S15", "U15"):
                        row[ii] = item.replace("'", "").replace('"', "")
                self.addHydrometeor(row)

    def writeFile(self, fname):
        """Write the table as an ASCII descriptor file (descriptorFile.py:58-70)."""
        assert len(self.names) == len(self.data.dtype.names)
        with open(fname, "w") as f:
            writer = csv.writer(f, delimiter=" ")
            for row in self.data:
                writer.writerow(list(row))

    def addHydrometeor(self, hydroTuple):
        """Append one species (descriptorFile.py:72-97).  Extends the parent's
        ``hydro_q``/``hydro_reff``/``hydro_n`` profile arrays with a missing-value
        slice, as the reference does."""
        assert hydroTuple[0] not in self.data["hydro_name"]
        assert len(list(self.dataFullSpec.keys())) == 0
        row = np.array(tuple(hydroTuple), dtype=list(zip(self.names, self.types)))
        self.data = np.append(self.data, row).view(np.recarray)
        self.nhydro += 1
        par = self.parent
        par._shape4D = (par.p["ngridx"], par.p["ngridy"], par.p["max_nlyrs"], self.nhydro)
        for key in ["hydro_q", "hydro_reff", "hydro_n"]:
            if key in par.p:
                par.p[key] = np.concatenate(
                    [par.p[key], np.ones(par._shape3D + (1,)) * missingNumber], axis=-1)

    def removeHydrometeor(self, hydroName):
        """Remove a species by name, or all with ``"all"`` (descriptorFile.py:99-133)."""
        assert len(list(self.dataFullSpec.keys())) == 0
        if hydroName == "all":
            self.__init__(self.parent)
            return
        matches = np.where(self.data["hydro_name"] == hydroName)[0]
        if len(matches) == 0:
            raise ValueError("Did not find " + hydroName)
        idx = matches[0]
        self.data = np.delete(self.data, idx).view(np.recarray)
        self.nhydro -= 1
        par = self.parent
        for key in ["hydro_q", "hydro_reff", "hydro_n"]:
            if key in par.p:
                par.p[key] = np.delete(par.p[key], idx, axis=-1)
        for key in list(self.data4D.keys()):
            self.data4D[key] = np.delete(self.data4D[key], idx, axis=-1)

    def add4D(self, key, arr):
        """Per-(x,y,layer,species) override of a numeric descriptor column
        (the reference's ``data4D``, libWrapper.py:117-121)."""
        assert key in self.names
        self.data4D[key] = np.asarray(arr, dtype=float)

    def addFullSpectra(self):
        """Create the full-spectrum arrays of ``dataFullSpec``, shaped
        (ngridx, ngridy, max_nlyrs, nhydro, nbin) (``d_bound_ds``: nbin + 1)
        and zero-filled, as descriptorFile.py:173-234 does; the caller fills
        them and sets ``nmlSet['hydro_fullspec'] = True``.  Species must be added
        first, all with the same ``nbin``; of their descriptor rows only
        ``liq_ice`` and ``scat_name`` are used then.  ``rho_ds`` is the particle
        density (kg/m3), ``d_ds`` the diameter the scattering is computed at
        (m), ``d_bound_ds`` the bin edges (m), ``n_ds`` the number
        concentration per bin (1/m3, not normalised by the bin width),
        ``mass_ds`` the particle mass (kg).  ``area_ds``, ``as_ratio``,
        ``canting``, ``fallvelocity`` and the ``rg_*`` parameters are created for
        the reference's radar and SSRGA paths and not read by the passive Mie
        path."""
        assert len(self.data) > 0
        assert np.min(self.data["nbin"]) == np.max(self.data["nbin"])
        self.fs_nbin = int(np.max(self.data["nbin"]))
        par = self.parent
        shp = par._shape4D + (self.fs_nbin,)
        par._shape5D = shp
        par._shape5Dplus = par._shape4D + (self.fs_nbin + 1,)
        for key in ("rho_ds", "d_ds", "n_ds", "mass_ds", "area_ds", "as_ratio", "canting", "fallvelocity"):
            self.dataFullSpec[key] = np.zeros(shp)
        self.dataFullSpec["d_bound_ds"] = np.zeros(par._shape5Dplus)
        for key, v in (("rg_kappa_ds", 0.19), ("rg_beta_ds", 0.23), ("rg_gamma_ds", 5. / 3.), ("rg_zeta_ds", 1.)):
            self.dataFullSpec[key] = np.full(shp, v)
