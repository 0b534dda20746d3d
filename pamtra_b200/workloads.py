"""Seeded synthetic workloads of the named shapes (shared by tests, smoke and
bench).  No dataset is involved: the reference publishes none for this path.

``golden_pam`` rebuilds the reference's golden regression column
(tests/_scenario.py:14-38 of the reference): rain (exp, N0 = 8e6, 30 bins)
at 1 g/kg in layer 1 and snow (exp_field_t) at 0.5 g/kg in layer 2 of a
U.S. standard atmosphere on hgt_lev = 0..3 km, at 10.65 and 35.5 GHz.

``c1_pam`` is the single-column workload: 50 layers over 0-12 km, seeded
standard-atmosphere T/p jitter, RH 40-95 %, cloud liquid (exp, 40 bins over
2-100 um, 0.3 g/kg) and rain (Marshall-Palmer, 50 bins over 0.1-6 mm,
0.5 g/kg) in layers 5-25, specular surface with emissivity 0.5 at 290 K.

``c2_pam`` is the batched workload: ``ncol`` seeded columns of 50 layers with
the same two species and mixing ratios log-uniform over 0.01-2 g/kg.
"""

import warnings

import numpy as np

from . import core, importer, meteoSI

GOLDEN_FREQS = [10.65, 35.5]
C1_FREQS = [23.8, 31.4, 89.0]
C2_FREQS = [23.8, 31.4, 89.0, 150.0]

RAIN_GOLDEN = ("rwc_q", -99.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 3, 30, "exp", -99.0, -99.0, 8.0e6, -99.0,
               1.0e-5, 6.0e-3, "mie-sphere", "khvorostyanov01_drops", -99.0)
SNOW_GOLDEN = ("swc_q", -99.0, -1, -99.0, 0.038, 2.0, 0.3971, 1.88, 3, 30, "exp_field_t", -99.0, -99.0, -99.0,
               -99.0, 0.51e-10, 2.0e-2, "mie-sphere", "heymsfield10_particles", -99.0)
# cloud liquid: exponential PSD with fixed effective radius p_2 = 10 um
CLOUD_C1 = ("cwc_q", -99.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 3, 40, "exp", -99.0, 1.0e-5, -99.0, -99.0,
            2.0e-6, 1.0e-4, "mie-sphere", "corPowerLaw_24388657.6_2.0", -99.0)
# rain: Marshall-Palmer (exponential, N0 = 8e6 m^-4)
RAIN_C1 = ("rwc_q", -99.0, 1, -99.0, -99.0, -99.0, -99.0, -99.0, 3, 50, "exp", -99.0, -99.0, 8.0e6, -99.0,
           1.0e-4, 6.0e-3, "mie-sphere", "khvorostyanov01_drops", -99.0)


def golden_pam():
    warnings.simplefilter("ignore")
    pam = core.pyPamtra()
    pam.df.addHydrometeor(RAIN_GOLDEN)
    pam.df.addHydrometeor(SNOW_GOLDEN)
    pam = importer.createUsStandardProfile(pam, hgt_lev=[0.0, 1000.0, 2000.0, 3000.0])
    pam.nmlSet["randomseed"] = 10
    pam.p["hydro_q"][0, 0, 1, 0] = 1e-3
    pam.p["hydro_q"][0, 0, 2, 1] = 5e-4
    return pam


def _columns(ncol, nlay, seed, q_cloud=None, q_rain=None):
    rng = np.random.default_rng(seed)
    hgt_lev = np.linspace(0.0, 12000.0, nlay + 1)
    _, p0, t0 = meteoSI.usStandard(hgt_lev)
    temp_lev = t0[None, :] + rng.uniform(-1.0, 1.0, (ncol, nlay + 1))
    press_lev = p0[None, :] * (1.0 + rng.uniform(-0.005, 0.005, (ncol, nlay + 1)))
    relhum_lev = rng.uniform(40.0, 95.0, (ncol, nlay + 1))
    hydro_q = np.zeros((ncol, nlay, 2))
    cloud = slice(5, 26)
    if q_cloud is None:
        hydro_q[:, cloud, 0] = 10 ** rng.uniform(np.log10(1e-5), np.log10(2e-3), (ncol, 21))
        hydro_q[:, cloud, 1] = 10 ** rng.uniform(np.log10(1e-5), np.log10(2e-3), (ncol, 21))
    else:
        hydro_q[:, cloud, 0] = q_cloud
        hydro_q[:, cloud, 1] = q_rain
    return dict(hgt_lev=np.repeat(hgt_lev[None, :], ncol, 0), temp_lev=temp_lev, press_lev=press_lev,
                relhum_lev=relhum_lev, hydro_q=hydro_q)


def _pam_from(cols, ncol, nlay):
    warnings.simplefilter("ignore")
    pam = core.pyPamtra()
    pam.df.addHydrometeor(CLOUD_C1)
    pam.df.addHydrometeor(RAIN_C1)
    pam.nmlSet["hydro_adaptive_grid"] = False
    pam.nmlSet["emissivity"] = 0.5
    pam.createProfile(hgt_lev=cols["hgt_lev"].reshape(ncol, 1, nlay + 1),
                      temp_lev=cols["temp_lev"].reshape(ncol, 1, nlay + 1),
                      press_lev=cols["press_lev"].reshape(ncol, 1, nlay + 1),
                      relhum_lev=cols["relhum_lev"].reshape(ncol, 1, nlay + 1),
                      hydro_q=cols["hydro_q"].reshape(ncol, 1, nlay, 2),
                      groundtemp=290.0, sfc_refl="S",
                      obs_height=np.tile([833000.0, 0.0], (ncol, 1, 1)))
    return pam


def c1_pam(seed=1):
    return _pam_from(_columns(1, 50, seed, q_cloud=3e-4, q_rain=5e-4), 1, 50)


def c2_pam(ncol=4096, seed=2):
    return _pam_from(_columns(ncol, 50, seed), ncol, 50)
