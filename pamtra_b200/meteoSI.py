"""Meteorological helpers used by the profile builders.

``usStandard`` restates the 1976 U.S. Standard Atmosphere, which the
reference imports from the third-party package ``meteo_si``
(``usStandard = meteo_si.atmosphere.usStandard``, python/pyPamtra/meteoSI.py:438,
``meteo_si>=0.2`` in pyproject.toml:33).  That package is not vendored with
the reference.  The published 1976 standard defines, below 86 km, seven layers
of constant lapse rate in geopotential altitude with the base values below;
pressure follows the hydrostatic barometric formula of each layer.
"""

import numpy as np

# 1976 U.S. Standard Atmosphere constants
G0 = 9.80665          # m s-2
M_AIR = 0.0289644     # kg mol-1
R_STAR = 8.31432      # J mol-1 K-1, gas constant of the 1976 standard
R_EARTH = 6371000.0   # m, mean Earth radius for geopotential altitude

_HB = np.array([0.0, 11000.0, 20000.0, 32000.0, 47000.0, 51000.0, 71000.0])
_TB = np.array([288.15, 216.65, 216.65, 228.65, 270.65, 270.65, 214.65])
_LB = np.array([-0.0065, 0.0, 0.001, 0.0028, 0.0, -0.0028, -0.002])
_PB = np.array([101325.0, 22632.1, 5474.89, 868.019, 110.906, 66.9389, 3.95642])

Rair = 287.04
Rvapor = 461.5


def usStandard(h, geopotential=True):
    """Density [kg m-3], pressure [Pa] and temperature [K] of the 1976 U.S.
    Standard Atmosphere at heights ``h`` [m].

    Geometric height is converted to geopotential height H = R h / (R + h)
    first (``geopotential=False`` uses ``h`` directly).  With these constants
    the reference's golden regression column (tests/golden/, built from
    hgt_lev = 0..3 km) is reproduced to 2e-8 relative in brightness
    temperature.
    """
    h = np.asarray(h, dtype=float)
    H = R_EARTH * h / (R_EARTH + h) if geopotential else h
    idx = np.clip(np.searchsorted(_HB, H, side="right") - 1, 0, len(_HB) - 1)
    hb, tb, lb, pb = _HB[idx], _TB[idx], _LB[idx], _PB[idx]
    T = tb + lb * (H - hb)
    with np.errstate(divide="ignore", invalid="ignore"):
        p_grad = pb * (tb / T) ** (G0 * M_AIR / (R_STAR * lb))
        p_iso = pb * np.exp(-G0 * M_AIR * (H - hb) / (R_STAR * tb))
    p = np.where(lb != 0.0, p_grad, p_iso)
    rho = p * M_AIR / (R_STAR * T)
    return rho, p, T


def e_sat_gg_water(T):
    """Saturation vapour pressure over water [hPa], Goff-Gratch (as the
    reference's src/e_sat_gg_water.f90)."""
    T = np.asarray(T, dtype=float)
    return 1013.246 * 10 ** (-7.90298 * (373.16 / T - 1) + 5.02808 * np.log10(373.16 / T)
                             - 1.3816e-7 * (10 ** (11.344 * (1 - T / 373.16)) - 1)
                             + 8.1328e-3 * (10 ** (-3.49149 * (373.16 / T - 1)) - 1))
