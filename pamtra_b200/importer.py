"""Profile builders (subset of python/pyPamtra/importer.py).

Only ``createUsStandardProfile`` (importer.py:3039-3093) is on the passive
path: the reference's golden regression scenario builds its column with it.
"""

import numpy as np

from .meteoSI import usStandard


def _createUsStandardProfile(**kwargs):
    """Level pressure/temperature of the U.S. standard atmosphere at
    ``hgt_lev``; other keyword arguments pass through; relative humidity is
    zero unless ``relhum_lev`` or ``q`` is given (importer.py:3056-3093)."""
    assert "hgt_lev" in kwargs
    hgt_lev = np.asarray(kwargs["hgt_lev"], dtype=float)
    pamData = dict()
    _, press, temp = usStandard(hgt_lev)
    pamData["press_lev"] = np.asarray(press, dtype=float)
    pamData["temp_lev"] = np.asarray(temp, dtype=float)
    for kk in kwargs:
        pamData[kk] = np.array(kwargs[kk])
    if "relhum_lev" not in kwargs and "q" not in kwargs:
        pamData["relhum_lev"] = np.zeros_like(hgt_lev)
    return pamData


def createUsStandardProfile(pam=None, **kwargs):
    """Create a clear-sky U.S. standard atmosphere profile on ``pam``
    (importer.py:3039)."""
    if pam is None:
        from .core import pyPamtra
        pam = pyPamtra()
    pam.createProfile(**_createUsStandardProfile(**kwargs))
    return pam
