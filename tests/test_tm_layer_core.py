"""The start of a scattering layer with T-matrix species in the layer
set-up's storage (pamtra_b200/csrc/tm_layer_core.cuh, host and device code,
compiled here with g++) against the oracle's layer start
(oracle layer_start: doubling count, INITIAL_SOURCE4, INITIALIZE4, and
CHECK_NORM4 as the forward run applies it): bit for bit, with and without
T-matrix arrays, with and without scatcnv's Mie part."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SHIM = r'''
#include "tm_layer_core.cuh"
using namespace pb;
// P1 / P2 of scatcnv (row-major [2][n][n]) -> the set-up's storage, T-matrix
// quadrants added, CHECK_NORM4, doublings, INITIALIZE4, INITIAL_SOURCE4.
extern "C" int start(int N, const double* mu, const double* wq, double zdiff, double gas, double planck0,
                     const double* scv, double ext, double emis, const double* tmq, const double* tm_ext,
                     const double* tm_emis, double* Rb, double* Tb, double* lin, double* maxnorm) {
  const int n = 2 * N, LD = n;
  for (int e = 0; e < n * n; e++) {
    const int row = e / n, col = e % n;
    Tb[col * LD + row] = scv[e];
    Rb[col * LD + row] = scv[n * n + e];
  }
  if (tmq)
    for (int e = 0; e < n * n; e++) tml_add_scatter(e, n, LD, tmq, Tb, Rb);
  double mx = 0.0;
  for (int t = 0; t < N; t++) {
    const double v = tml_norm(t, N, LD, wq, ext, emis, tm_ext, tm_emis, Tb, Rb);
    mx = v > mx ? v : mx;
  }
  *maxnorm = mx;
  double dz = 0.0;
  const int nd = tml_doublings(ext, tm_ext, gas, zdiff, &dz);
  for (int e = 0; e < n * n; e++) tml_init4(e, n, LD, mu, wq, dz, gas, ext, tm_ext, Rb, Tb);
  for (int t = 0; t < n; t++) lin[t] = tml_source(t, mu, planck0, dz, gas, emis, tm_emis);
  return nd;
}
'''


@pytest.fixture(scope="module")
def core():
    d = tempfile.mkdtemp(prefix="tmlcore_")
    src = os.path.join(d, "shim.cpp")
    so = os.path.join(d, "libshim.so")
    with open(src, "w") as f:
        f.write(SHIM)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I",
                    os.path.join(ROOT, "pamtra_b200", "csrc"), "-o", so, src], check=True)
    lib = ctypes.CDLL(so)
    vp = ctypes.c_void_p
    lib.start.restype = ctypes.c_int
    lib.start.argtypes = [ctypes.c_int, vp, vp] + [ctypes.c_double] * 3 + [vp, ctypes.c_double, ctypes.c_double] + \
        [vp] * 7
    return lib


def _ptr(a):
    return None if a is None else a.ctypes.data


@pytest.mark.parametrize("with_mie, with_tm", [(True, False), (False, True), (True, True)])
def test_layer_start_matches_oracle(core, oracle_mod, with_mie, with_tm):
    N, n = 16, 32
    mu, wq = oracle_mod.lobatto(N)
    zdiff, gas, planck0, planck1 = 250.0, 2.0e-4, 1.1e-7, 1.2e-7
    scv = np.zeros((4, n, n))
    ext = emis = 0.0
    if with_mie:
        # a scatcnv-like symmetric part: quadrants 1 = 4 and 2 = 3
        rng = np.random.default_rng(3)
        p1 = rng.uniform(0, 1e-5, (n, n))
        p2 = rng.uniform(0, 1e-5, (n, n))
        scv[0] = scv[3] = p1
        scv[1] = scv[2] = p2
        ext, emis = 4.0e-4, 1.5e-4
    tmq = tm_ext = tm_emis = None
    tot = scv.copy()
    if with_tm:
        r = oracle_mod.tmatrix_species(N, 89e9, 1.78, -0.003, 1, np.array([1.5e-3, 2.5e-3]), np.full(2, 1e-4),
                                       np.full(2, 2e7), np.full(2, 1000.0), np.array([0.8, 0.6]), np.zeros(2))
        S = r["scatter_matrix"]  # (i2, ll, i1, jj, kk)
        tmq = np.zeros((2, n, n))
        for kk in range(2):
            for ll in range(N):
                for jj in range(N):
                    for i2 in range(2):
                        for i1 in range(2):
                            tmq[kk, i2 + 2 * ll, i1 + 2 * jj] = S[i2, ll, i1, jj, kk]
        tot[0] = tmq[0] + scv[0]
        tot[3] = tmq[0] + scv[3]
        tot[1] = tmq[1] + scv[1]
        tot[2] = tmq[1] + scv[2]
        tm_ext = np.asfortranarray(r["extinct_matrix"]).ravel(order="F")
        tm_emis = np.asfortranarray(r["emis_vector"]).ravel(order="F")
    nd_o, R_o, T_o, lin_o, _ = oracle_mod.layer_start(N, zdiff, gas, planck0, planck1, tot.reshape(-1), ext, emis,
                                                      tm_ext, tm_emis)
    Rb, Tb, lin, mx = np.zeros(n * n), np.zeros(n * n), np.zeros(n), ctypes.c_double(0.0)
    tq = None if tmq is None else np.ascontiguousarray(tmq.reshape(-1))
    nd = core.start(N, _ptr(mu), _ptr(wq), zdiff, gas, planck0, _ptr(np.ascontiguousarray(scv[:2].reshape(-1))),
                    ext, emis, _ptr(tq), _ptr(tm_ext), _ptr(tm_emis), _ptr(Rb), _ptr(Tb), _ptr(lin), ctypes.byref(mx))
    assert nd == nd_o
    assert np.array_equal(Rb, R_o[:n * n]) and np.array_equal(Tb, T_o[:n * n])
    assert np.array_equal(lin, lin_o[:n])
    if with_tm and not with_mie:
        # the T-matrix matrices are normalised by construction (emission = extinction - scattering)
        assert mx.value < 5e-4
