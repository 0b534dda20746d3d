"""Double-double arithmetic of the extended-precision T-matrix solve
(pamtra_b200/csrc/ddreal.cuh) on the CPU: the header is host and device
code built from IEEE double operations and fma, so its host build (g++,
compiled here) gives the bits the device build will.  Checked against
50-digit mpmath arithmetic: basic operations to 1e-30 relative, the
elementary functions to 1e-29 (sin and cos absolute, scaled by 1 + |x|)."""
import ctypes
import os
import subprocess
import tempfile

import numpy as np
import pytest

mpmath = pytest.importorskip("mpmath")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SHIM = r'''
#include "ddreal.cuh"
using namespace pb;
extern "C" {
void t_bin(int op, int n, const double* a, const double* b, double* out) {
  for (int i = 0; i < n; i++) {
    const ddr x{a[2 * i], a[2 * i + 1]}, y{b[2 * i], b[2 * i + 1]};
    const ddr r = op == 0 ? x + y : op == 1 ? x - y : op == 2 ? x * y : op == 3 ? x / y : ddr_pow(x, y);
    out[2 * i] = r.hi;
    out[2 * i + 1] = r.lo;
  }
}
void t_un(int op, int n, const double* a, double* out) {
  for (int i = 0; i < n; i++) {
    const ddr x{a[2 * i], a[2 * i + 1]};
    ddr r, s, c;
    switch (op) {
      case 0: r = ddr_sqrt(x); break;
      case 1: r = ddr_exp(x); break;
      case 2: r = ddr_log(x); break;
      case 3: ddr_sincos(x, s, c); r = s; break;
      case 4: ddr_sincos(x, s, c); r = c; break;
      case 5: r = ddr_sinh(x); break;
      default: r = ddr_cosh(x); break;
    }
    out[2 * i] = r.hi;
    out[2 * i + 1] = r.lo;
  }
}
}
'''


@pytest.fixture(scope="module")
def ddlib():
    d = tempfile.mkdtemp(prefix="ddreal_")
    src = os.path.join(d, "shim.cpp")
    so = os.path.join(d, "libshim.so")
    with open(src, "w") as f:
        f.write(SHIM)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-I",
                    os.path.join(ROOT, "pamtra_b200", "csrc"), "-o", so, src], check=True)
    lib = ctypes.CDLL(so)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.t_bin.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp]
    lib.t_un.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp]
    return lib


def _dd(rng, lo, hi, n, log=False):
    h = np.exp(rng.uniform(np.log(lo), np.log(hi), n)) if log else rng.uniform(lo, hi, n)
    l = h * rng.uniform(-1, 1, n) * 1e-17
    s = h + l
    return np.stack([s, (h - s) + l], axis=1).copy()  # normalised pairs


def _mp(a):
    return [mpmath.mpf(float(x)) + mpmath.mpf(float(y)) for x, y in a]


def _got(out):
    return [mpmath.mpf(float(x)) + mpmath.mpf(float(y)) for x, y in out]


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("op, fn", [(0, lambda x, y: x + y), (1, lambda x, y: x - y), (2, lambda x, y: x * y),
                                    (3, lambda x, y: x / y)])
def test_ddreal_basic_operations(ddlib, op, fn):
    mpmath.mp.dps = 50
    rng = np.random.default_rng(op)
    a, b = _dd(rng, 1e-3, 1e3, 200, log=True), _dd(rng, 1e-3, 1e3, 200, log=True)
    b[::2] *= -1
    out = np.zeros_like(a)
    ddlib.t_bin(op, len(a), _p(a), _p(b), _p(out))
    for x, y, g in zip(_mp(a), _mp(b), _got(out)):
        ref = fn(x, y)
        assert abs(g - ref) <= mpmath.mpf("1e-30") * abs(ref), (op, x, y)


@pytest.mark.parametrize("op, fn, lo, hi, logr, absolute", [
    (0, mpmath.sqrt, 1e-3, 1e3, True, False),
    (1, mpmath.exp, -50.0, 50.0, False, False),
    (2, mpmath.log, 1e-3, 1e3, True, False),
    (3, mpmath.sin, -100.0, 100.0, False, True),
    (4, mpmath.cos, -100.0, 100.0, False, True),
    (5, mpmath.sinh, -20.0, 20.0, False, False),
    (6, mpmath.cosh, -20.0, 20.0, False, False),
])
def test_ddreal_elementary_functions(ddlib, op, fn, lo, hi, logr, absolute):
    mpmath.mp.dps = 50
    rng = np.random.default_rng(100 + op)
    a = _dd(rng, lo, hi, 200, log=logr)
    out = np.zeros_like(a)
    ddlib.t_un(op, len(a), _p(a), _p(out))
    for x, g in zip(_mp(a), _got(out)):
        ref = fn(x)
        tol = mpmath.mpf("1e-29") * ((1 + abs(x)) if absolute else abs(ref))
        assert abs(g - ref) <= tol, (op, x)


def test_ddreal_pow(ddlib):
    mpmath.mp.dps = 50
    rng = np.random.default_rng(7)
    a, b = _dd(rng, 0.1, 10.0, 200, log=True), _dd(rng, -3.0, 3.0, 200)
    out = np.zeros_like(a)
    ddlib.t_bin(4, len(a), _p(a), _p(b), _p(out))
    for x, y, g in zip(_mp(a), _mp(b), _got(out)):
        ref = mpmath.power(x, y)
        assert abs(g - ref) <= mpmath.mpf("1e-29") * abs(ref), (x, y)


def test_double_double_solve_compiles_for_sm100a(tmp_path):
    """The double-double T-matrix solve (tmatrix_dd.cuh) is not yet linked
    into the library; it must keep compiling for sm_100a until its GPU parity
    run enables it."""
    import shutil
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    src = tmp_path / "kdd.cu"
    src.write_text('#include "tmatrix_dd.cuh"\nusing namespace pb;\n'
                   '__global__ void __launch_bounds__(256, 1) kdd(double* s, double* sd, int* o) {\n'
                   '  __shared__ TmShared sh;\n'
                   '  if (!tdd_setup(sd, sh, 8, 16, 3.37e-3, 5.5, 2.9, 1e-3, 1.6)) { o[0] = -1; return; }\n'
                   '  o[0] = tdd_solve(s, sd, sh, 1, 8, 16, 3.37e-3, 5.5, 2.9);\n}\n')
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--fmad=false", "-std=c++17",
                    "-I", os.path.join(ROOT, "pamtra_b200", "csrc"), "-c", str(src), "-o", str(tmp_path / "kdd.o")],
                   check=True)
