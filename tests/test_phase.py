"""The Green kernels' sin/cos (beat_engine_b200/csrc/phase.cuh) against the C
library, compiled for the host from the same header the device code uses.

Error bound, over the phase range the kernels see (|k r| < 2000): within
2 ulp of the exact value, or within half an ulp of 1 in absolute terms where
the result is near a zero of sin or cos (there the reduction's own rounding,
n times the last split part of pi/2, dominates the tiny result's ulp)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER_DIR = os.path.join(ROOT, "beat_engine_b200", "csrc")

WRAPPER = r"""
#include "phase.cuh"
extern "C" void phase64(int n, const double *x, double *s, double *c) {
    for (int i = 0; i < n; ++i) bb::sincos_cw(x[i], s + i, c + i);
}
extern "C" void phase32(int n, const float *x, float *s, float *c) {
    for (int i = 0; i < n; ++i) bb::sincos_cw(x[i], s + i, c + i);
}
"""


@pytest.fixture(scope="module")
def phase_lib(tmp_path_factory):
    d = tmp_path_factory.mktemp("phase")
    src = d / "phase_wrap.cpp"
    src.write_text(WRAPPER)
    so = d / "libphase.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I", HEADER_DIR, str(src), "-o", str(so)],
                   check=True)
    L = ctypes.CDLL(str(so))
    dp, fp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)
    L.phase64.argtypes = [ctypes.c_int, dp, dp, dp]
    L.phase32.argtypes = [ctypes.c_int, fp, fp, fp]
    return L


def _ulp_err(got, ref, dtype):
    ref_t = ref.astype(dtype)
    spacing = np.spacing(np.maximum(np.abs(ref_t), np.finfo(dtype).tiny).astype(dtype)).astype(np.float64)
    # ulps, with the spacing floored at that of 0.5 (half an ulp of 1 = 1 ulp of 0.5)
    spacing = np.maximum(spacing, float(np.spacing(dtype(0.5))))
    return np.abs(got.astype(np.float64) - ref) / spacing


def test_fp64_phase_within_2ulp(phase_lib):
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-2000, 2000, 200000), rng.uniform(-4, 4, 100000),
                        np.arange(-64, 65) * (np.pi / 4)])
    s, c = np.empty_like(x), np.empty_like(x)
    dp = ctypes.POINTER(ctypes.c_double)
    phase_lib.phase64(len(x), x.ctypes.data_as(dp), s.ctypes.data_as(dp), c.ctypes.data_as(dp))
    # libm's sin/cos are accurate to < 1 ulp; compare in ulps of the reference
    assert np.max(_ulp_err(s, np.sin(x), np.float64)) <= 2.0
    assert np.max(_ulp_err(c, np.cos(x), np.float64)) <= 2.0


def test_fp32_phase_within_2ulp(phase_lib):
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(-2000, 2000, 200000), rng.uniform(-4, 4, 100000)]).astype(np.float32)
    s, c = np.empty_like(x), np.empty_like(x)
    fp = ctypes.POINTER(ctypes.c_float)
    phase_lib.phase32(len(x), x.ctypes.data_as(fp), s.ctypes.data_as(fp), c.ctypes.data_as(fp))
    xd = x.astype(np.float64)
    assert np.max(_ulp_err(s, np.sin(xd), np.float32)) <= 2.0
    assert np.max(_ulp_err(c, np.cos(xd), np.float32)) <= 2.0
