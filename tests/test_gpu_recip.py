"""The mixed form's Newton-refined reciprocal and reciprocal square root
(emergence_b200/csrc/physics.cuh: rcp_nr, rsqrt_nr) against CUDA's correctly
rounded division and square root, on the GPU (needs a B200).

The mixed form computes the HLLC star states, the characteristic eigenvector
coefficients and the sound speed of each midpoint with these in place of
IEEE division and square root; its error budget against the FP64 oracle is
1e-6 relative L1, so a relative error of about 1e-12 in each reciprocal is
far inside it. The plain FP64 form does not use them. The fast FP64 form's
one-ulp versions (rcp_f, rsqrt_f, sqrt_f) are checked here as well.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "recip_check.cu")
OUT = os.path.join(HERE, "native", "_build", "librecip_check.so")
PHYS = os.path.join(HERE, "..", "emergence_b200", "csrc", "physics.cuh")

# One Newton–Raphson step squares the relative error ε of the hardware
# estimate (about 2^-20): ε² for the reciprocal, 1.5·ε² for the reciprocal
# square root, ≈ 1.4e-12 at most.
REL_TOL = 2e-12


def _lib():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in (SRC, PHYS)):
        nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
        # the flags of the mixed sweep's translation unit
        subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
                        "-Xcompiler", "-fPIC", "-fmad=true", "-use_fast_math", SRC, "-o", OUT], check=True)
    lib = C.CDLL(OUT)
    lib.recip_check.restype = C.c_int
    lib.recip_check.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    return lib


def _run(y, fast=False):
    y = np.ascontiguousarray(y, dtype=np.float64)
    out = np.empty(6 * y.size)
    assert _lib().recip_check(y.ctypes.data, out.ctypes.data, y.size, 1 if fast else 0) == 0
    return out.reshape(6, y.size)


def test_refined_reciprocals_against_cuda_division_and_sqrt():
    rng = np.random.default_rng(20261203)
    n = 1 << 20
    # magnitudes log-uniform over 400 decades (no subnormal operand or result), both signs,
    # plus the values the Euler states of the workloads produce
    y = np.exp(rng.uniform(np.log(1e-200), np.log(1e200), n)) * rng.choice([-1.0, 1.0], n)
    y[:8] = [1.0, 2.0, 0.4, 1.4, 0.125, 3.0, 7.0, 0.1]
    o = _run(y)

    def rel(a, b):
        return float(np.max(np.abs(a - b) / np.abs(b)))

    e_rcp, e_rsqrt, e_sqrt = rel(o[0], o[1]), rel(o[2], o[3]), rel(o[4], o[5])
    print(f"max relative error: rcp_nr {e_rcp:.3e}, rsqrt_nr {e_rsqrt:.3e}, x*rsqrt_nr {e_sqrt:.3e}")
    assert e_rcp <= REL_TOL and e_rsqrt <= REL_TOL and e_sqrt <= REL_TOL, (e_rcp, e_rsqrt, e_sqrt)


def test_refined_reciprocals_of_zero_infinity_and_nan_are_not_finite():
    o = _run(np.array([0.0, -0.0, np.inf, -np.inf, np.nan]))
    assert not np.any(np.isfinite(o[0]))  # rcp_nr
    assert not np.any(np.isfinite(o[4]))  # x·rsqrt_nr(x), the mixed form's sound speed from c²


# The fast FP64 form's versions cube the estimate's error (2^-60) before the
# final rounding: within a few ulps of the correctly rounded results.
FAST_REL_TOL = 1e-15  # about 4.5 ulp


def test_fast_form_reciprocals_are_within_a_few_ulps():
    rng = np.random.default_rng(20261204)
    n = 1 << 20
    y = np.exp(rng.uniform(np.log(1e-200), np.log(1e200), n)) * rng.choice([-1.0, 1.0], n)
    y[:8] = [1.0, 2.0, 0.4, 1.4, 0.125, 3.0, 7.0, 0.1]
    o = _run(y, fast=True)

    def rel(a, b):
        return float(np.max(np.abs(a - b) / np.abs(b)))

    e = rel(o[0], o[1]), rel(o[2], o[3]), rel(o[4], o[5])
    print("max relative error: rcp_f %.3e, rsqrt_f %.3e, sqrt_f %.3e" % e)
    assert max(e) <= FAST_REL_TOL, e


def test_fast_form_square_root_of_zero_and_infinity():
    o = _run(np.array([0.0, np.inf, 4.0]), fast=True)
    assert o[4][0] == 0.0 and o[4][1] == np.inf and o[4][2] == 2.0
    assert not np.isfinite(o[0][0])  # rcp_f(0)
