"""Host-side checks of the same-box GPU baseline (oracle/ref_gpu.cu, built by
`make -C oracle refgpu` into oracle/_ref/ where the reference tree is present):
it exports the entry points bench.py's reference-GPU leg binds, and rejects bad
arguments before any device call (so these run without a GPU)."""
import ctypes as C
import os

import numpy as np
import pytest

from emergence_b200._abi import EmgBc, EmgEos, EmgMesh, EmgOpts

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "librefgpu.so")

pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="oracle/_ref/librefgpu.so is not built")

ENTRY_POINTS = ("refgpu_create", "refgpu_destroy", "refgpu_step", "refgpu_dt_cfl", "refgpu_advance",
                "refgpu_download", "refgpu_counters", "refgpu_stream", "refgpu_synchronize", "refgpu_last_error")


def lib():
    L = C.CDLL(LIB)
    L.refgpu_last_error.restype = C.c_char_p
    return L


def test_exports_the_bound_entry_points():
    L = lib()
    for name in ENTRY_POINTS:
        assert hasattr(L, name), name


def test_create_rejects_bad_arguments_before_device_work():
    L = lib()
    h = C.c_void_p()
    assert L.refgpu_create(None, None, None, None, None, C.c_size_t(0), C.byref(h)) == 1
    assert b"null" in L.refgpu_last_error()
    m = EmgMesh()
    for d, n in enumerate((8, 8, 1)):
        m.n[d] = n
        m.dx[d] = 1.0 / n
    m.ng = 6
    e, o, bc = EmgEos(1.4, 0, 0, 0, 1), EmgOpts(0.5, 1e-3, 1, 1, 0, 0), (EmgBc * 6)()
    u = np.zeros((20 * 20, 5))
    # 8×8 with 6 ghost layers on the two active axes is 20·20 cells: one short
    rc = L.refgpu_create(C.byref(m), C.byref(e), bc, C.byref(o), u.ctypes.data_as(C.POINTER(C.c_double)),
                         C.c_size_t(20 * 20 - 1), C.byref(h))
    assert rc == 1 and b"length" in L.refgpu_last_error() and not h.value
    m.n[0] = 0
    rc = L.refgpu_create(C.byref(m), C.byref(e), bc, C.byref(o), u.ctypes.data_as(C.POINTER(C.c_double)),
                         C.c_size_t(20 * 20), C.byref(h))
    assert rc == 1 and b"extents" in L.refgpu_last_error() and not h.value
