"""SAME-BOX GPU BASELINE — test and measurement infrastructure only.

ctypes wrapper of ``oracle/_ref/librefgpu.so``: the reference's own
uniform-solver CUDA kernels (fluid/crates/compressible-cuda/src/kernels.cu,
compiled unmodified for sm_100a by ``make -C oracle refgpu``) driven in the
launch order of its ``GpuSolver<f64>`` (fluid/crates/compressible-cuda/src/
lib.rs:186-461) by ``oracle/ref_gpu.cu``. Used by tests/ (parity of the
restated oracle against the reference's own arithmetic) and by bench.py's
reference-GPU baseline leg; the product package never imports it.

``RefGpuSolver`` takes the constructor arguments of ``emergence_b200.GpuSolver``
(Euler system, f64) and has its ``step``, ``dt_cfl``, ``advance``,
``download`` and ``counters`` (the reference's three: shock-path faces,
first-order fallbacks, positivity-limited faces).
"""
import ctypes as C
import os

import numpy as np

from emergence_b200._abi import EmgBc, EmgBc7, EmgEos, EmgFiveSystem, EmgMesh, EmgOpts
from emergence_b200.physics import Bc, FluxMode

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "librefgpu.so")

_D = C.POINTER(C.c_double)
_P = C.c_void_p
SIGS = {
    "refgpu_last_error": (C.c_char_p, []),
    "refgpu_create": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgEos), C.POINTER(EmgBc), C.POINTER(EmgOpts), _D,
                                C.c_size_t, C.POINTER(_P)]),
    "refgpu_five_create": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgFiveSystem), C.POINTER(EmgBc7),
                                     C.POINTER(EmgOpts), _D, C.c_size_t, C.POINTER(_P)]),
    "refgpu_destroy": (C.c_int, [_P]),
    "refgpu_step": (C.c_int, [_P, C.c_double]),
    "refgpu_dt_cfl": (C.c_int, [_P, _D]),
    "refgpu_advance": (C.c_int, [_P, C.c_uint64, C.POINTER(C.c_uint64)]),
    "refgpu_download": (C.c_int, [_P, _D, C.c_size_t]),
    "refgpu_counters": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "refgpu_stream": (C.c_void_p, [_P]),
    "refgpu_synchronize": (C.c_int, [_P]),
}
ENTRY_POINTS = tuple(SIGS)

_lib = None


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError("oracle/_ref/librefgpu.so is not built (make -C oracle refgpu, from the reference tree)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _chk(rc):
    if rc:
        raise RuntimeError("refgpu: " + lib().refgpu_last_error().decode())


def _c(mesh, eos, bc, cfl, mode, tol, positivity):
    m = EmgMesh()
    for d in range(3):
        m.n[d], m.lo[d], m.dx[d] = mesh.n[d], mesh.lo[d], mesh.dx[d]
    m.ng = mesh.ng
    e = EmgEos(eos.gamma, eos.p_inf, eos.b, eos.q, eos.cv)
    b = (EmgBc * 6)()
    for d in range(3):
        for s in range(2):
            b[2 * d + s].kind = bc[d][s].kind
            for k in range(5):
                b[2 * d + s].state[k] = bc[d][s].state[k]
    o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, 0, 0)
    return m, e, b, o


class RefGpuSolver:
    """The reference's GpuSolver<f64> for the Euler system on the current device."""

    def __init__(self, sys, mesh, u, bc=None, cfl=0.5, mode=FluxMode.Weno, tol=1e-3, positivity=True):
        self.mesh = mesh
        bc = bc if bc is not None else [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (mesh.len(), 5):
            raise ValueError(f"state must have shape {(mesh.len(), 5)}, got {u.shape}")
        self._args = _c(mesh, sys.eos, bc, cfl, mode, tol, positivity)
        m, e, b, o = self._args
        h = _P()
        _chk(lib().refgpu_create(C.byref(m), C.byref(e), b, C.byref(o), u.ctypes.data_as(_D), mesh.len(),
                                 C.byref(h)))
        self._h = h

    def step(self, dt):
        _chk(lib().refgpu_step(self._h, dt))

    def dt_cfl(self):
        v = C.c_double()
        _chk(lib().refgpu_dt_cfl(self._h, C.byref(v)))
        return v.value

    def advance(self, nsteps):
        """nsteps iterations of run_to's loop body (dt_cfl, then step)."""
        taken = C.c_uint64()
        _chk(lib().refgpu_advance(self._h, nsteps, C.byref(taken)))
        return taken.value

    nv = 5

    def download(self):
        out = np.empty((self.mesh.len(), self.nv))
        _chk(lib().refgpu_download(self._h, out.ctypes.data_as(_D), self.mesh.len()))
        return out

    def counters(self):
        out = (C.c_uint64 * 3)()
        _chk(lib().refgpu_counters(self._h, out))
        return list(out)

    def stream(self):
        return lib().refgpu_stream(self._h)

    def synchronize(self):
        _chk(lib().refgpu_synchronize(self._h))

    def close(self):
        if getattr(self, "_h", None):
            lib().refgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RefGpuFiveSolver(RefGpuSolver):
    """The reference's GpuSolver<f64> for GpuSystem::FiveEq (its `five`
    kernels, kernels.cu:116-256) on the current device."""

    nv = 7

    def __init__(self, sys, mesh, u, bc=None, cfl=0.5, mode=FluxMode.Weno, tol=1e-3, positivity=True):
        from emergence_b200.five import _c_bcs7, _c_system
        self.mesh = mesh
        bc = bc if bc is not None else [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (mesh.len(), 7):
            raise ValueError(f"state must have shape {(mesh.len(), 7)}, got {u.shape}")
        from emergence_b200.solver import _c_mesh
        m = _c_mesh(mesh)
        o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, 0, 0)
        s, b = _c_system(sys), _c_bcs7(bc)
        self._args = (m, s, b, o)
        h = _P()
        _chk(lib().refgpu_five_create(C.byref(m), C.byref(s), b, C.byref(o), u.ctypes.data_as(_D), mesh.len(),
                                      C.byref(h)))
        self._h = h
