"""GpuSolver: the device solver of one uniform grid, mirroring
compressible-cuda's ``GpuSolver`` (fluid/crates/compressible-cuda/src/
lib.rs:155-477) and the stepping API of ``compressible::Solver``
(fluid/crates/compressible/src/solver.rs:139-795).

All work runs in ``libemergence_b200.so`` on the current CUDA device; this
module only marshals arguments through the C ABI.
"""
import ctypes as C
import math

import numpy as np

from . import _abi
from ._abi import EmgBc, EmgEos, EmgMesh, EmgOpts, check, lib
from .physics import Bc, FluxMode, Precision


def _c_mesh(mesh):
    m = EmgMesh()
    for d in range(3):
        m.n[d] = mesh.n[d]
        m.lo[d] = mesh.lo[d]
        m.dx[d] = mesh.dx[d]
    m.ng = mesh.ng
    return m


def _c_eos(eos):
    return EmgEos(eos.gamma, eos.p_inf, eos.b, eos.q, eos.cv)


def _c_bcs(bc):
    arr = (EmgBc * 6)()
    for d in range(3):
        for s in range(2):
            b = bc[d][s]
            arr[2 * d + s].kind = b.kind
            for k in range(5):
                arr[2 * d + s].state[k] = b.state[k]
    return arr


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class GpuSolver:
    """Device solver of a ghost-padded conserved state.

    ``GpuSolver(sys, mesh, u, bc=..., cfl=0.5, mode=FluxMode.Weno, tol=1e-3,
    positivity=True, precision=Precision.F64, autotune=False)`` uploads ``u``
    (float64 ``[mesh.len(), 5]``) like ``GpuSolver::from_cpu``; ``autotune``
    times the sweep launch shapes on ``u`` at creation (EMG_OPT_AUTOTUNE).
    """

    def __init__(self, sys, mesh, u, bc=None, cfl=0.5, mode=FluxMode.Weno, tol=1e-3, positivity=True,
                 precision=Precision.F64, autotune=False):
        self.sys = sys
        self.mesh = mesh
        self.bc = bc if bc is not None else [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
        self.cfl = cfl
        self.mode = mode
        self.tol = tol
        self.positivity = positivity
        self.precision = precision
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (mesh.len(), 5):
            raise ValueError(f"state must have shape {(mesh.len(), 5)}, got {u.shape}")
        self._m = _c_mesh(mesh)
        self._e = _c_eos(sys.eos)
        self._b = _c_bcs(self.bc)
        self._o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, precision, 1 if autotune else 0)
        h = C.c_void_p()
        check(lib().emg_uniform_create(C.byref(self._m), C.byref(self._e), self._b, C.byref(self._o), _dptr(u),
                                       mesh.len(), C.byref(h)))
        self._h = h

    @classmethod
    def from_cpu(cls, cpu, precision=Precision.F64):
        """Build from any object with the fields of ``compressible::Solver``
        (sys, mesh, u, bc, cfl, mode, tol, positivity, t)."""
        s = cls(cpu.sys, cpu.mesh, cpu.u, bc=cpu.bc, cfl=cpu.cfl, mode=cpu.mode, tol=cpu.tol,
                positivity=cpu.positivity, precision=precision)
        if getattr(cpu, "t", 0.0):
            s.t = cpu.t
        return s

    # ---- lifetime
    def close(self):
        if getattr(self, "_h", None):
            lib().emg_uniform_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- stepping (Solver / GpuSolver API)
    def step(self, dt):
        check(lib().emg_uniform_step(self._h, float(dt)))

    def dt_cfl(self):
        v = C.c_double()
        check(lib().emg_uniform_dt_cfl(self._h, C.byref(v)))
        return v.value

    def run_to(self, t_end):
        n = C.c_uint64()
        check(lib().emg_uniform_run_to(self._h, float(t_end), C.byref(n)))
        return n.value

    def advance(self, nsteps, t_end=math.inf):
        """Take up to ``nsteps`` CFL steps with dt computed on the device."""
        n = C.c_uint64()
        check(lib().emg_uniform_advance(self._h, int(nsteps), float(t_end), C.byref(n)))
        return n.value

    # ---- state
    def download(self, out=None):
        """The conserved state as host AoS [cell][q]. ``out`` (optional): a
        C-contiguous float64 array of that shape to fill, e.g. a view of pinned
        (page-locked) host memory, which the copy reaches at full link speed."""
        if out is None:
            out = np.empty((self.mesh.len(), 5), dtype=np.float64)
        elif out.shape != (self.mesh.len(), 5) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float64 array of shape {(self.mesh.len(), 5)}")
        check(lib().emg_uniform_download(self._h, _dptr(out), self.mesh.len()))
        return out

    def upload(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        check(lib().emg_uniform_upload(self._h, _dptr(u), self.mesh.len()))

    def totals(self):
        out = np.empty(5, dtype=np.float64)
        check(lib().emg_uniform_totals(self._h, _dptr(out)))
        return out

    @staticmethod
    def nv():
        """Conserved variables per cell: 5 for the Euler system (GpuSolver::nv,
        fluid/crates/compressible-cuda/src/lib.rs:474-476)."""
        return 5

    def counters(self):
        """[faces, shock-path faces, first-order fallbacks, limited faces]."""
        out = (C.c_uint64 * 4)()
        check(lib().emg_uniform_counters(self._h, out))
        return list(out)

    @property
    def t(self):
        v = C.c_double()
        check(lib().emg_uniform_get_time(self._h, C.byref(v)))
        return v.value

    @t.setter
    def t(self, value):
        check(lib().emg_uniform_set_time(self._h, float(value)))

    def synchronize(self):
        check(lib().emg_uniform_synchronize(self._h))

    def stream(self):
        p = C.c_void_p()
        check(lib().emg_uniform_stream(self._h, C.byref(p)))
        return p.value

    def set_profiling(self, on=True):
        check(lib().emg_uniform_set_profiling(self._h, 1 if on else 0))

    def kernel_times(self):
        """{kind: (ms, launches)} accumulated since the last call."""
        ms = (C.c_double * _abi.EMG_K_COUNT)()
        n = (C.c_uint64 * _abi.EMG_K_COUNT)()
        check(lib().emg_uniform_kernel_times(self._h, ms, n))
        return {k: (ms[i], n[i]) for i, k in enumerate(_abi.KERNEL_KINDS)}

    def launch_count(self):
        n = C.c_uint64()
        check(lib().emg_uniform_launch_count(self._h, C.byref(n)))
        return n.value

    def features(self):
        """EMG_FEATURE_* bits of the device paths this solver uses (bit 0: TMA row staging)."""
        f = C.c_uint32()
        check(lib().emg_uniform_features(self._h, C.byref(f)))
        return f.value


def state_hash(mesh, u):
    """64-bit fingerprint of a ghost-padded AoS conserved state (host code, no
    device): the hash of fluid/crates/compressible/examples/cpu_validate.rs:7-22
    over the interior cells. Equal states, bit for bit, give equal hashes."""
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = C.c_uint64()
    check(lib().emg_state_hash(C.byref(_c_mesh(mesh)), _dptr(u), mesh.len(), C.byref(out)))
    return out.value


def device_count():
    n = C.c_int()
    check(lib().emg_device_count(C.byref(n)))
    return n.value


def release_memory():
    """Give the device memory that destroyed solvers left in the library's
    stream-ordered pools back to the device."""
    check(lib().emg_release_memory())
