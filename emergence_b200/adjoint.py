"""DifferentiableSolver: discrete adjoint of the uniform-grid FP64 step.

The reference solver (fluid/crates/compressible/src/solver.rs) only runs
forward; this module adds reverse-mode gradients of its step on the device,
through the ``emg_adjoint_*`` C ABI (emergence_b200/csrc/adjoint.cu). A
forward run is recorded with √N checkpoints; ``backward`` then returns the
gradient of a box objective (or of any seeded cotangent of the final state)
with respect to the initial conserved and primitive states and to γ.

The recorded time steps, the positivity limiter's blend weights and the
admissibility fallbacks are held fixed, so the gradient is that of the
discrete map the forward run applied (finite differences must use the same
time steps: ``forward(dts=...)``).
"""
import ctypes as C
import math

import numpy as np

from ._abi import EmgOpts, check, lib
from .physics import Bc, FluxMode, Precision
from .solver import _c_bcs, _c_eos, _c_mesh, _dptr

OBJ_PRESSURE, OBJ_ENERGY = 0, 1


class DifferentiableSolver:
    """Differentiable uniform-grid solver (FP64, WENO flux mode).

    ``DifferentiableSolver(sys, mesh, u, bc=..., cfl=0.5, positivity=True)``
    takes the padded AoS conserved state ``u`` like ``GpuSolver``.
    """

    def __init__(self, sys, mesh, u, bc=None, cfl=0.5, positivity=True):
        self.sys, self.mesh = sys, mesh
        self.bc = bc if bc is not None else [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
        u = np.ascontiguousarray(u, dtype=np.float64)
        self._m = _c_mesh(mesh)
        self._e = _c_eos(sys.eos)
        self._b = _c_bcs(self.bc)
        self._o = EmgOpts(cfl, 1e-3, FluxMode.Weno, 1 if positivity else 0, Precision.F64, 0)
        h = C.c_void_p()
        check(lib().emg_adjoint_create(C.byref(self._m), C.byref(self._e), self._b, C.byref(self._o), _dptr(u),
                                       mesh.len(), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().emg_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_initial(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        check(lib().emg_adjoint_set_initial(self._h, _dptr(u), self.mesh.len()))

    def forward(self, nsteps=None, t_end=math.inf, dts=None, checkpoint_every=0):
        """Record a forward run: ``nsteps`` CFL steps (stopping at ``t_end``),
        or exactly the time steps ``dts``. Returns the number of steps."""
        if dts is not None:
            dts = np.ascontiguousarray(dts, dtype=np.float64).reshape(-1)
            check(lib().emg_adjoint_forward_dts(self._h, _dptr(dts), dts.shape[0], int(checkpoint_every)))
            return dts.shape[0]
        taken = C.c_uint64()
        check(lib().emg_adjoint_forward(self._h, int(nsteps), float(t_end), int(checkpoint_every), C.byref(taken)))
        return taken.value

    def dts(self):
        n = C.c_uint64()
        check(lib().emg_adjoint_dts(self._h, None, 0, C.byref(n)))
        out = np.zeros(n.value)
        check(lib().emg_adjoint_dts(self._h, _dptr(out), out.shape[0], C.byref(n)))
        return out

    def download(self):
        out = np.zeros((self.mesh.len(), 5))
        check(lib().emg_adjoint_download(self._h, _dptr(out), self.mesh.len()))
        return out

    def objective(self, kind, box_lo, box_hi):
        """J of the final state; seeds the backward pass with ∂J/∂U."""
        J = C.c_double()
        lo = np.ascontiguousarray(box_lo, dtype=np.float64)
        hi = np.ascontiguousarray(box_hi, dtype=np.float64)
        check(lib().emg_adjoint_objective(self._h, int(kind), _dptr(lo), _dptr(hi), C.byref(J)))
        return J.value

    def seed(self, ubar):
        ubar = np.ascontiguousarray(ubar, dtype=np.float64)
        check(lib().emg_adjoint_seed(self._h, _dptr(ubar), self.mesh.len()))

    def backward(self):
        """Returns (ū⁰ conserved, w̄⁰ primitive, [γ̄ at fixed U⁰, γ̄ at fixed W⁰])."""
        ub = np.zeros((self.mesh.len(), 5))
        wb = np.zeros((self.mesh.len(), 5))
        g = np.zeros(2)
        check(lib().emg_adjoint_backward(self._h, _dptr(ub), _dptr(wb), _dptr(g)))
        return ub, wb, g

    def step_vjp(self, u, dt, ubar_next):
        """(∂U'/∂U)ᵀ·ū' and (∂U'/∂γ)ᵀ·ū' for one step U' = step(U, dt)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        yb = np.ascontiguousarray(ubar_next, dtype=np.float64)
        out = np.zeros((self.mesh.len(), 5))
        g = C.c_double()
        check(lib().emg_adjoint_step_vjp(self._h, _dptr(u), self.mesh.len(), float(dt), _dptr(yb), _dptr(out),
                                         C.byref(g)))
        return out, g.value

    def times(self):
        """Device ms of [last forward run, checkpoint recompute, reverse sweeps]."""
        ms = np.zeros(3)
        check(lib().emg_adjoint_times(self._h, _dptr(ms)))
        return ms

    def stream(self):
        s = C.c_void_p()
        check(lib().emg_adjoint_stream(self._h, C.byref(s)))
        return s.value or 0
