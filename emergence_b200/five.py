"""Two-phase five-equation system (Kapila's model) on uniform grids.

``FiveEq`` mirrors ``compressible::multiphase::FiveEq``
(fluid/crates/compressible/src/multiphase.rs:24-392): conserved
(α1ρ1, α2ρ2, ρu, ρv, ρw, E, α1), primitive (α1ρ1, α2ρ2, u, v, w, p, α1), a
NASG equation of state per phase. ``GpuFiveSolver`` is the device solver of
``Solver<7, FiveEq>`` (compressible-cuda's ``GpuSolver`` with
``GpuSystem::FiveEq``), driven through the ``emg_five_*`` C ABI; state arrays
are ``float64[len, 7]`` in the ghost-padded AoS layout.
"""
import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from ._abi import EmgBc7, EmgEos, EmgFiveSystem, EmgOpts, check, lib
from .physics import Bc, FluxMode, Nasg, Precision

IA, IP = 6, 5


@dataclass(frozen=True)
class FiveEq:
    eos: tuple  # (Nasg, Nasg): phase 1, phase 2
    kapila: bool = True

    # multiphase.rs:58-69 (vectorised, same operation order)
    def db(self, w):
        al = (w[..., IA], 1.0 - w[..., IA])
        d = np.zeros(w.shape[:-1])
        b = np.zeros(w.shape[:-1])
        for k in range(2):
            e = self.eos[k]
            vol = al[k] - e.b * w[..., k]
            d = d + vol / (e.gamma - 1.0)
            b = b + e.gamma * e.p_inf * vol / (e.gamma - 1.0) + e.q * w[..., k]
        return d, b

    def to_cons(self, w):
        """multiphase.rs:152-163."""
        w = np.asarray(w, dtype=np.float64)
        r = w[..., 0] + w[..., 1]
        d, b = self.db(w)
        u = np.empty_like(w)
        u[..., 0] = w[..., 0]
        u[..., 1] = w[..., 1]
        u[..., 2] = r * w[..., 2]
        u[..., 3] = r * w[..., 3]
        u[..., 4] = r * w[..., 4]
        u[..., 5] = (w[..., IP] * d + b) + 0.5 * r * (w[..., 2] * w[..., 2] + w[..., 3] * w[..., 3] + w[..., 4] * w[..., 4])
        u[..., 6] = w[..., IA]
        return u

    def to_prim(self, u):
        """multiphase.rs:131-146."""
        u = np.asarray(u, dtype=np.float64)
        r = u[..., 0] + u[..., 1]
        w = np.empty_like(u)
        w[..., 0] = u[..., 0]
        w[..., 1] = u[..., 1]
        w[..., 2] = u[..., 2] / r
        w[..., 3] = u[..., 3] / r
        w[..., 4] = u[..., 4] / r
        w[..., IA] = u[..., 6]
        rhoe = u[..., 5] - 0.5 * r * (w[..., 2] * w[..., 2] + w[..., 3] * w[..., 3] + w[..., 4] * w[..., 4])
        d, b = self.db(w)
        w[..., IP] = (rhoe - b) / d
        return w


def five_initial_state(sys, mesh, w_interior):
    """Padded AoS conserved state float64[len, 7] from interior primitives."""
    u = np.zeros((mesh.len(), 7), dtype=np.float64)
    mesh.interior(u)[...] = sys.to_cons(w_interior)
    return u


def _c_system(sys):
    s = EmgFiveSystem()
    for k in range(2):
        e = sys.eos[k]
        s.eos[k] = EmgEos(e.gamma, e.p_inf, e.b, e.q, e.cv)
    s.kapila = 1 if sys.kapila else 0
    return s


def _c_bcs7(bc):
    arr = (EmgBc7 * 6)()
    for d in range(3):
        for s in range(2):
            b = bc[d][s]
            arr[2 * d + s].kind = b.kind
            st = tuple(b.state) + (0.0,) * (7 - len(b.state))
            for k in range(7):
                arr[2 * d + s].state[k] = st[k]
    return arr


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class GpuFiveSolver:
    """Device solver of a ghost-padded five-equation state (plain FP64 form,
    or the fast FP64 form with ``precision=Precision.F64Fast``).

    ``GpuFiveSolver(sys, mesh, u, bc=..., cfl=0.5, mode=FluxMode.Weno,
    tol=1e-3, positivity=True)``; ``bc[d][s]`` are ``Bc`` values whose
    Dirichlet / far-field states hold 7 conserved values.
    """

    def __init__(self, sys, mesh, u, bc=None, cfl=0.5, mode=FluxMode.Weno, tol=1e-3, positivity=True,
                 precision=Precision.F64):
        self.sys, self.mesh = sys, mesh
        self.bc = bc if bc is not None else [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (mesh.len(), 7):
            raise ValueError(f"state must have shape {(mesh.len(), 7)}, got {u.shape}")
        from .solver import _c_mesh
        self._m = _c_mesh(mesh)
        self._s = _c_system(sys)
        self._b = _c_bcs7(self.bc)
        self._o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, precision, 0)
        h = C.c_void_p()
        check(lib().emg_five_create(C.byref(self._m), C.byref(self._s), self._b, C.byref(self._o), _dptr(u),
                                    mesh.len(), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().emg_five_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt):
        check(lib().emg_five_step(self._h, float(dt)))

    def dt_cfl(self):
        v = C.c_double()
        check(lib().emg_five_dt_cfl(self._h, C.byref(v)))
        return v.value

    def run_to(self, t_end):
        n = C.c_uint64()
        check(lib().emg_five_run_to(self._h, float(t_end), C.byref(n)))
        return n.value

    def download(self):
        out = np.empty((self.mesh.len(), 7))
        check(lib().emg_five_download(self._h, _dptr(out), self.mesh.len()))
        return out

    def counters(self):
        out = (C.c_uint64 * 4)()
        check(lib().emg_five_counters(self._h, out))
        return list(out)

    def totals(self):
        out = np.empty(7)
        check(lib().emg_five_totals(self._h, _dptr(out)))
        return out

    def launch_count(self):
        n = C.c_uint64()
        check(lib().emg_five_launch_count(self._h, C.byref(n)))
        return n.value

    def stream(self):
        """The solver's CUDA stream handle (int)."""
        s = C.c_void_p()
        check(lib().emg_five_stream(self._h, C.byref(s)))
        return s.value or 0

    @property
    def t(self):
        v = C.c_double()
        check(lib().emg_five_get_time(self._h, C.byref(v)))
        return v.value
