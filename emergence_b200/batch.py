"""GpuBatch1D: many independent 1-D problems advanced together on the device
(each instance follows Solver::run_to of the reference on a 1-D mesh,
fluid/crates/compressible/src/solver.rs:758-768, with its own CFL dt)."""
import ctypes as C

import numpy as np

from ._abi import EmgBc, EmgEos, EmgOpts, check, lib
from .physics import Bc, FluxMode, Precision


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class GpuBatch1D:
    """``n[i]`` cells of size ``dx[i]`` per instance; ``u`` is the
    concatenated interior conserved data (float64 [Σn, 5])."""

    def __init__(self, sys, n, dx, u, bc=(Bc.Outflow, Bc.Outflow), cfl=0.5, mode=FluxMode.Weno, tol=1e-3,
                 positivity=True, precision=Precision.F64):
        self.n = np.ascontiguousarray(n, dtype=np.int64)
        self.dx = np.ascontiguousarray(dx, dtype=np.float64)
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != (int(self.n.sum()), 5):
            raise ValueError("u must have shape (sum(n), 5)")
        self._e = EmgEos(sys.eos.gamma, sys.eos.p_inf, sys.eos.b, sys.eos.q, sys.eos.cv)
        self._o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, precision, 0)
        self._b = (EmgBc * 2)()
        for s in range(2):
            self._b[s].kind = bc[s].kind
            for k in range(5):
                self._b[s].state[k] = bc[s].state[k]
        h = C.c_void_p()
        check(lib().emg_batch1d_create(C.byref(self._e), C.byref(self._o), self._b, len(self.n),
                                       self.n.ctypes.data_as(C.POINTER(C.c_int64)), _dptr(self.dx), _dptr(u),
                                       C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().emg_batch1d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run_to(self, t_end):
        n = C.c_uint64()
        check(lib().emg_batch1d_run_to(self._h, float(t_end), C.byref(n)))
        return n.value

    def download(self):
        out = np.zeros((int(self.n.sum()), 5))
        check(lib().emg_batch1d_download(self._h, _dptr(out)))
        return out

    def status(self):
        t = np.zeros(len(self.n))
        s = np.zeros(len(self.n), dtype=np.uint64)
        check(lib().emg_batch1d_status(self._h, _dptr(t), s.ctypes.data_as(C.POINTER(C.c_uint64))))
        return t, s

    def stream(self):
        p = C.c_void_p()
        check(lib().emg_batch1d_stream(self._h, C.byref(p)))
        return p.value

    def split(self, u):
        """Per-instance views of a concatenated [Σn, 5] array."""
        return np.split(u, np.cumsum(self.n)[:-1])

    # ---- discrete adjoint of a batched run (FP64 batches, WENO mode)
    def record(self, t_end, checkpoint_every=0):
        """Record an FP64 run of every instance from the initial state to
        t_end; returns the number of batch steps."""
        n = C.c_uint64()
        check(lib().emg_batch1d_record(self._h, float(t_end), int(checkpoint_every), C.byref(n)))
        return n.value

    def objective(self, kind, x_lo, x_hi):
        """Per-instance J over cells with centre in [x_lo, x_hi] (kind 0: Σ p·dx,
        1: Σ E·dx) on the recorded final state; seeds the backward pass."""
        J = np.zeros(len(self.n))
        check(lib().emg_batch1d_objective(self._h, int(kind), float(x_lo), float(x_hi), _dptr(J)))
        return J

    def backward(self, x_split, want_wbar=False):
        """∂J_i/∂(ρ_L, u_L, p_L, ρ_R, u_R, p_R) per instance ([ninst, 6]) for
        initial data constant on either side of x_split; with want_wbar also
        ∂J/∂W⁰ per cell ([Σn, 5])."""
        g = np.zeros((len(self.n), 6))
        wb = np.zeros((int(self.n.sum()), 5)) if want_wbar else None
        check(lib().emg_batch1d_backward(self._h, float(x_split), _dptr(g), _dptr(wb) if want_wbar else None))
        return (g, wb) if want_wbar else g

    def adjoint_times(self):
        """Device ms of [last recorded run, checkpoint recompute, reverse sweeps]."""
        ms = np.zeros(3)
        check(lib().emg_batch1d_adjoint_times(self._h, _dptr(ms)))
        return ms
