"""Batched adjoint gradients of independent 1-D Riemann problems (needs a B200).

Each instance's gradient of the right-half total energy with respect to its
six initial values (ρ, u, p left and right of x = 0.5) from one batched
backward pass is checked against the CPU dual-number run of the oracle's
restatement of the reference scheme, per instance and per direction, on the
same (recorded) time steps; and against central finite differences of the
batched GPU forward run.
"""
import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.adjoint import OBJ_ENERGY
from emergence_b200.physics import Bc, FluxMode, Mesh
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def batch(ninst=6, nmin=48, nmax=160, seed=7):
    return W.riemann_batch(ninst=ninst, nmin=nmin, nmax=nmax, seed=seed)


def make(sys_, n, dx, u):
    from emergence_b200 import GpuBatch1D
    return GpuBatch1D(sys_, n, dx, u, bc=(Bc.Outflow, Bc.Outflow))


def instance_prims(n_i, st, dx_i):
    x = (np.arange(n_i) + 0.5) * dx_i
    left = x < 0.5
    w = np.zeros((n_i, 5))
    w[:, 0] = np.where(left, st[0], st[3])
    w[:, 1] = np.where(left, st[1], st[4])
    w[:, 4] = np.where(left, st[2], st[5])
    return w, left


def test_batched_gradients_match_dual_numbers_per_instance():
    sys_, n, dx, u, st = batch()
    g = make(sys_, n, dx, u)
    B = g.record(0.15)
    assert B > 0
    J = g.objective(OBJ_ENERGY, 0.5, 1.0)
    grad = g.backward(0.5)
    g.close()
    bc = [[Bc.Outflow, Bc.Outflow], [Bc.Periodic, Bc.Periodic], [Bc.Periodic, Bc.Periodic]]
    offs = np.concatenate([[0], np.cumsum(n)])
    for i in range(len(n)):
        mesh = Mesh.new((int(n[i]), 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ng=6)
        uu = np.zeros((mesh.len(), 5))
        mesh.interior(uu)[...] = u[offs[i]:offs[i + 1]].reshape(int(n[i]), 1, 1, 5)
        o = O.OracleSolver(sys_, mesh, uu, bc=bc, mode=FluxMode.Weno)
        dts = []
        while o.t < 0.15 - 1e-10 * 0.15:
            dts.append(min(o.dt_cfl(), 0.15 - o.t))
            o.step(dts[-1])
        w, left = instance_prims(int(n[i]), st[i], dx[i])
        wp = np.zeros((mesh.len(), 5))
        mesh.interior(wp)[...] = w.reshape(int(n[i]), 1, 1, 5)
        for q, (side, field) in enumerate([(True, 0), (True, 1), (True, 4), (False, 0), (False, 1), (False, 4)]):
            dw = np.zeros_like(wp)
            sel = left if side else ~left
            mesh.interior(dw)[sel.reshape(-1, 1, 1), field] = 1.0
            Jd, dJ = O.dual_run(sys_, mesh, wp, dw, 0.0, dts, OBJ_ENERGY, [0.5, 0, 0], [1.0, 0, 0], bc)
            assert abs(J[i] - Jd) <= 1e-12 * abs(Jd), (i, J[i], Jd)
            assert abs(grad[i, q] - dJ) <= 1e-9 * max(abs(dJ), 1e-12), (i, q, grad[i, q], dJ)


def test_batched_gradients_match_finite_differences():
    sys_, n, dx, u, st = batch(ninst=4, seed=11)
    g = make(sys_, n, dx, u)
    g.record(0.15)
    g.objective(OBJ_ENERGY, 0.5, 1.0)
    grad = g.backward(0.5)
    g.close()
    h = 1e-6
    for q in range(6):
        Js = []
        for sgn in (1.0, -1.0):
            st2 = st.copy()
            st2[:, q] += sgn * h
            parts = []
            for i in range(len(n)):
                w, _ = instance_prims(int(n[i]), st2[i], dx[i])
                parts.append(sys_.to_cons(w))
            g2 = make(sys_, n, dx, np.concatenate(parts))
            g2.record(0.15)
            Js.append(g2.objective(OBJ_ENERGY, 0.5, 1.0))
            g2.close()
        fd = (Js[0] - Js[1]) / (2 * h)
        # the perturbed runs take their own CFL steps, so the quotient also
        # carries the small time-step sensitivity that the frozen-step adjoint
        # leaves out
        assert np.all(np.abs(fd - grad[:, q]) <= 1e-3 * np.maximum(np.abs(grad[:, q]), 1e-3)), (q, fd, grad[:, q])


def test_mixed_batch_gradients_follow_the_fp64_gradients():
    """A mixed (FP32-flux, FP64-state) batch records its own run and is
    differentiated with the FP64 step's transposed Jacobian at its recorded
    stage states: its gradients agree with the FP64 batch's to the mixed
    form's own error level (1e-6 relative), and its objective with the FP64
    objective likewise."""
    from emergence_b200 import GpuBatch1D
    from emergence_b200.physics import Precision
    sys_, n, dx, u, st = batch(ninst=8, seed=13)
    out = {}
    for prec in (Precision.F64, Precision.Mixed):
        g = GpuBatch1D(sys_, n, dx, u, bc=(Bc.Outflow, Bc.Outflow), precision=prec)
        g.record(0.15)
        J = g.objective(OBJ_ENERGY, 0.5, 1.0)
        out[prec] = (J, g.backward(0.5))
        g.close()
    (J64, g64), (Jm, gm) = out[Precision.F64], out[Precision.Mixed]
    assert np.all(np.abs(Jm - J64) <= 1e-6 * np.abs(J64)), (Jm, J64)
    scale = np.abs(g64).max(axis=1, keepdims=True)
    err = np.abs(gm - g64) / scale
    print("mixed vs FP64 batched gradients, max rel err", err.max())
    assert np.all(err <= 1e-6), err
