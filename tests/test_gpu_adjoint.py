"""Discrete adjoint of the uniform-grid FP64 step on the GPU (needs a B200).

The reference has no adjoint; its gradients are pinned two ways on the same
inputs and the same (recorded, frozen) time steps:
  * the CPU f64 forward-mode dual-number run of the oracle's restatement of
    the reference scheme (oracle/dual.hpp): <∇J, δ> must equal the dual
    directional derivative to rounding (relative 1e-10);
  * central finite differences of the GPU forward run with h = 1e-6 along a
    seeded direction (relative 1e-5, the stated bar).
"""
import math

import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.adjoint import OBJ_ENERGY, OBJ_PRESSURE
from emergence_b200.physics import Bc, Euler, FluxMode, Mesh, Nasg, initial_state
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

DUAL_TOL = 1e-10
FD_TOL = 1e-5


def make(sys_, mesh, u, bc, **k):
    from emergence_b200 import DifferentiableSolver
    return DifferentiableSolver(sys_, mesh, u, bc=bc, **k)


def padded(mesh, w):
    out = np.zeros((mesh.len(), 5))
    mesh.interior(out)[...] = w
    return out


def cons_of(sys_, mesh, wp, bc):
    """to_cons of padded primitives computed by the oracle (as the dual run does)."""
    _, _, u, _ = O.dual_run(sys_, mesh, wp, np.zeros_like(wp), 0.0, [], OBJ_PRESSURE, [0, 0, 0], [0, 0, 0], bc,
                            want_state=True)
    return u


def direction(mesh, seed, fields=(0,)):
    rng = np.random.default_rng(seed)
    d = np.zeros((mesh.len(), 5))
    di = mesh.interior(d)
    for k in fields:
        di[..., k] = rng.uniform(-1.0, 1.0, di.shape[:-1])
    return d


def check_against_dual(sys_, mesh, w, bc, nsteps, box, kind=OBJ_PRESSURE, fields=(0,), dgamma=0.37, seed=5,
                       positivity=True, every=0):
    wp = padded(mesh, w)
    u0 = cons_of(sys_, mesh, wp, bc)
    g = make(sys_, mesh, u0, bc, positivity=positivity)
    taken = g.forward(nsteps, checkpoint_every=every)
    assert taken == nsteps
    dts = g.dts()
    J = g.objective(kind, box[0], box[1])
    ub, wb, gam = g.backward()
    dw = direction(mesh, seed, fields)
    Jd, dJ = O.dual_run(sys_, mesh, wp, dw, dgamma, dts, kind, box[0], box[1], bc, positivity=positivity)
    adj = float((mesh.interior(wb) * mesh.interior(dw)).sum() + gam[1] * dgamma)
    assert abs(J - Jd) <= 1e-13 * abs(Jd), (J, Jd)
    assert abs(adj - dJ) <= DUAL_TOL * max(abs(dJ), 1e-30), (adj, dJ, abs(adj - dJ) / abs(dJ))
    g.close()
    return adj, dJ


def test_forward_run_matches_the_oracle_bitwise():
    sys_, mesh, w, bc = W.explosion_prim((40, 36, 1), 0.3)
    wp = padded(mesh, w)
    u0 = cons_of(sys_, mesh, wp, bc)
    g = make(sys_, mesh, u0, bc)
    assert g.forward(10) == 10
    o = O.OracleSolver(sys_, mesh, u0, bc=bc, mode=FluxMode.Weno)
    dts = []
    for _ in range(10):
        dts.append(o.dt_cfl())
        o.step(dts[-1])
    assert np.array_equal(g.dts(), np.array(dts))
    assert np.array_equal(mesh.interior(g.download()), mesh.interior(o.download()))
    g.close()


def test_explosion_2d_gradient_matches_dual_numbers():
    sys_, mesh, w, bc = W.explosion_prim((40, 36, 1), 0.3)
    check_against_dual(sys_, mesh, w, bc, 16, ([0.6, 0.6, 0.0], [0.9, 0.9, 0.0]))


def test_energy_objective_and_all_primitive_directions():
    sys_, mesh, w, bc = W.explosion_prim((32, 30, 1), 0.3)
    w = w.copy()
    rng = np.random.default_rng(2)
    w[..., 1] = 0.1 * rng.uniform(-1, 1, w.shape[:-1])  # moving gas: every field enters
    w[..., 2] = 0.1 * rng.uniform(-1, 1, w.shape[:-1])
    check_against_dual(sys_, mesh, w, bc, 10, ([0.5, 0.0, 0.0], [1.0, 1.0, 0.0]), kind=OBJ_ENERGY,
                       fields=(0, 1, 2, 4))


@pytest.mark.parametrize("kinds", [(Bc.Periodic, Bc.Periodic), (Bc.Reflect, Bc.Outflow)])
def test_3d_gradient_with_periodic_and_reflecting_boundaries(kinds):
    sys_, mesh, w, _ = W.explosion_prim((12, 10, 8), 0.3)
    bc = [[kinds[0], kinds[1]] for _ in range(3)]
    w = w.copy()
    w[..., 3] = 0.05
    check_against_dual(sys_, mesh, w, bc, 6, ([0.5, 0.0, 0.0], [1.0, 0.6, 1.0]), fields=(0, 3, 4))


def test_1d_gradient_with_a_dirichlet_inflow():
    sys_ = Euler(Nasg.ideal(1.4))
    n = 64
    mesh = Mesh.new((n, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ng=6)
    x = (np.arange(n) + 0.5) / n
    w = np.zeros((n, 1, 1, 5))
    w[:, 0, 0, 0] = np.where(x < 0.5, 1.0, 0.125)
    w[:, 0, 0, 1] = 0.2
    w[:, 0, 0, 4] = np.where(x < 0.5, 1.0, 0.1)
    inflow = sys_.to_cons(np.array([1.0, 0.2, 0.0, 0.0, 1.0]))
    bc = [[Bc.dirichlet(inflow), Bc.Outflow], [Bc.Periodic, Bc.Periodic], [Bc.Periodic, Bc.Periodic]]
    check_against_dual(sys_, mesh, w, bc, 20, ([0.5, 0, 0], [1.0, 0, 0]), fields=(0, 1, 4))


def test_limited_faces_are_differentiated_with_the_blend_held_fixed():
    """A 10^5 pressure jump (tests/cpu.rs:134-152): the positivity limiter
    fires, its blend weight is recorded and held, and the gradient still
    matches the dual-number run (whose bisection weight has zero tangent)."""
    sys_ = Euler(Nasg.ideal(1.4))
    n = 48
    mesh = Mesh.new((n, 1, 1), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ng=6)
    x = (np.arange(n) + 0.5) / n
    w = np.zeros((n, 1, 1, 5))
    w[:, 0, 0, 0] = np.where(x < 0.5, 1.0, 0.01)
    w[:, 0, 0, 4] = np.where(x < 0.5, 1000.0, 0.01)
    bc = [[Bc.Outflow, Bc.Outflow], [Bc.Periodic, Bc.Periodic], [Bc.Periodic, Bc.Periodic]]
    wp = padded(mesh, w)
    u0 = cons_of(sys_, mesh, wp, bc)
    o = O.OracleSolver(sys_, mesh, u0, bc=bc, mode=FluxMode.Weno)
    for _ in range(6):
        o.step(o.dt_cfl())
    assert o.counters()[3] > 0  # limited faces occurred
    check_against_dual(sys_, mesh, w, bc, 6, ([0.3, 0, 0], [0.9, 0, 0]), fields=(0, 4))


def test_checkpoint_interval_does_not_change_the_gradient():
    sys_, mesh, w, bc = W.explosion_prim((24, 20, 1), 0.3)
    u0 = initial_state(sys_, mesh, w)
    out = []
    for every in (1, 3, 0, 12):
        g = make(sys_, mesh, u0, bc)
        g.forward(12, checkpoint_every=every)
        g.objective(OBJ_PRESSURE, [0.5, 0.5, 0], [1, 1, 0])
        out.append(g.backward())
        g.close()
    for ub, wb, gam in out[1:]:
        assert np.array_equal(ub, out[0][0]) and np.array_equal(wb, out[0][1]) and np.array_equal(gam, out[0][2])


def test_step_vjp_equals_a_one_step_backward_pass():
    sys_, mesh, w, bc = W.explosion_prim((24, 20, 1), 0.3)
    u0 = initial_state(sys_, mesh, w)
    g = make(sys_, mesh, u0, bc)
    g.forward(1)
    dt = g.dts()[0]
    rng = np.random.default_rng(9)
    ybar = padded(mesh, rng.normal(size=mesh.interior(u0).shape))
    g.seed(ybar)
    ub, _, gam = g.backward()
    ub1, g1 = g.step_vjp(u0, dt, ybar)
    assert np.array_equal(mesh.interior(ub), mesh.interior(ub1))
    assert gam[0] == g1
    g.close()


def test_gradient_matches_central_finite_differences():
    """FD of the GPU forward run along a seeded direction of (ρ⁰, γ), h = 1e-6,
    with the recorded time steps held fixed."""
    sys_, mesh, w, bc = W.explosion_prim((48, 48, 1), 0.3)
    box = ([0.7, 0.7, 0.0], [0.9, 0.9, 0.0])
    u0 = initial_state(sys_, mesh, w)
    g = make(sys_, mesh, u0, bc)
    g.forward(40)
    dts = g.dts()
    g.objective(OBJ_PRESSURE, *box)
    _, wb, gam = g.backward()
    dw = direction(mesh, 11)
    dgamma = 0.5
    adj = float((mesh.interior(wb) * mesh.interior(dw)).sum() + gam[1] * dgamma)
    h = 1e-6

    def J(s):
        sys2 = Euler(Nasg.ideal(1.4 + s * dgamma))
        w2 = w + s * mesh.interior(dw)
        g2 = make(sys2, mesh, initial_state(sys2, mesh, w2), bc)
        g2.forward(dts=dts)
        v = g2.objective(OBJ_PRESSURE, *box)
        g2.close()
        return v

    fd = (J(h) - J(-h)) / (2 * h)
    assert abs(fd - adj) <= FD_TOL * abs(adj), (fd, adj, abs(fd - adj) / abs(adj))
    g.close()


def test_invalid_options_are_rejected():
    from emergence_b200 import DifferentiableSolver, EmgError
    sys_, mesh, u, bc = W.explosion((16, 16, 1), 0.3)
    with pytest.raises(EmgError):
        DifferentiableSolver(sys_, mesh, u, bc=[[Bc.characteristic(sys_.to_cons(np.array([1, 0, 0, 0, 1.0]))),
                                                 Bc.Outflow]] * 3)
    g = make(sys_, mesh, u, bc)
    with pytest.raises(EmgError):
        g.backward()  # no recorded run
    g.forward(2)
    with pytest.raises(EmgError):
        g.backward()  # nothing seeded
    g.close()


def test_step_vjp_matches_the_cpu_restatement_at_a_shock():
    """One step's reverse on the GPU against tests/native's plain-loop CPU
    restatement built from the same vector–Jacobian products, on a state
    with a shock (2-D explosion after 8 steps)."""
    import ctypes as C
    import os
    import subprocess
    import test_adjoint_host as H
    os.makedirs(os.path.dirname(H.OUT), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-Wno-unknown-pragmas",
                    "-I", "/usr/local/cuda/include", H.SRC, "-o", H.OUT], check=True)
    L = C.CDLL(H.OUT)
    sys_, mesh, u0, bc = W.explosion((32, 28, 1), 0.3)
    o = O.OracleSolver(sys_, mesh, u0, bc=bc, mode=FluxMode.Weno)
    for _ in range(8):
        o.step(o.dt_cfl())
    u = o.download()
    dt = o.dt_cfl()
    rng = np.random.default_rng(4)
    yb = padded(mesh, rng.normal(size=mesh.interior(u).shape))
    g = make(sys_, mesh, u, bc)
    ub_gpu, gb_gpu = g.step_vjp(u, dt, yb)
    g.close()
    ub_cpu, gb_cpu = H.step_vjp_cpu(L, mesh, H.eos_of(), bc, True, u, dt, yb)
    scale = np.abs(ub_cpu).max()
    assert np.abs(mesh.interior(ub_gpu) - mesh.interior(ub_cpu)).max() <= 1e-10 * scale
    assert abs(gb_gpu - gb_cpu) <= 1e-10 * abs(gb_cpu)
