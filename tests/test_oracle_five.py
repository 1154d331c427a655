"""Pinning of the five-equation oracle (oracle/five_oracle.hpp, host only).

The restatement of fluid/crates/compressible/src/multiphase.rs and of the
system-generic step it drives is held to what the reference itself states:
its integration tests for the five-equation CFL step
(fluid/crates/compressible/tests/cpu.rs:1-55), and its published validation
results for the model (analysis/compressible.md:27-29 from
examples/multiphase_validate.rs): Wood's mixture sound speed at every
fraction, an interface advected one period keeping pressure and velocity
uniform, and the water/air shock tube converging to the exact solution.
"""
import numpy as np
import pytest

from emergence_b200.five import FiveEq, five_initial_state
from emergence_b200.physics import Bc, FluxMode, Mesh, Nasg
from oracle import pyoracle as O

AIR = Nasg(1.4, 0.0, 0.0, 0.0, 717.5)           # eos.rs:86
WATER_SG = Nasg(4.4, 6.0e8, 0.0, 0.0, 1.0)      # eos.rs:88
EPS = 1e-8                                       # multiphase_validate.rs:14


def prim(alpha, rho_w, rho_a, u, p):
    """multiphase_validate.rs:17-25."""
    w = np.zeros(7)
    w[0] = alpha * rho_w
    w[1] = (1.0 - alpha) * rho_a
    w[2] = u
    w[5] = p
    w[6] = alpha
    return w


def test_mixture_sound_speed_is_woods():
    """multiphase_validate.rs:120-134; analysis/compressible.md:27 (1625 m/s →
    119 m/s at 1 % air → 23.6 m/s at 50 %)."""
    sys = FiveEq((WATER_SG, AIR), kapila=True)
    p = 1e5
    seen = {}
    for a_air in (0.0, 1e-4, 1e-2, 0.1, 0.5, 0.9, 1.0):
        alpha = min(max(1.0 - a_air, EPS), 1.0 - EPS)
        w = prim(alpha, 1000.0, 1.2, 0.0, p)
        rho = w[0] + w[1]
        zw = WATER_SG.gamma * (p + WATER_SG.p_inf)
        za = AIR.gamma * p
        wood = np.sqrt(1.0 / (rho * (alpha / zw + (1.0 - alpha) / za)))
        c = O.five_props(sys, w)[0]
        assert abs(c / wood - 1.0) < 1e-9, (a_air, c, wood)
        seen[a_air] = c
    assert abs(seen[0.0] - 1625.0) < 0.5
    assert abs(seen[1e-2] - 119.0) < 0.5
    assert abs(seen[0.5] - 23.6) < 0.05


def gas_liquid(bc):
    """tests/cpu.rs:2-24: 8 cells of a liquid-dominated mixture moving at 0.2."""
    sys = FiveEq((Nasg(2.0, 1e6), Nasg.ideal(1.4)), kapila=True)
    mesh = Mesh.new((8, 1, 1), (0, 0, 0), (1, 1, 1), ng=6)
    w0 = np.array([0.99999 * 1000.0, 0.00001 * 0.001, 0.2, 0.0, 0.0, 100.0, 0.99999])
    u = five_initial_state(sys, mesh, np.broadcast_to(w0, (8, 1, 1, 7)).copy())
    # s.prim(0, 0, 0): the primitive state of the stored conserved one
    return sys, mesh, u, sys.to_prim(mesh.interior(u)[0, 0, 0])


def test_cfl_at_a_reflecting_wall_includes_the_dilatation_limit():
    """tests/cpu.rs:25-43: with reflecting walls the boundary cells see
    ∇·u = u/dx, so dt = min(acoustic, 0.5/dilatation rate), and poisoning only
    the ghost cells does not change it."""
    sys, mesh, u, w = gas_liquid(None)
    bc = [[Bc.Reflect, Bc.Reflect], [Bc.Periodic] * 2, [Bc.Periodic] * 2]
    c, _, _, _ = O.five_props(sys, w)
    dx = mesh.dx[0]
    acoustic = 0.5 * dx / (abs(w[2]) + c)
    source = 0.5 / O.five_props(sys, w, w[2] / dx)[1]
    expected = min(acoustic, source)
    assert source < 0.1 * acoustic
    o = O.FiveOracleSolver(sys, mesh, u, bc=bc)
    assert abs(o.dt_cfl() / expected - 1.0) < 1e-13
    bad = u.copy()
    g = mesh.g(0)
    for i in range(mesh.m(0)):
        if i < g or i >= g + 8:
            bad[i] = np.nan
    o2 = O.FiveOracleSolver(sys, mesh, bad, bc=bc)
    assert abs(o2.dt_cfl() / expected - 1.0) < 1e-13


@pytest.mark.parametrize("kind", [Bc.Periodic, Bc.Outflow])
def test_uniform_flow_gets_no_spurious_boundary_limit(kind):
    """tests/cpu.rs:44-54."""
    sys, mesh, u, w = gas_liquid(None)
    bc = [[kind, kind], [Bc.Periodic] * 2, [Bc.Periodic] * 2]
    c = O.five_props(sys, w)[0]
    expected = 0.5 * mesh.dx[0] / (abs(w[2]) + c)
    o = O.FiveOracleSolver(sys, mesh, u, bc=bc)
    assert abs(o.dt_cfl() / expected - 1.0) < 1e-13


@pytest.mark.parametrize("mode", [FluxMode.Weno, FluxMode.Hybrid])
def test_interface_advection_keeps_pressure_and_velocity_uniform(mode):
    """multiphase_validate.rs:27-58; analysis/compressible.md:28: a water slab
    in air advected one period at u = 100, p = 1 bar keeps |Δp|/p ≤ 2e-10 and
    |Δu|/u ≤ 1e-11."""
    sys = FiveEq((WATER_SG, AIR), kapila=True)
    u0, p0, n = 100.0, 1e5, 100
    mesh = Mesh.new((n, 1, 1), (0, 0, 0), (1, 1, 1), ng=6)
    x = mesh.centres()[0]
    w = np.zeros((n, 1, 1, 7))
    for i in range(n):
        a = 1.0 - EPS if 0.25 <= x[i, 0, 0] < 0.75 else EPS
        w[i, 0, 0] = prim(a, 1000.0, 1.2, u0, p0)
    u = five_initial_state(sys, mesh, w)
    o = O.FiveOracleSolver(sys, mesh, u, cfl=0.4, mode=mode)
    o.run_to(1.0 / u0)
    wf = sys.to_prim(mesh.interior(o.download()).reshape(n, 7))
    dp = np.max(np.abs(wf[:, 5] - p0)) / p0
    du = np.max(np.abs(wf[:, 2] - u0)) / u0
    print(mode, "dp/p", dp, "du/u", du)
    assert dp <= 2e-10 and du <= 1e-11


def test_water_air_tube_converges_to_the_exact_solution():
    """multiphase_validate.rs:59-100; analysis/compressible.md:29 (L1(ρ)
    1.0e-3 and L1(p) 3.8e-4 at N = 1600): at N = 200 and 400 the errors fall
    at about first order toward those values."""
    sys = FiveEq((WATER_SG, AIR), kapila=True)
    rw, pw, ra, pa = 1000.0, 1e9, 50.0, 1e5
    x0, t_end = 0.7, 2.4e-4
    errs = []
    for n in (200, 400):
        mesh = Mesh.new((n, 1, 1), (0, 0, 0), (1, 1, 1), ng=6)
        x = mesh.centres()[0][:, 0, 0]
        w = np.array([prim(1.0 - EPS, rw, ra, 0.0, pw) if xi < x0 else prim(EPS, rw, ra, 0.0, pa) for xi in x])
        u = five_initial_state(sys, mesh, w.reshape(n, 1, 1, 7))
        bc = [[Bc.Outflow, Bc.Outflow], [Bc.Periodic] * 2, [Bc.Periodic] * 2]
        o = O.FiveOracleSolver(sys, mesh, u, bc=bc, cfl=0.4, mode=FluxMode.Weno)
        o.run_to(t_end)
        wf = sys.to_prim(mesh.interior(o.download()).reshape(n, 7))
        ex = O.exact_sample([rw, 0.0, pw], [ra, 0.0, pa], (x - x0) / t_end, WATER_SG, AIR)
        rho = wf[:, 0] + wf[:, 1]
        e_rho = np.mean(np.abs(rho - ex[:, 0])) / np.mean(ex[:, 0])
        e_p = np.mean(np.abs(wf[:, 5] - ex[:, 2])) / pw
        errs.append((e_rho, e_p))
        print("N", n, "L1(rho)/rho", e_rho, "L1(p)/pL", e_p)
    (r1, p1), (r2, p2) = errs
    # first order toward 1.0e-3 / 3.8e-4 at N = 1600
    assert r2 < r1 and p2 < p1
    assert r2 < 8 * 1.0e-3 * 1.6 and p2 < 8 * 3.8e-4 * 1.6
