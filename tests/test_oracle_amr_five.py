"""CPU checks of the block-AMR oracle for the five-equation system
(Amr<7, FiveEq>, fluid/crates/compressible/src/amr.rs with multiphase.rs).

The reference has no asserted AMR tests; as for the Euler hierarchy
(tests/test_oracle_amr.py), the AMR restatement is pinned to the uniform
five-equation solver (itself pinned to the reference's tests and published
results, tests/test_oracle_five.py): a one-level hierarchy and a fully refined
one must advance like the uniform grid of the same spacing, up to the rounding
of dividing by dx (amr.rs:1273) where the uniform solver multiplies by 1/dx
(solver.rs:438), including the α equation's non-conservative term and the
dilatation limit of the CFL step. Refluxing keeps the conserved variables
(partial densities, momentum, energy) exact across levels."""
import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.five import five_initial_state
from emergence_b200.physics import Bc, FluxMode, Mesh
from oracle import pyoracle as O


def leaf_field(a, cfg, level):
    b = cfg["b"]
    nb = cfg["base_blocks"][0] << level
    st, data = a.structure(), a.download()
    out = np.full((nb * b, nb * b, 7), np.nan)
    for bid, (l, i, j, k, leaf) in enumerate(st):
        if l == level and leaf:
            out[i * b:(i + 1) * b, j * b:(j + 1) * b] = data[bid].reshape(b, b, 7)
    return out


def uniform(sys_, n, init, bc, mode):
    mesh = Mesh.new((n, n, 1), (0, 0, 0), (1, 1, 1), ng=5)
    x = np.stack([c.ravel() for c in mesh.centres()], axis=1)
    u = five_initial_state(sys_, mesh, init(x).reshape(n, n, 1, 7))
    return O.FiveOracleSolver(sys_, mesh, u, bc=bc, mode=mode, cfl=0.4), mesh


@pytest.mark.parametrize("mode", [FluxMode.Weno, FluxMode.Hybrid])
def test_single_level_hierarchy_matches_the_uniform_five_equation_solver(mode):
    sys_, cfg, lo, hi, bc, init = W.two_phase_amr_bubble(dim=2, base=4, levels=1)
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=mode)
    n = cfg["base_blocks"][0] * cfg["b"]
    u, mesh = uniform(sys_, n, init, bc, mode)
    for _ in range(4):
        dt = a.dt_cfl()
        assert abs(dt / u.dt_cfl() - 1.0) < 1e-14  # acoustic and dilatation limits alike
        a.step(dt)
        u.step(dt)
    fa = leaf_field(a, cfg, 0)
    fu = mesh.interior(u.download())[:, :, 0, :]
    err = np.abs(fa - fu).sum(axis=(0, 1)) / np.maximum(np.abs(fu).sum(axis=(0, 1)), 1e-300)
    assert np.all(err[[0, 1, 2, 5, 6]] < 1e-13), err


def test_fully_refined_hierarchy_matches_the_uniform_finest_grid():
    sys_, cfg, lo, hi, bc, init = W.two_phase_amr_bubble(dim=2, base=2, levels=2, eps=0.0)
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    st = a.structure()
    assert (st[st[:, 4] == 1, 0] == 1).all()
    n = cfg["base_blocks"][0] * cfg["b"] * 2
    u, mesh = uniform(sys_, n, init, bc, FluxMode.Weno)
    for _ in range(3):
        dt = a.dt_cfl()
        a.step(dt)
        u.step(dt)
    fa = leaf_field(a, cfg, 1)
    fu = mesh.interior(u.download())[:, :, 0, :]
    err = np.abs(fa - fu).sum(axis=(0, 1)) / np.maximum(np.abs(fu).sum(axis=(0, 1)), 1e-300)
    assert np.all(err[[0, 1, 2, 5, 6]] < 1e-13), err


def test_refluxing_conserves_the_conserved_variables_across_levels():
    """Periodic sides and a threshold at which the hierarchy stays fixed: the
    partial densities, the momentum and the energy are conserved to rounding
    across coarse–fine faces (the α equation is non-conservative)."""
    sys_, cfg, lo, hi, bc, init = W.two_phase_amr_bubble(dim=2, base=4, levels=3, eps=0.03)
    bc = [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    st0 = a.structure()
    assert len(set(st0[st0[:, 4] == 1, 0].tolist())) >= 2
    t0 = a.totals()
    for _ in range(4):
        a.step(a.dt_cfl())
    assert np.array_equal(a.structure(), st0)
    t1 = a.totals()
    for q in (0, 1, 2, 5):
        assert abs(t1[q] - t0[q]) <= 1e-12 * abs(t0[q]), (q, t0, t1)
