"""CPU checks of the block-AMR oracle (C++ restatement of
fluid/crates/compressible/src/amr.rs). The reference has no asserted AMR
tests; these pin the properties its design documents state: exact
conservation across levels by refluxing (amr.rs:30-33), 2:1 balance
(amr.rs:23), agreement with the uniform solver when the hierarchy is one
level or fully refined (the comparison examples/amr_validate.rs makes)."""
import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.physics import Bc, Euler, FluxMode, Mesh, Nasg, initial_state
from oracle import pyoracle as O


def leaf_field(a, cfg, level):
    """Assemble the leaves of one level into a dense 2-D array (NaN where absent)."""
    b = cfg["b"]
    nb = cfg["base_blocks"][0] << level
    st, data = a.structure(), a.download()
    out = np.full((nb * b, nb * b, 5), np.nan)
    for bid, (l, i, j, k, leaf) in enumerate(st):
        if l == level and leaf:
            out[i * b:(i + 1) * b, j * b:(j + 1) * b] = data[bid].reshape(b, b, 5)
    return out


def uniform_reference(n, init, bc, mode, steps, dt_fn=None):
    sys_ = Euler(Nasg.ideal(1.4))
    mesh = Mesh.new((n, n, 1), (0, 0, 0), (1, 1, 1), ng=5)
    x = np.stack([c.ravel() for c in mesh.centres()], axis=1)
    w = init(x).reshape(n, n, 1, 5)
    u = initial_state(sys_, mesh, w)
    return O.OracleSolver(sys_, mesh, u, bc=bc, mode=mode, cfl=0.4), mesh


def test_refluxing_conserves_mass_and_energy_across_levels():
    sys_, cfg, lo, hi, bc, init = W.amr_explosion(dim=2, base=4, levels=3, radius=0.25)
    bc = [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    st = a.structure()
    assert len(set(st[st[:, 4] == 1, 0])) >= 2  # leaves on more than one level
    t0 = a.totals()
    for _ in range(3):  # the first regrid is due after step 4; regrids are not conservative
        a.step(a.dt_cfl())
    t1 = a.totals()
    assert abs(t1[0] - t0[0]) <= 1e-13 * abs(t0[0])
    assert abs(t1[4] - t0[4]) <= 1e-13 * abs(t0[4])


def test_neighbouring_leaves_differ_by_at_most_one_level():
    sys_, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    for _ in range(6):
        a.step(a.dt_cfl())
    b = cfg["b"]
    lv = cfg["levels"] - 1
    n = cfg["base_blocks"][0] * b << lv
    level_of = np.full((n, n), -1)
    for (l, i, j, k, leaf) in a.structure():
        if leaf:
            s = b << (lv - l)
            level_of[i * s:(i + 1) * s, j * s:(j + 1) * s] = l
    assert (level_of >= 0).all()
    assert np.abs(np.diff(level_of, axis=0)).max() <= 1
    assert np.abs(np.diff(level_of, axis=1)).max() <= 1


@pytest.mark.parametrize("mode", [FluxMode.Weno, FluxMode.Hybrid])
def test_single_level_hierarchy_matches_the_uniform_solver(mode):
    sys_, cfg, lo, hi, bc, init = W.amr_explosion(dim=2, base=4, levels=1, radius=0.3)
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=mode)
    n = cfg["base_blocks"][0] * cfg["b"]
    u, mesh = uniform_reference(n, init, bc, mode, 0)
    for _ in range(4):
        dt = a.dt_cfl()
        assert abs(dt / u.dt_cfl() - 1.0) < 1e-14
        a.step(dt)
        u.step(dt)
    fa = leaf_field(a, cfg, 0)
    fu = mesh.interior(u.download())[:, :, 0, :]
    # AMR divides by dx where the uniform solver multiplies by 1/dx
    # (C/amr.rs:1263 vs C/solver.rs:431-438): equal up to rounding
    err = np.abs(fa - fu).sum(axis=(0, 1)) / np.maximum(np.abs(fu).sum(axis=(0, 1)), 1e-300)
    assert np.all(err[[0, 4]] < 1e-13), err


def test_fully_refined_hierarchy_matches_the_uniform_finest_grid():
    sys_, cfg, lo, hi, bc, init = W.amr_explosion(dim=2, base=2, levels=2, radius=0.3, eps=0.0)
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    st = a.structure()
    assert (st[st[:, 4] == 1, 0] == 1).all()  # every leaf on the finest level
    n = cfg["base_blocks"][0] * cfg["b"] * 2
    u, mesh = uniform_reference(n, init, bc, FluxMode.Weno, 0)
    for _ in range(3):
        dt = a.dt_cfl()
        a.step(dt)
        u.step(dt)
    fa = leaf_field(a, cfg, 1)
    fu = mesh.interior(u.download())[:, :, 0, :]
    err = np.abs(fa - fu).sum(axis=(0, 1)) / np.maximum(np.abs(fu).sum(axis=(0, 1)), 1e-300)
    assert np.all(err[[0, 4]] < 1e-13), err


def test_regrid_refines_where_the_detail_is_large_and_coarsens_smooth_regions():
    sys_, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    a = O.OracleAmr(sys_, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    det = a.details()
    st = a.structure()
    leaves = st[:, 4] == 1
    fine = leaves & (st[:, 0] == cfg["levels"] - 1)
    coarse = leaves & (st[:, 0] < cfg["levels"] - 1)
    # refined leaves sit on the features; leaves left coarse are below eps
    assert fine.any() and coarse.any()
    assert det[coarse].max() <= cfg["eps"]
