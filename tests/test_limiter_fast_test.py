"""The division-free admissibility test that the sweep's positivity limiter
tries first (Sweep::surely_admissible, ideal gas) never accepts a state that
the reference's test (to_prim then admissible, C/system.rs:197-203,404-407)
rejects, so the limiter decides exactly as the reference does. Restated here
with numpy in the same IEEE double operations (host, no GPU), over states
spread across the admissibility boundary."""
import numpy as np


def surely_admissible(a):
    r, E = a[:, 0], a[:, 4]
    ok = (r > 1e-100) & (r < 1e100) & (E > 1e-100) & (E < 1e100)
    for k in (1, 2, 3):
        ok &= np.abs(a[:, k]) < 1e100
    m2 = a[:, 1] * a[:, 1] + a[:, 2] * a[:, 2] + a[:, 3] * a[:, 3]
    twore = 2.0 * r * E
    return ok & (twore - m2 > 1e-11 * (twore + m2))


def reference_admissible(a, gamma):
    with np.errstate(all="ignore"):
        rho = a[:, 0]
        vx, vy, vz = a[:, 1] / rho, a[:, 2] / rho, a[:, 3] / rho
        ein = a[:, 4] / rho - 0.5 * (vx * vx + vy * vy + vz * vz)
        v = 1.0 / rho
        p = (gamma - 1.0) * (ein - 0.0) / (v - 0.0) - gamma * 0.0
        return np.isfinite(rho) & np.isfinite(p) & (rho > 0) & (1.0 / rho > 0.0) & (p + 0.0 > 0)


def states(n, rng, rel):
    """Conserved states whose 2ρE − |ρu|² is rel·(2ρE + |ρu|²)-ish."""
    rho = 10.0 ** rng.uniform(-6, 6, n)
    m = rng.normal(size=(n, 3)) * 10.0 ** rng.uniform(-6, 6, (n, 1))
    m2 = (m * m).sum(axis=1)
    E = m2 / (2 * rho) * (1 + rel)
    a = np.column_stack([rho, m, E])
    return a


def test_fast_test_never_accepts_what_the_reference_rejects():
    rng = np.random.default_rng(20261203)
    for gamma in (1.4, 5.0 / 3.0, 1.1, 50.0):
        for rel in (rng.uniform(-1e-9, 1e-9, 200000), rng.uniform(-1e-13, 1e-13, 200000),
                    rng.uniform(-1.0, 1.0, 200000), 10.0 ** rng.uniform(-16, 2, 200000)):
            a = states(len(rel), rng, rel)
            fast, ref = surely_admissible(a), reference_admissible(a, gamma)
            assert not np.any(fast & ~ref), int(np.sum(fast & ~ref))


def test_fast_test_accepts_ordinary_states():
    rng = np.random.default_rng(7)
    rho = rng.uniform(0.1, 10, 100000)
    u = rng.uniform(-3, 3, (100000, 3))
    p = rng.uniform(0.01, 10, 100000)
    E = p / 0.4 + 0.5 * rho * (u * u).sum(axis=1)
    a = np.column_stack([rho, rho[:, None] * u, E])
    assert surely_admissible(a).mean() > 0.999


def test_fast_test_rejects_extremes_and_non_finite_values():
    a = np.array([[1.0, 0, 0, 0, 1.0],          # ordinary
                  [0.0, 0, 0, 0, 1.0],          # ρ = 0
                  [-1.0, 0, 0, 0, 1.0],         # ρ < 0
                  [1.0, 2.0, 0, 0, 1.0],        # p < 0
                  [np.nan, 0, 0, 0, 1.0],
                  [1.0, 0, 0, 0, np.inf],
                  [1e-200, 0, 0, 0, 1e-200]])   # outside the bounded range: left to the full test
    assert list(surely_admissible(a)) == [True, False, False, False, False, False, False]
