"""Seeded synthetic initial data of the benchmark workloads.

Noise: SplitMix64 keyed by (seed, global interior cell index) → uniform in
[−1, 1) from the top 53 bits, so any sub-box or any rank regenerates the same
values. The default seed is 20261203.
"""
import numpy as np

from .physics import Bc, Euler, Mesh, Nasg, initial_state

SEED = 20261203
_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    """SplitMix64 finaliser of uint64 array x (wrapping arithmetic)."""
    with np.errstate(over="ignore"):
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform_pm1(seed, index):
    """Uniform in [−1, 1) for each uint64 index, keyed by seed."""
    with np.errstate(over="ignore"):
        key = splitmix64(np.uint64(seed) * np.uint64(0x100000001B3)) ^ index.astype(np.uint64)
        r = splitmix64(key) >> np.uint64(11)
    return r.astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0


def explosion(n, radius, seed=SEED, gamma=1.4, noise=0.01, ng=6):
    """Circular/spherical explosion on [0,1]^D: ρ = 1, p = 1 for r < radius
    about the centre, ρ = 0.125, p = 0.1 outside, u = 0, with ρ ← ρ(1 + noise·ξ).
    Returns (sys, mesh, u_padded, bc) with transmissive (Outflow) boundaries."""
    n = tuple(list(n) + [1] * (3 - len(n)))
    sys = Euler(Nasg.ideal(gamma))
    lo = (0.0, 0.0, 0.0)
    hi = tuple(1.0 if n[d] > 1 else 1.0 for d in range(3))
    mesh = Mesh.new(n, lo, hi, ng=ng)
    x = mesh.centres()
    r2 = np.zeros(n)
    for d in range(3):
        if n[d] > 1:
            r2 = r2 + (x[d] - 0.5) ** 2
    inside = np.sqrt(r2) < radius
    idx = np.arange(mesh.cells(), dtype=np.uint64).reshape(n)
    xi = uniform_pm1(seed, idx)
    w = np.zeros(n + (5,))
    w[..., 0] = np.where(inside, 1.0, 0.125) * (1.0 + noise * xi)
    w[..., 4] = np.where(inside, 1.0, 0.1)
    u = initial_state(sys, mesh, w)
    bc = [[Bc.Outflow, Bc.Outflow] for _ in range(3)]
    return sys, mesh, u, bc


def explosion_2d(n=256, seed=SEED):
    """2-D circular explosion, radius 0.4 (the reference CPU-path case)."""
    return explosion((n, n, 1), 0.4, seed)


def explosion_3d(n=256, seed=SEED):
    """3-D spherical explosion, radius 0.3."""
    return explosion((n, n, n), 0.3, seed)
