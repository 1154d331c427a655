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
    sys, mesh, w, bc = explosion_prim(n, radius, seed, gamma, noise, ng)
    return sys, mesh, initial_state(sys, mesh, w), bc


def explosion_prim(n, radius, seed=SEED, gamma=1.4, noise=0.01, ng=6):
    """The explosion of ``explosion`` as interior primitives: (sys, mesh, w, bc)
    with w of shape n + (5,)."""
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
    bc = [[Bc.Outflow, Bc.Outflow] for _ in range(3)]
    return sys, mesh, w, bc


def explosion_2d(n=256, seed=SEED):
    """2-D circular explosion, radius 0.4 (the reference CPU-path case)."""
    return explosion((n, n, 1), 0.4, seed)


def explosion_3d(n=256, seed=SEED):
    """3-D spherical explosion, radius 0.3."""
    return explosion((n, n, n), 0.3, seed)


# ---------------------------------------------------------------- block AMR
def rankine_hugoniot(mach, gamma=1.4, rho1=1.0, p1=1.0):
    """Post-shock (ρ, u, p) and shock speed of a shock moving into gas at rest."""
    m2 = mach * mach
    rho2 = rho1 * (gamma + 1.0) * m2 / ((gamma - 1.0) * m2 + 2.0)
    p2 = p1 * (1.0 + 2.0 * gamma / (gamma + 1.0) * (m2 - 1.0))
    s = mach * np.sqrt(gamma * p1 / rho1)
    return rho2, s * (1.0 - rho1 / rho2), p2, s


def _interface_noise(seed, theta, phi, modes=4):
    """Seeded low-mode angular perturbation in [-1, 1] (sum of products of
    cos(nθ) and cos(mφ + φ_nm), n ≤ modes, m ≤ n, normalised)."""
    rng = np.random.default_rng(seed)
    xi = np.zeros_like(theta)
    norm = 0.0
    for n in range(1, modes + 1):
        for m in range(0, n + 1):
            a, ph = rng.uniform(-1.0, 1.0), rng.uniform(0.0, 2 * np.pi)
            xi = xi + a * np.cos(n * theta) * np.cos(m * phi + ph)
            norm += abs(a)
    return xi / norm


def shock_bubble(dim=3, base=8, b=16, levels=3, eps=1e-3, regrid_every=4, seed=SEED, x_shock=0.2, radius=0.15,
                 rho_bubble=0.138, mach=2.0, gamma=1.4, ghosts=5):
    """Mach-2 planar shock (moving +x) hitting a light bubble in pressure
    equilibrium on [0,1]^dim. Returns (sys, cfg, lo, hi, bc, init) where
    init(x[n,3]) -> primitive w[n,5]. Inflow (x low) is Dirichlet at the
    post-shock state, all other sides outflow."""
    from .physics import Bc, Euler, Nasg
    sys_ = Euler(Nasg.ideal(gamma))
    rho2, u2, p2, _ = rankine_hugoniot(mach, gamma)
    cfg = dict(b=b, levels=levels, eps=eps, regrid_every=regrid_every,
               base_blocks=[base] * dim + [0] * (3 - dim), ghosts=ghosts)
    lo = (0.0, 0.0, 0.0)
    hi = (1.0, 1.0, 1.0)
    centre = np.array([0.5, 0.5, 0.5])

    def init(x):
        rel = x - centre
        if dim == 2:
            rel[:, 2] = 0.0
        r = np.sqrt((rel * rel).sum(axis=1))
        theta = np.arccos(np.clip(np.where(r > 0, rel[:, 2] / np.where(r > 0, r, 1), 0.0), -1, 1))
        phi = np.arctan2(rel[:, 1], rel[:, 0])
        rb = radius * (1.0 + 0.005 * _interface_noise(seed, theta, phi))
        w = np.zeros((x.shape[0], 5))
        w[:, 0] = np.where(r < rb, rho_bubble, 1.0)
        w[:, 4] = 1.0
        post = x[:, 0] < x_shock
        w[post, 0] = rho2
        w[post, 1] = u2
        w[post, 4] = p2
        return w

    far = sys_.to_cons(np.array([rho2, u2, 0.0, 0.0, p2]))
    bc = [[Bc.dirichlet(far), Bc.Outflow], [Bc.Outflow, Bc.Outflow], [Bc.Outflow, Bc.Outflow]]
    return sys_, cfg, lo, hi, bc, init


def amr_explosion(dim=2, base=4, b=16, levels=3, eps=1e-3, regrid_every=4, radius=0.3, seed=SEED, noise=0.0):
    """Circular/spherical explosion on the block-AMR grid (outflow sides)."""
    from .physics import Bc, Euler, Nasg
    sys_ = Euler(Nasg.ideal(1.4))
    cfg = dict(b=b, levels=levels, eps=eps, regrid_every=regrid_every,
               base_blocks=[base] * dim + [0] * (3 - dim), ghosts=5)

    def init(x):
        rel = x - 0.5
        if dim == 2:
            rel[:, 2] = 0.0
        r = np.sqrt((rel * rel).sum(axis=1))
        w = np.zeros((x.shape[0], 5))
        w[:, 0] = np.where(r < radius, 1.0, 0.125)
        w[:, 4] = np.where(r < radius, 1.0, 0.1)
        if noise:
            key = np.floor(x * 1e6).astype(np.int64)
            idx = (key[:, 0] * 73856093 ^ key[:, 1] * 19349663 ^ key[:, 2] * 83492791).astype(np.uint64)
            w[:, 0] *= 1.0 + noise * uniform_pm1(seed, idx)
        return w

    bc = [[Bc.Outflow, Bc.Outflow] for _ in range(3)]
    return sys_, cfg, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), bc, init


# ---------------------------------------------------------------- batched 1-D Riemann problems
def riemann_batch(ninst=4096, nmin=64, nmax=2048, seed=SEED, gamma=1.4, x0=0.5):
    """Independent 1-D Riemann problems on [0,1]: cells log-uniform in
    [nmin, nmax], left/right states ρ ∈ U[0.1,2], u ∈ U[−1,1], p ∈ U[0.1,2],
    interface at x0. Returns (sys, n, dx, u, states) with u the concatenated
    interior conserved data and states[i] = (ρL, uL, pL, ρR, uR, pR)."""
    from .physics import Euler, Nasg
    sys_ = Euler(Nasg.ideal(gamma))
    rng = np.random.default_rng(seed)
    n = np.floor(np.exp(rng.uniform(np.log(nmin), np.log(nmax + 1), ninst))).astype(np.int64).clip(nmin, nmax)
    st = np.stack([rng.uniform(0.1, 2.0, ninst), rng.uniform(-1.0, 1.0, ninst), rng.uniform(0.1, 2.0, ninst),
                   rng.uniform(0.1, 2.0, ninst), rng.uniform(-1.0, 1.0, ninst), rng.uniform(0.1, 2.0, ninst)], axis=1)
    parts = []
    dx = 1.0 / n.astype(np.float64)
    for i in range(ninst):
        x = (np.arange(n[i]) + 0.5) * dx[i]  # cell centres as the device forms them, (c + ½)·dx
        left = x < x0
        w = np.zeros((n[i], 5))
        w[:, 0] = np.where(left, st[i, 0], st[i, 3])
        w[:, 1] = np.where(left, st[i, 1], st[i, 4])
        w[:, 4] = np.where(left, st[i, 2], st[i, 5])
        parts.append(sys_.to_cons(w))
    return sys_, n, dx, np.concatenate(parts), st


# ---------------------------------------------------------------- five-equation system
def two_phase_shock_bubble(n=128, mach=2.0, radius=0.15, eps=1e-8, seed=SEED, ng=6):
    """Two-phase shock–bubble on [0,1]^3 with n^3 cells for the five-equation
    system: phase 1 a light gas (γ 1.67, ρ 0.138) filling a sphere of radius
    0.15 about (0.5, 0.5, 0.5) (radius perturbed by ±0.5 % of a seeded
    low-mode harmonic sum), phase 2 air (γ 1.4, ρ 1, p 1) elsewhere, with
    volume fraction 1 − eps / eps; a Mach-2 shock in air at x < 0.2 moving +x
    (Rankine–Hugoniot post-shock state). Outflow boundaries.
    Returns (FiveEq, mesh, u_padded float64[len, 7], bc)."""
    from .five import FiveEq, five_initial_state
    sys = FiveEq((Nasg(1.67), Nasg(1.4)), kapila=True)
    mesh = Mesh.new((n, n, n), (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), ng=ng)
    x = mesh.centres()
    r = np.sqrt((x[0] - 0.5) ** 2 + (x[1] - 0.5) ** 2 + (x[2] - 0.5) ** 2)
    th = np.arccos(np.clip((x[2] - 0.5) / np.maximum(r, 1e-300), -1.0, 1.0))
    ph = np.arctan2(x[1] - 0.5, x[0] - 0.5)
    inside = r < radius * (1.0 + 0.005 * _interface_noise(seed, th, ph))
    rho2, u2, p2, _ = rankine_hugoniot(mach)
    post = x[0] < 0.2
    a = np.where(inside, 1.0 - eps, eps)
    w = np.zeros((n, n, n, 7))
    w[..., 0] = a * 0.138
    w[..., 1] = (1.0 - a) * np.where(post, rho2, 1.0)
    w[..., 2] = np.where(post, u2, 0.0)
    w[..., 5] = np.where(post, p2, 1.0)
    w[..., 6] = a
    bc = [[Bc.Outflow, Bc.Outflow] for _ in range(3)]
    return sys, mesh, five_initial_state(sys, mesh, w), bc


def two_phase_amr_bubble(dim=3, base=4, b=16, levels=3, eps=1e-3, regrid_every=4, seed=SEED, x_shock=0.2,
                         radius=0.15, mach=2.0, alpha_eps=1e-8, ghosts=5):
    """The two-phase shock–bubble of two_phase_shock_bubble on the block-AMR
    grid (five-equation system): a sphere (circle in 2-D) of light gas
    (γ 1.67, ρ 0.138, radius 0.15 ± 0.5 % seeded perturbation) in air (γ 1.4,
    ρ 1, p 1), volume fraction 1 − alpha_eps inside / alpha_eps outside, a
    Mach-2 shock in air at x < x_shock moving +x; inflow (x low) Dirichlet at
    the post-shock state, all other sides outflow. Returns (sys, cfg, lo, hi,
    bc, init) with init(x[n,3]) -> primitive w[n,7] = (α1ρ1, α2ρ2, u, v, w,
    p, α1)."""
    from .five import FiveEq
    sys_ = FiveEq((Nasg(1.67), Nasg(1.4)), kapila=True)
    rho2, u2, p2, _ = rankine_hugoniot(mach)
    cfg = dict(b=b, levels=levels, eps=eps, regrid_every=regrid_every,
               base_blocks=[base] * dim + [0] * (3 - dim), ghosts=ghosts)
    centre = np.array([0.5, 0.5, 0.5])

    def init(x):
        rel = x - centre
        if dim == 2:
            rel[:, 2] = 0.0
        r = np.sqrt((rel * rel).sum(axis=1))
        theta = np.arccos(np.clip(np.where(r > 0, rel[:, 2] / np.where(r > 0, r, 1), 0.0), -1, 1))
        phi = np.arctan2(rel[:, 1], rel[:, 0])
        inside = r < radius * (1.0 + 0.005 * _interface_noise(seed, theta, phi))
        post = x[:, 0] < x_shock
        a = np.where(inside, 1.0 - alpha_eps, alpha_eps)
        w = np.zeros((x.shape[0], 7))
        w[:, 0] = a * 0.138
        w[:, 1] = (1.0 - a) * np.where(post, rho2, 1.0)
        w[:, 2] = np.where(post, u2, 0.0)
        w[:, 5] = np.where(post, p2, 1.0)
        w[:, 6] = a
        return w

    far_w = np.array([alpha_eps * 0.138, (1.0 - alpha_eps) * rho2, u2, 0.0, 0.0, p2, alpha_eps])
    far = sys_.to_cons(far_w)
    bc = [[Bc.dirichlet(far), Bc.Outflow], [Bc.Outflow, Bc.Outflow], [Bc.Outflow, Bc.Outflow]]
    return sys_, cfg, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), bc, init
