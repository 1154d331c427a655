"""Host-side mirror of the reference solver types.

Names and meanings follow fluid/crates/compressible/src: ``Nasg``
(eos.rs:12-35), ``Euler`` (system.rs:190-217), ``Mesh`` (solver.rs:22-86),
``Bc`` (solver.rs:8-20), ``FluxMode`` (scheme.rs:39-47). The state arrays are
numpy ``float64[len, 5]`` in the reference's ghost-padded AoS layout.
"""
from dataclasses import dataclass, field
import numpy as np


@dataclass(frozen=True)
class Nasg:
    gamma: float
    p_inf: float = 0.0
    b: float = 0.0
    q: float = 0.0
    cv: float = 1.0

    @staticmethod
    def ideal(gamma):
        return Nasg(gamma)

    @staticmethod
    def stiffened(gamma, p_inf):
        return Nasg(gamma, p_inf)

    # eos.rs:44-54 (vectorised, same operation order)
    def rho_e(self, rho, p):
        v = 1.0 / rho
        return rho * ((p + self.gamma * self.p_inf) * (v - self.b) / (self.gamma - 1.0) + self.q)

    def pressure(self, rho, e):
        v = 1.0 / rho
        return (self.gamma - 1.0) * (e - self.q) / (v - self.b) - self.gamma * self.p_inf


@dataclass(frozen=True)
class Euler:
    """Single-material Euler equations, w = (ρ,u,v,w,p), u = (ρ,ρu,ρv,ρw,E)."""
    eos: Nasg

    def to_cons(self, w):
        w = np.asarray(w, dtype=np.float64)
        rho = w[..., 0]
        ke = 0.5 * rho * (w[..., 1] * w[..., 1] + w[..., 2] * w[..., 2] + w[..., 3] * w[..., 3])
        out = np.empty_like(w)
        out[..., 0] = rho
        out[..., 1] = rho * w[..., 1]
        out[..., 2] = rho * w[..., 2]
        out[..., 3] = rho * w[..., 3]
        out[..., 4] = self.eos.rho_e(rho, w[..., 4]) + ke
        return out

    def to_prim(self, u):
        u = np.asarray(u, dtype=np.float64)
        rho = u[..., 0]
        vx, vy, vz = u[..., 1] / rho, u[..., 2] / rho, u[..., 3] / rho
        e = u[..., 4] / rho - 0.5 * (vx * vx + vy * vy + vz * vz)
        return np.stack([rho, vx, vy, vz, self.eos.pressure(rho, e)], axis=-1)


class FluxMode:
    Hybrid = 0
    Weno = 1
    Central = 2


class Precision:
    F64 = 0
    Mixed = 1
    F64Fast = 2  # fast FP64 form (uniform grids): within 1e-12 relative L1 of F64 instead of bitwise


@dataclass(frozen=True)
class Bc:
    kind: int
    state: tuple = (0.0, 0.0, 0.0, 0.0, 0.0)

    PERIODIC = 0
    OUTFLOW = 1
    REFLECT = 2
    DIRICHLET = 3
    CHARACTERISTIC = 4

    @staticmethod
    def dirichlet(u):
        return Bc(Bc.DIRICHLET, tuple(float(x) for x in u))

    @staticmethod
    def characteristic(u):
        return Bc(Bc.CHARACTERISTIC, tuple(float(x) for x in u))


Bc.Periodic = Bc(Bc.PERIODIC)
Bc.Outflow = Bc(Bc.OUTFLOW)
Bc.Reflect = Bc(Bc.REFLECT)


@dataclass
class Mesh:
    """Uniform mesh: n cells per axis (1 = inactive), lower corner, cell size, ghosts."""
    n: tuple
    lo: tuple
    dx: tuple
    ng: int = 6

    @staticmethod
    def new(n, lo, hi, ng=6):
        n = tuple(int(x) for x in n)
        dx = tuple((hi[d] - lo[d]) / n[d] for d in range(3))
        return Mesh(n, tuple(float(x) for x in lo), dx, ng)

    def with_ghosts(self, ng):
        return Mesh(self.n, self.lo, self.dx, ng)

    def active(self, d):
        return self.n[d] > 1

    def m(self, d):
        return self.n[d] + 2 * self.ng if self.active(d) else 1

    def g(self, d):
        return self.ng if self.active(d) else 0

    def idx(self, i, j, k):
        return (i * self.m(1) + j) * self.m(2) + k

    def len(self):
        return self.m(0) * self.m(1) * self.m(2)

    def cells(self):
        return self.n[0] * self.n[1] * self.n[2]

    def ndim(self):
        return sum(1 for d in range(3) if self.active(d))

    def padded_shape(self):
        return (self.m(0), self.m(1), self.m(2))

    def interior(self, a):
        """View of the interior cells of a padded array of shape (len, ...)."""
        a = a.reshape(self.padded_shape() + a.shape[1:])
        s = tuple(slice(self.g(d), self.g(d) + self.n[d]) for d in range(3))
        return a[s]

    def centres(self):
        """Cell-centre coordinates of the interior cells, each of shape n."""
        axes = [self.lo[d] + (np.arange(self.n[d], dtype=np.float64) + 0.5) * self.dx[d] for d in range(3)]
        return np.meshgrid(*axes, indexing="ij")


def initial_state(sys, mesh, w_interior):
    """Padded AoS conserved state from interior primitives (Solver::new,
    solver.rs:199-208); ghost cells are zero until the first ghost fill."""
    u = np.zeros((mesh.len(), 5), dtype=np.float64)
    mesh.interior(u)[...] = sys.to_cons(w_interior)
    return u
