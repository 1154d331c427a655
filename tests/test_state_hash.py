"""The state fingerprint (emg_state_hash), host code checked on the CPU
against a plain-loop restatement of the reference's hash
(fluid/crates/compressible/examples/cpu_validate.rs:7-22)."""
import numpy as np
import pytest

from emergence_b200 import state_hash
from emergence_b200.physics import Mesh

MASK = (1 << 64) - 1


def reference_hash(mesh, u):
    h = 0xCBF29CE484222325
    bits = np.ascontiguousarray(u).view(np.uint64)
    for i in range(mesh.n[0]):
        for j in range(mesh.n[1]):
            for k in range(mesh.n[2]):
                c = mesh.idx(i + mesh.g(0), j + mesh.g(1), k + mesh.g(2))
                for q in range(5):
                    h = ((h ^ int(bits[c, q])) * 0x100000001B3) & MASK
    return h


@pytest.mark.parametrize("n", [(7, 1, 1), (5, 4, 1), (3, 4, 5)])
def test_matches_the_reference_hash(n):
    mesh = Mesh.new(n, (0, 0, 0), (1, 1, 1), ng=6)
    u = np.random.default_rng(3).normal(size=(mesh.len(), 5))
    assert state_hash(mesh, u) == reference_hash(mesh, u)


def test_sees_every_interior_bit_and_no_ghost():
    mesh = Mesh.new((4, 3, 2), (0, 0, 0), (1, 1, 1), ng=5)
    u = np.random.default_rng(4).normal(size=(mesh.len(), 5))
    h0 = state_hash(mesh, u)
    ghost = mesh.idx(0, 0, 0)
    v = u.copy()
    v[ghost] = np.nan
    assert state_hash(mesh, v) == h0
    c = mesh.idx(mesh.g(0) + 1, mesh.g(1) + 2, mesh.g(2))
    w = u.copy()
    w[c, 3] = np.nextafter(w[c, 3], np.inf)  # one ulp
    assert state_hash(mesh, w) != h0


def test_oracle_and_library_hashes_agree():
    from oracle import pyoracle as O
    mesh = Mesh.new((6, 5, 4), (0, 0, 0), (1, 1, 1), ng=6)
    u = np.random.default_rng(5).normal(size=(mesh.len(), 5))
    assert O.state_hash(mesh, u) == state_hash(mesh, u) == reference_hash(mesh, u)
