"""Batched independent 1-D Riemann problems on the device vs per-instance
oracle runs (needs a B200)."""
import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.physics import Bc, FluxMode, Mesh, Precision, initial_state
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu


def oracle_instance(sys_, n, u0, t_end, mode=FluxMode.Weno):
    mesh = Mesh.new((int(n), 1, 1), (0, 0, 0), (1, 1, 1), ng=6)
    u = np.zeros((mesh.len(), 5))
    u[mesh.g(0):mesh.g(0) + n] = u0
    bc = [[Bc.Outflow, Bc.Outflow], [Bc.Periodic] * 2, [Bc.Periodic] * 2]
    o = O.OracleSolver(sys_, mesh, u, bc=bc, mode=mode, cfl=0.5)
    steps = o.run_to(t_end)
    return o.download()[mesh.g(0):mesh.g(0) + n], steps, o.t


@pytest.mark.parametrize("mode", [FluxMode.Weno, FluxMode.Hybrid])
def test_batched_lines_match_per_instance_oracle_runs(mode):
    from emergence_b200 import GpuBatch1D
    sys_, n, dx, u, st = W.riemann_batch(ninst=48, nmin=64, nmax=200, seed=5)
    g = GpuBatch1D(sys_, n, dx, u, mode=mode)
    g.run_to(0.15)
    t, steps = g.status()
    out = g.split(g.download())
    ins = g.split(u)
    for i in range(len(n)):
        ref, osteps, ot = oracle_instance(sys_, n[i], ins[i], 0.15, mode)
        assert int(steps[i]) == osteps and t[i] == ot, i
        if mode == FluxMode.Weno:
            assert np.array_equal(out[i], ref), (i, float(np.max(np.abs(out[i] - ref))))
        else:
            # the hybrid sensor takes logarithms, whose last ulp may differ
            # between the device and the host C library: 1e-12 L1 gate
            err = np.abs(out[i] - ref).sum(axis=0) / np.abs(ref).sum(axis=0).clip(1e-300)
            assert np.all(err <= 1e-12), (i, err)


def test_batched_mixed_precision_error():
    from emergence_b200 import GpuBatch1D
    sys_, n, dx, u, st = W.riemann_batch(ninst=32, nmin=64, nmax=300, seed=9)
    g = GpuBatch1D(sys_, n, dx, u, precision=Precision.Mixed)
    g.run_to(0.15)
    out = g.split(g.download())
    ins = g.split(u)
    live = [0, 1, 4]  # ρ, ρu, E; the transverse momenta of a 1-D line stay exactly zero
    num = np.zeros(len(live))
    den = np.zeros(len(live))
    for i in range(len(n)):
        ref, _, _ = oracle_instance(sys_, n[i], ins[i], 0.15)
        assert not np.any(out[i][:, 2:4]), i
        num += np.abs(out[i] - ref)[:, live].sum(axis=0)
        den += np.abs(ref)[:, live].sum(axis=0)
    err = num / den
    print("batched mixed rel L1 (rho, rho u, E)", err)
    assert np.all(err <= 1e-5)


def test_segments_split_long_instances():
    """Instances longer than one 64-cell segment and shorter ones in one launch."""
    from emergence_b200 import GpuBatch1D
    sys_, n, dx, u, st = W.riemann_batch(ninst=6, nmin=300, nmax=700, seed=2)
    n = np.concatenate([n, [7, 64, 65]])
    extra = []
    for m in (7, 64, 65):
        x = (np.arange(m) + 0.5) / m
        w = np.zeros((m, 5))
        w[:, 0] = np.where(x < 0.5, 1.0, 0.125)
        w[:, 4] = np.where(x < 0.5, 1.0, 0.1)
        extra.append(sys_.to_cons(w))
    u = np.concatenate([u] + extra)
    g = GpuBatch1D(sys_, n, 1.0 / n, u)
    g.run_to(0.1)
    out = g.split(g.download())
    ins = g.split(u)
    for i in range(len(n)):
        ref, _, _ = oracle_instance(sys_, n[i], ins[i], 0.1)
        assert np.array_equal(out[i], ref), i
