"""The 3-D explosion at its full size, 256³ (16.8 M cells), against the oracle
(needs a B200; the oracle's 10 steps take about a minute on 16 host threads).

The other parity tests run small grids, where every launch shape differs from
the one the benchmark uses (whole 256-cell pencils, 32 pencils per CTA,
2048 CTAs per sweep). Here both forms run the benchmark's grid for 10 steps
from the same initial state with the oracle's time steps:

* plain FP64 form: bit-exact with the oracle (and so within the parity
  tolerance of 1e-12 relative L1 per conserved field), counters equal;
* mixed form (FP32 WENO-Z and wave-speed bounds, FP64 state): relative L1
  per conserved field within 1e-6 of the oracle, the stated error bound of
  that form; L∞ is reported.
* fast FP64 form (FMA contraction, Newton-refined reciprocals): relative L1
  within 1e-12.
"""
import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.physics import FluxMode, Precision
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

N, STEPS = 256, 10
F64_TOL = 1e-12
MIXED_TOL = 1e-6


def rel_l1(a, b, mesh):
    ai, bi = mesh.interior(a).reshape(-1, 5), mesh.interior(b).reshape(-1, 5)
    num = np.abs(ai - bi).sum(axis=0)
    den = np.abs(bi).sum(axis=0)
    # the momenta of the explosion sum to about zero in |.|-weight only through
    # noise; measure them against the density's L1 norm when they are tiny
    return num / np.maximum(den, 1e-3 * den[0])


@pytest.fixture(scope="module")
def oracle_run():
    sys_, mesh, u, bc = W.explosion((N, N, N), 0.3)
    o = O.OracleSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5)
    dts = []
    for _ in range(STEPS):
        dts.append(o.dt_cfl())
        o.step(dts[-1])
    out = (sys_, mesh, u, bc, dts, o.download(), o.counters())
    o.close()
    return out


def run_gpu(oracle_run, precision):
    from emergence_b200 import GpuSolver
    sys_, mesh, u, bc, dts, _, _ = oracle_run
    g = GpuSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5, precision=precision)
    for dt in dts:
        g.step(dt)
    out = g.download(), g.counters()
    g.close()
    return out


def test_fp64_form_is_bit_exact_with_the_oracle_at_256_cubed(oracle_run):
    _, mesh, _, _, _, uo, co = oracle_run
    ug, cg = run_gpu(oracle_run, Precision.F64)
    err = rel_l1(ug, uo, mesh)
    print("256^3 FP64 rel L1 vs oracle", err)
    assert np.all(err <= F64_TOL), err
    assert np.array_equal(mesh.interior(ug), mesh.interior(uo))
    assert cg == co


def test_mixed_form_error_against_the_oracle_at_256_cubed(oracle_run):
    mesh, uo = oracle_run[1], oracle_run[5]
    um, _ = run_gpu(oracle_run, Precision.Mixed)
    err = rel_l1(um, uo, mesh)
    linf = np.abs(mesh.interior(um) - mesh.interior(uo)).reshape(-1, 5).max(axis=0)
    print("256^3 mixed rel L1 vs oracle", err, "Linf", linf)
    assert np.all(err <= MIXED_TOL), err


def test_fast_fp64_form_error_against_the_oracle_at_256_cubed(oracle_run):
    """Fast FP64 form (FMA contraction, Newton-refined reciprocals): within the
    plain form's 1e-12 relative L1 per conserved field."""
    mesh, uo = oracle_run[1], oracle_run[5]
    uf, _ = run_gpu(oracle_run, Precision.F64Fast)
    err = rel_l1(uf, uo, mesh)
    linf = np.abs(mesh.interior(uf) - mesh.interior(uo)).reshape(-1, 5).max(axis=0)
    print("256^3 fast FP64 rel L1 vs oracle", err, "Linf", linf)
    assert np.all(err <= F64_TOL), err
