"""Parity cases run against the bounds-check build (libemergence_b200_bc.so,
loaded when EMG_BOUNDS_CHECK=1): every global index of the sweeps, the
uniform ghost fill and the AMR pool accesses is checked on the device, and
any index out of range would come back as EMG_ERR_BOUNDS (an EmgError here).
Run as a script by tests/test_gpu_bounds_check.py in a child process; prints
one line per case and exits non-zero on the first failure."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from emergence_b200 import GpuAmr, GpuBatch1D, GpuSolver, _abi, workloads as W  # noqa: E402
from emergence_b200.physics import Bc, FluxMode, Precision  # noqa: E402
from oracle import pyoracle as O  # noqa: E402


def uniform_cases():
    out = []
    refl = [[Bc.Reflect, Bc.Reflect]] * 3
    for shape, bc in (((40, 1, 1), None), ((24, 20, 1), None), ((12, 10, 14), None), ((8, 3, 1), refl),
                      ((2, 3, 4), [[Bc.Periodic, Bc.Periodic]] * 3)):
        for mode in (FluxMode.Weno, FluxMode.Hybrid, FluxMode.Central):
            out.append((shape, bc, mode))
    return out


def run_uniform(shape, bc, mode):
    sys_, mesh, u, bce = W.explosion(shape, 0.3)
    bc = bce if bc is None else bc
    o = O.OracleSolver(sys_, mesh, u, bc=bc, mode=mode)
    g = GpuSolver(sys_, mesh, u, bc=bc, mode=mode)
    gm = GpuSolver(sys_, mesh, u, bc=bc, mode=mode, precision=Precision.Mixed)
    for _ in range(3):
        dt = o.dt_cfl()
        o.step(dt)
        g.step(dt)
        gm.step(dt)
    ug, uo = mesh.interior(g.download()), mesh.interior(o.download())
    err = np.abs(ug - uo).reshape(-1, 5).sum(axis=0) / np.maximum(np.abs(uo).reshape(-1, 5).sum(axis=0), 1e-300)
    assert np.all(err <= 1e-12), (shape, mode, err)
    g.advance(2)
    gm.advance(2)
    g.close()
    gm.close()
    return float(err.max())


def run_amr():
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g = GpuAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    for _ in range(5):  # a regrid after step 4
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    st = o.structure()
    assert np.array_equal(st, g.structure())
    leaves = st[:, 4] == 1
    ug, uo = g.download()[leaves], o.download()[leaves]
    err = np.abs(ug - uo).reshape(-1, 5).sum(axis=0) / np.maximum(np.abs(uo).reshape(-1, 5).sum(axis=0), 1e-300)
    assert np.all(err <= 1e-12), err
    g.close()
    return float(err.max())


def run_amr_subcycled():
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno, subcycle=True)
    g = GpuAmr(s, cfg, lo, hi, bc, mode=FluxMode.Weno, blocks=(o.structure(), o.download()), subcycle=True)
    for _ in range(3):  # a regrid after each subcycled step
        dt = o.dt_cfl_subcycled()
        g.step_subcycled(dt)
        o.step_subcycled(dt)
    st = o.structure()
    assert np.array_equal(st, g.structure())
    ug, uo = g.download(), o.download()
    err = np.abs(ug - uo).reshape(-1, 5).sum(axis=0) / np.maximum(np.abs(uo).reshape(-1, 5).sum(axis=0), 1e-300)
    assert np.all(err <= 1e-12), err
    g.close()
    return float(err.max())


def run_amr_five():
    s, cfg, lo, hi, bc, init = W.two_phase_amr_bubble(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g = GpuAmr(s, cfg, lo, hi, bc, mode=FluxMode.Weno, blocks=(o.structure(), o.download()))
    for _ in range(5):  # a regrid after step 4
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    assert np.array_equal(o.structure(), g.structure())
    ug, uo = g.download(), o.download()
    err = np.abs(ug - uo).reshape(-1, 7).sum(axis=0) / np.maximum(np.abs(uo).reshape(-1, 7).sum(axis=0), 1e-300)
    assert np.all(err <= 1e-12), err
    g.close()
    return float(err.max())


def run_five():
    from emergence_b200 import GpuFiveSolver
    sys5, mesh, u, bc = W.two_phase_shock_bubble(n=24)
    g = GpuFiveSolver(sys5, mesh, u, bc=bc)
    for _ in range(3):
        g.step(g.dt_cfl())
    assert np.all(np.isfinite(g.download()))
    g.close()
    return 0.0


def run_batch():
    sys_, n, dx, u, st = W.riemann_batch(ninst=24, nmin=64, nmax=200, seed=5)
    for prec in (Precision.F64, Precision.Mixed):
        g = GpuBatch1D(sys_, n, dx, u, precision=prec)
        g.run_to(0.05)
        g.close()
    return 0.0


def main():
    assert os.environ.get("EMG_BOUNDS_CHECK") == "1" and _abi.lib_path().endswith("_bc.so")
    for shape, bc, mode in uniform_cases():
        print("uniform", shape, "reflect" if bc else "default", mode, "rel L1", run_uniform(shape, bc, mode), flush=True)
    print("amr 2-D shock-bubble with a regrid: rel L1", run_amr(), flush=True)
    print("subcycled amr 2-D shock-bubble with regrids: rel L1", run_amr_subcycled(), flush=True)
    run_five()
    print("five-equation 3-D shock-bubble 24^3: ok", flush=True)
    print("five-equation AMR 2-D shock-bubble with a regrid: rel L1", run_amr_five(), flush=True)
    run_batch()
    print("batched lines: ok", flush=True)
    print("BOUNDS_CHECK_OK")


if __name__ == "__main__":
    main()
