"""The allocation-free step (emg_uniform_step_noalloc) against the solver
that owns its buffers (needs a B200).

Some callers cannot call cudaMalloc — code running where a framework or a
pooling allocator owns all device memory, or inside phases that must not
allocate — so this entry point takes caller-owned input and output states and
works in a fixed static scratch area of the library. This test allocates the
caller's buffers itself (through torch, standing in for such a framework),
calls the entry point twice in a row through the C ABI, and checks each
result against the allocating solver's step with the same dt.
"""
import ctypes as C

import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.physics import FluxMode, Precision

pytestmark = pytest.mark.gpu

F64_TOL = 1e-12  # relative L1 per conserved field, as the other parity tests


def _explosion_3d():
    return W.explosion((40, 36, 30), 0.3)


def _short_reflecting_2d():
    """2-D explosion with a reflecting axis of 4 cells, shorter than the 6
    ghost layers: its ghosts are deep reflected images."""
    from emergence_b200.physics import Bc
    sys_, mesh, u, _ = W.explosion((48, 4, 1), 0.3)
    bc = [[Bc.Outflow, Bc.Outflow], [Bc.Reflect, Bc.Reflect], [Bc.Outflow, Bc.Outflow]]
    return sys_, mesh, u, bc


CASES = {"explosion_3d": _explosion_3d, "short_reflecting_2d": _short_reflecting_2d}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("mode", [FluxMode.Weno, FluxMode.Hybrid, FluxMode.Central])
@pytest.mark.parametrize("precision", [Precision.F64, Precision.Mixed])
def test_noalloc_step_matches_the_allocating_solver_twice(precision, mode, case):
    import torch
    from emergence_b200 import GpuSolver
    from emergence_b200._abi import EmgOpts, check, lib
    from emergence_b200.solver import _c_bcs, _c_eos, _c_mesh

    sys_, mesh, u, bc = CASES[case]()
    assert mesh.len() <= 131072  # within EMG_NOALLOC_MAX_CELLS
    g = GpuSolver(sys_, mesh, u, bc=bc, mode=mode, precision=precision)
    m, e, b = _c_mesh(mesh), _c_eos(sys_.eos), _c_bcs(bc)
    o = EmgOpts(0.5, 1e-3, mode, 1, precision, 0)
    stream = torch.cuda.current_stream()
    cur = torch.tensor(np.ascontiguousarray(u.T), dtype=torch.float64, device="cuda")  # SoA [5][ncell]
    for call in range(2):
        dt = g.dt_cfl()
        g.step(dt)
        ref = g.download()
        out = torch.empty_like(cur)
        check(lib().emg_uniform_step_noalloc(C.byref(m), C.byref(e), b, C.byref(o), C.c_void_p(cur.data_ptr()),
                                             C.c_void_p(out.data_ptr()), dt, C.c_void_p(stream.cuda_stream)))
        stream.synchronize()
        got = out.cpu().numpy().T.copy()
        gi = mesh.interior(got).reshape(-1, 5)
        ri = mesh.interior(ref).reshape(-1, 5)
        den = np.abs(ri).sum(axis=0)
        err = np.abs(gi - ri).sum(axis=0) / np.where(den > 0, den, 1.0)
        assert np.all(err <= F64_TOL), (call, err)
        assert np.array_equal(got, ref), call  # same kernels, same order: bit for bit, ghosts included
        cur = out
    g.close()


def test_noalloc_rejects_grids_above_the_scratch_limit():
    import torch
    from emergence_b200._abi import EmgOpts, lib
    from emergence_b200.solver import _c_bcs, _c_eos, _c_mesh

    sys_, mesh, u, bc = W.explosion((64, 64, 40), 0.3)  # 76*76*52 padded cells > 131072
    m, e, b = _c_mesh(mesh), _c_eos(sys_.eos), _c_bcs(bc)
    o = EmgOpts(0.5, 1e-3, FluxMode.Weno, 1, Precision.F64, 0)
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib().emg_uniform_step_noalloc(C.byref(m), C.byref(e), b, C.byref(o), C.c_void_p(x.data_ptr()),
                                        C.c_void_p(x.data_ptr() + 8), 1e-3, None)
    assert rc == 1 and b"EMG_NOALLOC_MAX_CELLS" in lib().emg_last_error()
