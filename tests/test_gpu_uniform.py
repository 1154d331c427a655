"""Parity of the CUDA uniform-grid solver with the CPU oracle (needs a B200).

Every test drives the CUDA library through its C ABI (GpuSolver) and the
oracle through the same calls, on bit-identical inputs. The plain FP64 form
is held to the parity tolerance of 1e-12 relative L1 per conserved field
(it is built without FMA contraction and is expected to be bit-exact); the
mixed form to its stated error bound.
"""
import math

import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.physics import Bc, Euler, FluxMode, Mesh, Nasg, Precision, initial_state
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

GAS = Nasg.ideal(1.4)
SYS = Euler(GAS)
F64_TOL = 1e-12  # relative L1 per conserved field (plain FP64 form)


def gpu_solver(*a, **k):
    from emergence_b200 import GpuSolver
    return GpuSolver(*a, **k)


def rel_l1(a, b, mesh):
    ai, bi = mesh.interior(a).reshape(-1, 5), mesh.interior(b).reshape(-1, 5)
    num = np.abs(ai - bi).sum(axis=0)
    den = np.abs(bi).sum(axis=0)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def linf(a, b, mesh):
    return np.abs(mesh.interior(a) - mesh.interior(b)).reshape(-1, 5).max(axis=0)


def random_state(n, seed, ng=6, jump=True):
    """Smooth random Fourier modes (plus small white noise and, optionally, a
    planar jump) of ρ, u and p: finite under every boundary condition,
    including deep characteristic extrapolation."""
    rng = np.random.default_rng(seed)
    mesh = Mesh.new(n, (0, 0, 0), (1, 1, 1), ng=ng)
    x = mesh.centres()

    def field(scale):
        f = np.zeros(n)
        for _ in range(4):
            k = rng.integers(1, 3, size=3)
            ph = rng.random(3) * 2 * np.pi
            f += scale * rng.random() * np.sin(2 * np.pi * k[0] * x[0] + ph[0]) * np.cos(
                2 * np.pi * k[1] * x[1] + ph[1]) * np.cos(2 * np.pi * k[2] * x[2] + ph[2])
        return f + 0.01 * scale * (rng.random(n) - 0.5)

    w = np.zeros(tuple(n) + (5,))
    w[..., 0] = 1.0 + field(0.1)
    for d in range(3):
        w[..., 1 + d] = field(0.3) if n[d] > 1 else 0.0
    w[..., 4] = 1.0 + field(0.1)
    if jump:
        hot = x[0] + 0.7 * x[1] + 0.3 * x[2] < 0.8
        w[..., 0] = np.where(hot, 4.0 * w[..., 0], w[..., 0])
        w[..., 4] = np.where(hot, 10.0 * w[..., 4], w[..., 4])
    return mesh, initial_state(SYS, mesh, w)


FAR = tuple(SYS.to_cons(np.array([1.1, 0.1, -0.05, 0.02, 1.2])))
BC_SETS = {
    "outflow": [[Bc.Outflow, Bc.Outflow]] * 3,
    "periodic": [[Bc.Periodic, Bc.Periodic]] * 3,
    "reflect": [[Bc.Reflect, Bc.Reflect]] * 3,
    "mixed": [[Bc.Reflect, Bc.dirichlet(FAR)], [Bc.Outflow, Bc.characteristic(FAR)], [Bc.Periodic, Bc.Periodic]],
    "characteristic": [[Bc.characteristic(FAR), Bc.characteristic(FAR)]] * 3,
}
SHAPES = [(40, 1, 1), (1, 33, 1), (24, 20, 1), (1, 17, 19), (12, 10, 14)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("bcname", list(BC_SETS))
def test_one_step_matches_the_oracle_bitwise(shape, bcname):
    # a jump crossing a characteristic boundary is extrapolated linearly into
    # the ghost layers (C/boundary.rs:80-95) and can leave them inadmissible
    mesh, u = random_state(shape, seed=10 * SHAPES.index(shape) + list(BC_SETS).index(bcname),
                           jump=bcname not in ("mixed", "characteristic"))
    bc = BC_SETS[bcname]
    g = gpu_solver(SYS, mesh, u, bc=bc, mode=FluxMode.Weno)
    o = O.OracleSolver(SYS, mesh, u, bc=bc, mode=FluxMode.Weno)
    dt = o.dt_cfl()
    assert g.dt_cfl() == dt
    g.step(dt)
    o.step(dt)
    ug, uo = g.download(), o.download()
    assert np.all(rel_l1(ug, uo, mesh) <= F64_TOL)
    # interior and ghost layers (filled at stage 1) bit for bit, up to the sign of zero
    assert np.array_equal(ug, uo, equal_nan=True), float(np.nanmax(np.abs(ug - uo)))
    assert g.counters() == o.counters()
    assert g.t == o.t


@pytest.mark.parametrize("shape", [(2, 3, 4), (8, 2, 1), (3, 1, 1)])
@pytest.mark.parametrize("bcname", ["periodic", "reflect"])
def test_short_axes_use_deep_ghost_images(shape, bcname):
    mesh, u = random_state(shape, seed=7, ng=6, jump=False)
    bc = BC_SETS[bcname]
    g = gpu_solver(SYS, mesh, u, bc=bc, mode=FluxMode.Weno)
    o = O.OracleSolver(SYS, mesh, u, bc=bc, mode=FluxMode.Weno)
    for _ in range(2):
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    assert np.array_equal(g.download(), o.download())


@pytest.mark.parametrize("precision", [Precision.F64, Precision.Mixed])
@pytest.mark.parametrize("shape", [(40, 36, 30), (24, 22, 64)])
def test_tma_row_staging_gives_the_plain_loads_results(shape, precision, monkeypatch):
    """With EMG_TMA=1, 3-D WENO grids with ng and n2 even stage the sweeps'
    rows by TMA (EMG_FEATURE_TMA): bit for bit the oracle's results in the
    FP64 form, and the same bits as the per-thread loads (the default) in
    both forms."""
    sys, mesh, u, bc = W.explosion(shape, 0.3)
    monkeypatch.setenv("EMG_TMA", "1")
    g = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno, precision=precision)
    assert g.features() & 1
    monkeypatch.delenv("EMG_TMA")
    p = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno, precision=precision)
    assert not p.features() & 1
    o = O.OracleSolver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
    for _ in range(3):
        dt = o.dt_cfl()
        g.step(dt)
        p.step(dt)
        o.step(dt)
    assert g.advance(2) == 2 and p.advance(2) == 2
    for _ in range(2):
        o.step(o.dt_cfl())
    ug = g.download()
    assert np.array_equal(ug, p.download())
    if precision == Precision.F64:
        assert np.array_equal(mesh.interior(ug), mesh.interior(o.download()))
        assert g.counters() == o.counters()


def test_uniform_flow_is_preserved():
    w0 = np.array([1.0, 0.3, -0.2, 0.1, 1.0])
    mesh = Mesh.new((9, 7, 6), (0, 0, 0), (1, 1, 1), ng=6)
    u = initial_state(SYS, mesh, np.broadcast_to(w0, mesh.n + (5,)).copy())
    g = gpu_solver(SYS, mesh, u, bc=BC_SETS["periodic"], mode=FluxMode.Weno)
    g.step(1e-4)
    w = SYS.to_prim(mesh.interior(g.download()))
    assert np.all(np.abs(w - w0) < 1e-13)


def test_explosion_2d_256_to_t_0_2_matches_the_oracle():
    """The 2-D circular explosion 256², t_end = 0.2, CFL 0.5 (reference CPU-path case)."""
    sys, mesh, u, bc = W.explosion_2d(256)
    g = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5)
    o = O.OracleSolver(sys, mesh, u, bc=bc, mode=FluxMode.Weno, cfl=0.5)
    ng_steps = g.run_to(0.2)
    no_steps = o.run_to(0.2)
    assert ng_steps == no_steps
    assert g.t == o.t
    ug, uo = g.download(), o.download()
    err = rel_l1(ug, uo, mesh)
    print("explosion_2d rel L1 per field", err, "Linf", linf(ug, uo, mesh))
    assert np.all(err <= F64_TOL)
    assert np.array_equal(mesh.interior(ug), mesh.interior(uo))
    assert np.allclose(g.totals(), o.totals(), rtol=1e-13, atol=1e-15)
    assert g.counters() == o.counters()


def test_explosion_3d_short_run_matches_the_oracle():
    sys, mesh, u, bc = W.explosion((40, 36, 32), 0.3)
    g = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
    o = O.OracleSolver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
    assert g.advance(6) == 6
    o.advance(6)
    ug, uo = g.download(), o.download()
    assert np.all(rel_l1(ug, uo, mesh) <= F64_TOL)
    assert np.array_equal(mesh.interior(ug), mesh.interior(uo))
    assert g.t == o.t


def test_device_driven_steps_equal_host_driven_steps():
    sys, mesh, u, bc = W.explosion((48, 48, 1), 0.4)
    a = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
    b = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
    a.advance(5)
    for _ in range(5):
        b.step(b.dt_cfl())
    assert np.array_equal(a.download(), b.download())
    assert a.t == b.t


def test_runs_are_bitwise_deterministic():
    sys, mesh, u, bc = W.explosion((64, 64, 16), 0.3)
    r = []
    for _ in range(2):
        g = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
        g.advance(3)
        r.append(g.download())
    assert np.array_equal(r[0], r[1])


def test_mixed_precision_error_against_the_fp64_oracle():
    sys, mesh, u, bc = W.explosion((96, 96, 1), 0.4)
    g = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno, precision=Precision.Mixed)
    o = O.OracleSolver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
    for _ in range(20):
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    err = rel_l1(g.download(), o.download(), mesh)
    print("mixed rel L1 per field after 20 steps", err)
    # FP32 WENO-Z on deviations from FP64 characteristic values (scaled weights),
    # everything else FP64; bound 1e-6 relative L1
    assert np.all(err <= 1e-6), err
    assert g.counters()[2] == o.counters()[2] == 0  # no first-order fallbacks in either


def test_collapsed_time_step_is_reported_not_trapped():
    """A cell whose wave speed explodes drives dt below 1e-12·t_end: run_to
    returns EMG_ERR_DT_COLLAPSED (C/solver.rs:763) and the handle stays usable."""
    sys, mesh, u, bc = W.explosion((16, 16, 1), 0.4)
    bad = u.copy()
    bad[mesh.idx(mesh.g(0) + 5, mesh.g(1) + 7, 0), 4] = 1e300
    g = gpu_solver(sys, mesh, bad, bc=bc, mode=FluxMode.Weno)
    o = O.OracleSolver(sys, mesh, bad, bc=bc, mode=FluxMode.Weno)
    from emergence_b200 import EmgError
    with pytest.raises(EmgError) as e:
        g.run_to(0.1)
    assert e.value.code == 3
    with pytest.raises(RuntimeError):
        o.run_to(0.1)
    g.upload(u)
    assert g.dt_cfl() == O.OracleSolver(sys, mesh, u, bc=bc, mode=FluxMode.Weno).dt_cfl()


@pytest.mark.parametrize("poison", ["nan_density", "negative_density", "negative_pressure", "nan_ghost"])
def test_inadmissible_state_is_reported_by_the_cfl_reduction(poison):
    """A host-poisoned interior cell (NaN, ρ < 0, or an energy below the
    kinetic energy) is reported as EMG_ERR_INADMISSIBLE by dt_cfl and by
    advance before any step is taken, and by a host-given step whose result
    is still inadmissible; nothing traps and the handle stays usable. NaN in a ghost layer only is not an error: ghost
    layers are refilled before they are read (tests/cpu.rs:25-52)."""
    from emergence_b200 import EmgError
    sys, mesh, u, bc = W.explosion((16, 16, 1), 0.4)
    bad = u.copy()
    c = mesh.idx(mesh.g(0) + 5, mesh.g(1) + 7, 0)
    if poison == "nan_density":
        bad[c, 0] = float("nan")
    elif poison == "negative_density":
        bad[c, 0] = -bad[c, 0]
    elif poison == "negative_pressure":
        bad[c, 4] = 0.0  # E = 0 with momentum 0: p = 0, not > 0
        bad[c, 1] = 0.1
    else:
        bad[mesh.idx(0, mesh.g(1) + 7, 0), 0] = float("nan")
    g = gpu_solver(sys, mesh, bad, bc=bc, mode=FluxMode.Weno)
    if poison == "nan_ghost":
        o = O.OracleSolver(sys, mesh, bad, bc=bc, mode=FluxMode.Weno)
        assert g.dt_cfl() == o.dt_cfl()
        g.step(o.dt_cfl())
        return
    for call in ("dt_cfl", "advance"):
        with pytest.raises(EmgError) as e:
            if call == "dt_cfl":
                g.dt_cfl()
            else:
                g.advance(3)
        assert e.value.code == 4, (call, e.value)
    if poison == "nan_density":
        # a host-given step is checked on its result: a NaN stays in the state
        # (a negative ρ or p may be repaired by the fluxes of one step)
        with pytest.raises(EmgError) as e:
            g.step(1e-4)
        assert e.value.code == 4
    g.upload(u)
    assert g.dt_cfl() == O.OracleSolver(sys, mesh, u, bc=bc, mode=FluxMode.Weno).dt_cfl()
    g.advance(2)


def test_unsupported_options_are_rejected():
    sys, mesh, u, bc = W.explosion((16, 16, 1), 0.4)
    from emergence_b200 import EmgError
    with pytest.raises(EmgError):
        gpu_solver(sys, mesh.with_ghosts(4), np.zeros((mesh.with_ghosts(4).len(), 5)), bc=bc, mode=FluxMode.Weno)


@pytest.mark.parametrize("shape", [(64, 1, 1), (48, 40, 1), (20, 18, 16)])
def test_central_mode_matches_the_oracle_bitwise(shape):
    mesh, u = random_state(shape, seed=3, jump=False)
    bc = BC_SETS["periodic"]
    g = gpu_solver(SYS, mesh, u, bc=bc, mode=FluxMode.Central)
    o = O.OracleSolver(SYS, mesh, u, bc=bc, mode=FluxMode.Central)
    for _ in range(3):
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    assert np.array_equal(g.download(), o.download())
    assert g.counters() == o.counters()


@pytest.mark.parametrize("n", [(2, 1, 1), (1, 3, 1), (1, 1, 2), (2, 3, 4)])
@pytest.mark.parametrize("ng", [6, 10])
def test_periodic_axes_shorter_than_the_ghost_width_preserve_uniform_flow(n, ng):
    """tests/cpu.rs:266-298 on the device (central mode, no limiter)."""
    expected = np.array([1.0, 0.3, -0.2, 0.1, 1.0])
    mesh = Mesh.new(n, (0, 0, 0), (1, 1, 1), ng=ng)
    u = initial_state(SYS, mesh, np.broadcast_to(expected, mesh.n + (5,)).copy())
    g = gpu_solver(SYS, mesh, u, bc=BC_SETS["periodic"], mode=FluxMode.Central, positivity=False)
    g.step(1e-5)
    w = SYS.to_prim(mesh.interior(g.download()))
    assert np.all(np.abs(w - expected) < 1e-13)


@pytest.mark.parametrize("shape", [(96, 1, 1), (64, 56, 1), (24, 20, 18)])
def test_hybrid_mode_matches_the_oracle(shape):
    """Default reference mode: δ⁴ sensor switch between KEEP-PE central and WCNS."""
    sys_, mesh, u, bc = W.explosion(shape, 0.3 if shape[2] > 1 else 0.4)
    g = gpu_solver(sys_, mesh, u, bc=bc, mode=FluxMode.Hybrid)
    o = O.OracleSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Hybrid)
    for _ in range(5):
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    ug, uo = g.download(), o.download()
    err = rel_l1(ug, uo, mesh)
    print("hybrid", shape, "rel L1", err, "bitwise", np.array_equal(mesh.interior(ug), mesh.interior(uo)))
    assert np.all(err <= F64_TOL)
    cg, co = g.counters(), o.counters()
    assert cg[0] == co[0]
    assert 0 < co[1] <= co[0]
    if shape[1] > 1:
        assert co[1] < co[0]  # a genuine mix of central and shock-path faces
    # the sensor's log may round differently from the host's in the last ulp,
    # which can move a face across θ = 0 in rare cases
    assert abs(cg[1] - co[1]) <= 0.001 * co[1]


def test_hybrid_explosion_2d_256_short_run():
    sys_, mesh, u, bc = W.explosion_2d(256)
    g = gpu_solver(sys_, mesh, u, bc=bc, mode=FluxMode.Hybrid)
    o = O.OracleSolver(sys_, mesh, u, bc=bc, mode=FluxMode.Hybrid)
    assert g.advance(20) == 20
    o.advance(20)
    err = rel_l1(g.download(), o.download(), mesh)
    print("hybrid explosion_2d 20 steps rel L1", err)
    assert np.all(err <= F64_TOL)


def test_autotuned_launch_shapes_give_identical_results():
    """The autotuner only changes the sweep launch shapes; the state after a
    few steps is bitwise the same as with the planned shapes."""
    sys_, mesh, u, bc = W.explosion((40, 36, 28), 0.3)
    g0 = gpu_solver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno)
    g1 = gpu_solver(sys_, mesh, u, bc=bc, mode=FluxMode.Weno, autotune=True)
    for g in (g0, g1):
        g.advance(3)
    assert np.array_equal(g0.download(), g1.download())
    assert g0.counters() == g1.counters()
    g0.close()
    g1.close()


def test_download_into_a_pinned_host_buffer():
    """download(out=...) fills a caller's buffer (here page-locked memory from
    torch) with the same bytes as a fresh download; wrong shapes are refused."""
    import torch
    sys, mesh, u, bc = W.explosion((24, 20, 16), 0.3)
    g = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
    g.advance(3)
    ref = g.download()
    pinned = torch.empty(tuple(ref.shape), dtype=torch.float64, pin_memory=True).numpy()
    assert g.download(out=pinned) is pinned
    assert np.array_equal(pinned, ref)
    with pytest.raises(ValueError):
        g.download(out=np.empty((3, 5)))


def test_solvers_built_on_reused_pool_memory_give_identical_results():
    """The state arrays of a destroyed solver return to the library's memory
    pool and the next solver of the same size is built on them, stale data
    and all: its steps are bit for bit those of the first solver, and so are
    those of a solver built after the pool was trimmed."""
    from emergence_b200 import release_memory
    sys, mesh, u, bc = W.explosion((48, 40, 24), 0.3)
    r = []
    for trim in (False, False, True):
        if trim:
            release_memory()
        g = gpu_solver(sys, mesh, u, bc=bc, mode=FluxMode.Weno)
        g.advance(4)
        r.append((g.download(), g.t))
        g.close()
    assert all(np.array_equal(r[0][0], x[0]) and r[0][1] == x[1] for x in r[1:])
