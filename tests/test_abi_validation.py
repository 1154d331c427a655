"""Argument checks of the C ABI, on any host (no GPU needed).

Every create entry point validates its arguments before it touches a device,
so a bad call is reported as EMG_ERR_INVALID with a message that names the
problem, also on a machine without a GPU. Where the reference rejects an input
(an unpaired periodic axis, C/solver.rs:41-60; the WCNS stencil's ghost depth,
C/amr.rs:61 and C/solver.rs:33), the message says so.
"""
import ctypes as C

import numpy as np
import pytest

from emergence_b200 import _abi
from emergence_b200._abi import EmgAmrConfig, EmgBc, EmgEos, EmgMesh, EmgOpts, INIT_FN

INVALID, NO_DEVICE = 1, 7
PERIODIC, OUTFLOW, REFLECT, DIRICHLET, CHARACTERISTIC = range(5)
HYBRID, WENO, CENTRAL = range(3)


def lib():
    return _abi.lib()


def no_gpu():
    n = C.c_int(-1)
    assert lib().emg_device_count(C.byref(n)) == 0
    return n.value == 0


def err():
    return lib().emg_last_error().decode()


def bcs(kinds):
    arr = (EmgBc * 6)()
    for i, k in enumerate(kinds):
        arr[i].kind = k
    return arr


def mesh(n=(8, 8, 1), ng=6):
    m = EmgMesh()
    for d in range(3):
        m.n[d] = n[d]
        m.dx[d] = 1.0 / max(n[d], 1)
    m.ng = ng
    return m


def padded(m):
    return int(np.prod([m.n[d] + 2 * m.ng if m.n[d] > 1 else 1 for d in range(3)]))


EOS = EmgEos(1.4, 0.0, 0.0, 0.0, 1.0)


def uniform_create(m, bc, opts, length=None):
    length = padded(m) if length is None else length
    u = np.zeros((max(length, 1), 5))
    h = C.c_void_p()
    rc = lib().emg_uniform_create(C.byref(m), C.byref(EOS), bc, C.byref(opts),
                                  u.ctypes.data_as(C.POINTER(C.c_double)), length, C.byref(h))
    assert not h.value  # nothing is handed out on failure
    return rc


def opts(mode=WENO, tol=1e-3, precision=0):
    return EmgOpts(0.5, tol, mode, 1, precision, 0)


OUT6 = [OUTFLOW] * 6


@pytest.mark.parametrize("case, want", [
    (dict(m=mesh(ng=4)), "ng >= 5"),
    (dict(m=mesh(n=(1, 1, 1))), "no active axis"),
    (dict(m=mesh(n=(0, 8, 1))), "extents"),
    (dict(m=mesh(), dx0=0.0), "dx must be > 0"),
    (dict(o=opts(mode=7)), "flux mode"),
    (dict(o=opts(mode=HYBRID, tol=0.0)), "tol > 0"),
    (dict(o=opts(precision=5)), "precision"),
    (dict(bc=[9, 1, 1, 1, 1, 1]), "boundary condition"),
    (dict(bc=[PERIODIC, OUTFLOW, 1, 1, 1, 1]), "paired"),
    (dict(length=17), "length"),
])
def test_uniform_create_rejects_bad_arguments(case, want):
    m = case.get("m", mesh())
    if "dx0" in case:
        m.dx[0] = case["dx0"]
    rc = uniform_create(m, bcs(case.get("bc", OUT6)), case.get("o", opts()), case.get("length"))
    assert rc == INVALID and want in err(), (rc, err())


def test_uniform_create_with_valid_arguments_reaches_the_device_check():
    if not no_gpu():
        pytest.skip("a GPU is visible: the valid call would create a solver")
    rc = uniform_create(mesh(), bcs(OUT6), opts())
    assert rc == NO_DEVICE and "device" in err()


def test_periodic_pairing_only_matters_on_active_axes():
    if not no_gpu():
        pytest.skip("a GPU is visible")
    # the third axis is inactive (n = 1): its sides are never filled
    rc = uniform_create(mesh(n=(8, 8, 1)), bcs([OUTFLOW] * 4 + [PERIODIC, OUTFLOW]), opts())
    assert rc == NO_DEVICE


def test_noalloc_step_rejects_bad_arguments():
    m, bc, o = mesh(), bcs(OUT6), opts()
    n = padded(m) * 5 * 8  # bytes of one state
    buf = (C.c_char * (3 * n))()
    p = C.cast(buf, C.c_void_p).value
    f = lib().emg_uniform_step_noalloc

    def call(m=m, bc=bc, o=o, a=p, b=p + n, dt=1e-3):
        return f(C.byref(m), C.byref(EOS), bc, C.byref(o), C.c_void_p(a), C.c_void_p(b), dt, None)

    assert call(a=None) == INVALID and "null" in err()
    assert call(b=p) == INVALID and "overlap" in err()
    # partial overlaps either way round
    assert call(b=p + n - 8) == INVALID and "overlap" in err()
    assert call(a=p + n - 8) == INVALID and "overlap" in err()
    assert call(m=mesh(n=(64, 64, 40))) == INVALID and "EMG_NOALLOC_MAX_CELLS" in err()
    assert call(m=mesh(ng=3)) == INVALID and "ng >= 5" in err()
    # the checks emg_uniform_create makes apply here too
    assert call(o=opts(mode=HYBRID, tol=0.0)) == INVALID and "tol > 0" in err()
    assert call(bc=bcs([PERIODIC, OUTFLOW, OUTFLOW, OUTFLOW, OUTFLOW, OUTFLOW])) == INVALID
    assert "paired" in err()
    for dt in (0.0, -1e-3, float("nan"), float("inf")):
        assert call(dt=dt) == INVALID and "dt" in err(), dt


def batch_create(n, dx, bc=(OUTFLOW, OUTFLOW), o=None):
    o = opts() if o is None else o
    n = np.asarray(n, dtype=np.int64)
    dx = np.asarray(dx, dtype=np.float64)
    u = np.zeros((max(int(n.clip(0).sum()), 1), 5))
    arr = (EmgBc * 2)()
    arr[0].kind, arr[1].kind = bc
    h = C.c_void_p()
    rc = lib().emg_batch1d_create(C.byref(EOS), C.byref(o), arr, len(n), n.ctypes.data_as(C.POINTER(C.c_int64)),
                                  dx.ctypes.data_as(C.POINTER(C.c_double)), u.ctypes.data_as(C.POINTER(C.c_double)),
                                  C.byref(h))
    assert not h.value
    return rc


@pytest.mark.parametrize("args, want", [
    (dict(n=[64, 1], dx=[0.1, 0.1]), "at least 2 cells"),
    (dict(n=[64, 4], dx=[0.1, 0.1], bc=(REFLECT, OUTFLOW)), "at least 6 cells"),
    (dict(n=[64, 64], dx=[0.1, 0.0]), "dx must be > 0"),
    (dict(n=[64], dx=[0.1], bc=(PERIODIC, OUTFLOW)), "paired"),
    (dict(n=[64], dx=[0.1], bc=(CHARACTERISTIC, OUTFLOW)), "boundaries"),
    (dict(n=[64], dx=[0.1], o=opts(mode=5)), "mode"),
    (dict(n=[64], dx=[0.1], o=opts(precision=3)), "precision"),
])
def test_batch1d_create_rejects_bad_arguments(args, want):
    rc = batch_create(**args)
    assert rc == INVALID and want in err(), (rc, err())


def amr_create(cfg=None, bc=None, o=None, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 0.0)):
    if cfg is None:
        cfg = EmgAmrConfig(16, 2, 1e-3, 4, (4, 4, 0), 5)
    bc = bcs(OUT6) if bc is None else bc
    o = opts() if o is None else o
    lo_a, hi_a = (C.c_double * 3)(*lo), (C.c_double * 3)(*hi)
    calls = []
    init = INIT_FN(lambda ctx, x, n, w: calls.append(n))
    h = C.c_void_p()
    rc = lib().emg_amr_create(C.byref(cfg), C.byref(EOS), lo_a, hi_a, bc, C.byref(o), init, None, C.byref(h))
    assert not h.value and not calls  # rejected before any block is initialised
    return rc


@pytest.mark.parametrize("args, want", [
    (dict(cfg=EmgAmrConfig(4, 2, 1e-3, 4, (4, 4, 0), 5)), "b >= 6"),
    (dict(cfg=EmgAmrConfig(16, 0, 1e-3, 4, (4, 4, 0), 5)), "levels"),
    (dict(cfg=EmgAmrConfig(16, 2, 1e-3, 0, (4, 4, 0), 5)), "regrid_every"),
    (dict(cfg=EmgAmrConfig(64, 2, 1e-3, 4, (4, 4, 0), 5)), "above 32"),
    (dict(cfg=EmgAmrConfig(16, 2, 1e-3, 4, (0, 0, 0), 5)), "no active axis"),
    (dict(bc=bcs([CHARACTERISTIC] + [OUTFLOW] * 5)), "characteristic"),
    (dict(bc=bcs([7] + [OUTFLOW] * 5)), "boundary condition"),
    (dict(bc=bcs([OUTFLOW, PERIODIC] + [OUTFLOW] * 4)), "paired"),
    (dict(o=opts(mode=9)), "flux mode"),
    (dict(o=opts(mode=HYBRID, tol=-1.0)), "tol > 0"),
    (dict(o=opts(precision=3)), "precision"),
])
def test_amr_create_rejects_bad_arguments(args, want):
    rc = amr_create(**args)
    assert rc == INVALID and want in err(), (rc, err())


def test_adjoint_create_rejects_forms_it_does_not_differentiate():
    m = mesh()
    u = np.zeros((padded(m), 5))
    for o, want in ((opts(precision=1), "FP64"), (opts(mode=HYBRID), "WENO")):
        h = C.c_void_p()
        rc = lib().emg_adjoint_create(C.byref(m), C.byref(EOS), bcs(OUT6), C.byref(o),
                                      u.ctypes.data_as(C.POINTER(C.c_double)), padded(m), C.byref(h))
        assert rc == INVALID and want in err() and not h.value


def test_amr_create_from_blocks_rejects_an_empty_hierarchy():
    cfg = EmgAmrConfig(16, 2, 1e-3, 4, (4, 4, 0), 5)
    lo_a, hi_a = (C.c_double * 3)(0.0, 0.0, 0.0), (C.c_double * 3)(1.0, 1.0, 0.0)
    desc = (C.c_int64 * 5)()
    u = (C.c_double * 5)()
    h = C.c_void_p()
    rc = lib().emg_amr_create_from_blocks(C.byref(cfg), C.byref(EOS), lo_a, hi_a, bcs(OUT6), C.byref(opts()), desc, 0,
                                          u, C.byref(h))
    assert rc == INVALID and "at least one block" in err() and not h.value


UNFILLABLE = 5


def from_blocks(blocks, levels=3, bc=None):
    """emg_amr_create_from_blocks on a 2-D 4×4-block base (16² cells per
    block) with the given (level, i, j, k, leaf) rows; the data are zeros
    (the hierarchy is checked before the data are read)."""
    cfg = EmgAmrConfig(16, levels, 1e-3, 4, (4, 4, 0), 5)
    lo_a, hi_a = (C.c_double * 3)(0.0, 0.0, 0.0), (C.c_double * 3)(1.0, 1.0, 0.0)
    desc = np.asarray(blocks, dtype=np.int64).reshape(-1, 5)
    u = np.zeros((len(desc), 16 * 16, 5))
    h = C.c_void_p()
    rc = lib().emg_amr_create_from_blocks(C.byref(cfg), C.byref(EOS), lo_a, hi_a, bcs(OUT6) if bc is None else bc,
                                          C.byref(opts()), desc.ctypes.data_as(C.POINTER(C.c_int64)), len(desc),
                                          u.ctypes.data_as(C.POINTER(C.c_double)), C.byref(h))
    if rc == 0:
        lib().emg_amr_destroy(h)
    else:
        assert not h.value
    return rc


def base(leaf_except=()):
    return [[0, i, j, 0, 0 if (i, j) in leaf_except else 1] for i in range(4) for j in range(4)]


def children(l, i, j, leaf=1):
    return [[l + 1, 2 * i + a, 2 * j + b, 0, leaf] for a in range(2) for b in range(2)]


def balanced():
    """Every base block refined once, and the level-1 block (3,3) once more:
    every block's parent has all its same-level neighbours."""
    rows = base(leaf_except=[(i, j) for i in range(4) for j in range(4)])
    for i in range(4):
        for j in range(4):
            rows += children(0, i, j)
    rows = [r if r[:3] != [1, 3, 3] else [1, 3, 3, 0, 0] for r in rows]
    return rows + children(1, 3, 3)


def test_create_from_blocks_accepts_a_balanced_hierarchy_before_device_work():
    if not no_gpu():
        pytest.skip("a GPU is visible")
    # the hierarchy passes its checks; only then is the (absent) device asked for
    assert from_blocks(balanced()) == NO_DEVICE


def test_create_from_blocks_reports_ghosts_without_a_source():
    """Hierarchies the reference's Amr never produces (it keeps 2:1 balance,
    C/amr.rs:951-972, and every base block): their ghost cells have no source
    within one coarser level, so they are rejected as EMG_ERR_UNFILLABLE
    before any device work, not discovered by a kernel."""
    rows = [r for r in base() if (r[1], r[2]) != (2, 2)]
    assert from_blocks(rows) == UNFILLABLE and "base block" in err()
    # a level-2 block next to a level-0 leaf: the base block (0,0) refined,
    # its child (1, 1,1) refined again, nothing else
    rows = base(leaf_except=[(0, 0)]) + children(0, 0, 0)
    rows = [r if r[:3] != [1, 1, 1] else [1, 1, 1, 0, 0] for r in rows] + children(1, 1, 1)
    assert from_blocks(rows) == UNFILLABLE and "2:1" in err()


@pytest.mark.parametrize("case, want", [
    ("duplicate", "twice"),
    ("outside", "outside"),
    ("leaf_with_children", "leaf block has children"),
    ("ancestor_missing_child", "lacks some of its children"),
    ("orphan", "without its parent"),
])
def test_create_from_blocks_rejects_inconsistent_hierarchies(case, want):
    rows = base()
    if case == "duplicate":
        rows = rows + [rows[0]]
    elif case == "outside":
        rows = rows + [[0, 4, 0, 0, 1]]
    elif case == "leaf_with_children":
        rows = rows + children(0, 1, 1)
    elif case == "ancestor_missing_child":
        rows = base(leaf_except=[(1, 1)]) + children(0, 1, 1)[:3]
    elif case == "orphan":
        rows = rows + [[2, 4, 4, 0, 1]]
    assert from_blocks(rows) == INVALID and want in err(), err()
