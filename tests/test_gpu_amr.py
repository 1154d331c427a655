"""Parity of the device block-AMR solver with the AMR oracle (needs a B200).

The device keeps the reference's block ids, so hierarchies are compared block
by block: structure (level, coordinates, leaf flag) exactly, block data to the
parity bound of 1e-12 relative L1 (and, where the arithmetic order is the same,
bit for bit)."""
import numpy as np
import pytest

from emergence_b200 import workloads as W
from emergence_b200.physics import Bc, Euler, FluxMode, Nasg, Precision
from oracle import pyoracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12


def gpu_amr(*a, **k):
    from emergence_b200 import GpuAmr
    return GpuAmr(*a, **k)


def rel_l1_blocks(a, b, structure):
    leaves = structure[:, 4] == 1
    da, db = a[leaves], b[leaves]
    num = np.abs(da - db).reshape(-1, 5).sum(axis=0)
    den = np.abs(db).reshape(-1, 5).sum(axis=0)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def compare(g, o, bitwise=True):
    sg, so = g.structure(), o.structure()
    assert sg.shape == so.shape and np.array_equal(sg, so), "hierarchies differ"
    ug, uo = g.download(), o.download()
    err = rel_l1_blocks(ug, uo, so)
    assert np.all(err <= TOL), err
    if bitwise:
        leaves = so[:, 4] == 1
        assert np.array_equal(ug[leaves], uo[leaves]), float(np.nanmax(np.abs(ug[leaves] - uo[leaves])))
    return err


@pytest.mark.parametrize("case", ["explosion2d", "bubble2d"])
def test_initial_hierarchy_matches_the_oracle(case):
    if case == "explosion2d":
        s, cfg, lo, hi, bc, init = W.amr_explosion(dim=2, base=4, levels=3)
    else:
        s, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g = gpu_amr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    compare(g, o)
    assert g.block_count() == o.block_count()


def test_steps_from_the_same_hierarchy_match_bitwise():
    s, cfg, lo, hi, bc, init = W.amr_explosion(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g = gpu_amr(s, cfg, lo, hi, bc, mode=FluxMode.Weno, blocks=(o.structure(), o.download()))
    for _ in range(3):  # no regrid yet (due after step 4)
        dt = o.dt_cfl()
        assert g.dt_cfl() == dt
        g.step(dt)
        o.step(dt)
        compare(g, o)
    assert g.counters() == o.counters()


@pytest.mark.parametrize("mode", [FluxMode.Weno, FluxMode.Hybrid])
def test_shock_bubble_2d_with_regrids(mode):
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=mode)
    g = gpu_amr(s, cfg, lo, hi, bc, init, mode=mode)
    compare(g, o)
    for i in range(10):  # regrids after steps 4 and 8
        dt = o.dt_cfl()
        assert abs(g.dt_cfl() / dt - 1.0) < 1e-14
        g.step(dt)
        o.step(dt)
        err = compare(g, o, bitwise=False)
    print("shock-bubble 2-D", "mode", mode, "leaves", o.block_count(), "rel L1", err)
    assert abs(g.t - o.t) <= 1e-15 * o.t


def test_shock_bubble_3d_small():
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=3, base=2, levels=2)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g = gpu_amr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    compare(g, o)
    for _ in range(5):
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    err = compare(g, o, bitwise=False)
    print("shock-bubble 3-D small: leaves", o.block_count(), "rel L1", err)


def test_amr_mixed_precision_error():
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g = gpu_amr(s, cfg, lo, hi, bc, mode=FluxMode.Weno, precision=Precision.Mixed,
                blocks=(o.structure(), o.download()))
    for _ in range(3):
        dt = o.dt_cfl()
        g.step(dt)
        o.step(dt)
    st = o.structure()
    ug, uo = g.download(), o.download()
    leaves = st[:, 4] == 1
    num = np.abs(ug[leaves] - uo[leaves]).reshape(-1, 5).sum(axis=0)
    den = np.abs(uo[leaves]).reshape(-1, 5).sum(axis=0)
    # fields that are (nearly) zero in the oracle — the transverse momenta
    # before the shock reaches the bubble — are measured against the density
    den = np.maximum(den, 1e-3 * den[0])
    err = num / den
    print("AMR mixed rel L1", err)
    assert np.all(err <= 1e-6), err


def test_conservation_across_levels_on_the_device():
    s, cfg, lo, hi, bc, init = W.amr_explosion(dim=2, base=4, levels=3, radius=0.25)
    bc = [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
    g = gpu_amr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    t0 = g.totals()
    for _ in range(3):
        g.step(g.dt_cfl())
    t1 = g.totals()
    assert abs(t1[0] - t0[0]) <= 1e-13 * abs(t0[0])
    assert abs(t1[4] - t0[4]) <= 1e-13 * abs(t0[4])


def _contact_strip(base=4, levels=3, b=8, x0=0.85, width=0.1, u=3.0):
    """A dense strip (ρ = 2 in ρ = 1, p = 1) carried at u = 3 towards the
    outflow side: the hierarchy refines ahead of it and coarsens behind it,
    several levels in one regrid."""
    s = Euler(Nasg.ideal(1.4))
    cfg = dict(b=b, levels=levels, eps=1e-3, regrid_every=2, base_blocks=[base, base, 0], ghosts=5)

    def init(x):
        w = np.zeros((x.shape[0], 5))
        inside = (np.abs(x[:, 0] - x0) < width / 2) & (np.abs(x[:, 1] - 0.5) < 0.3)
        w[:, 0] = np.where(inside, 2.0, 1.0)
        w[:, 1] = u
        w[:, 4] = 1.0
        return w

    far = s.to_cons(np.array([1.0, u, 0.0, 0.0, 1.0]))
    bc = [[Bc.dirichlet(far), Bc.Outflow], [Bc.Outflow, Bc.Outflow], [Bc.Outflow, Bc.Outflow]]
    return s, cfg, (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), bc, init


def test_batched_regrids_match_the_sequential_oracle():
    """Regrids refine and coarsen many blocks of several levels at once; the
    device predicts each level's refinements in one launch and restricts each
    level's coarsenings in one set of launches. Hierarchy and block data must
    equal the oracle's one-at-a-time order bit for bit after every step."""
    s, cfg, lo, hi, bc, init = _contact_strip()
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g = gpu_amr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    compare(g, o)
    added = removed = 0
    multi_level = False
    for _ in range(18):
        before = {tuple(r[:4]) for r in o.structure()}
        dt = o.dt_cfl()
        assert g.dt_cfl() == dt
        g.step(dt)
        o.step(dt)
        compare(g, o)
        after = {tuple(r[:4]) for r in o.structure()}
        added += len(after - before)
        removed += len(before - after)
        multi_level |= len({k[0] for k in before - after}) > 1
    print("batched regrids: blocks added", added, "removed", removed)
    assert added >= 40 and removed >= 80 and multi_level


def test_autotuned_amr_sweeps_give_identical_results():
    """The AMR autotuner only changes the batched sweeps' CTA shape; hierarchy
    and data after steps with a regrid equal the untuned run bit for bit."""
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=3, base=2, levels=2)
    g0 = gpu_amr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    g1 = gpu_amr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno, autotune=True)
    for _ in range(5):
        dt = g0.dt_cfl()
        assert g1.dt_cfl() == dt
        g0.step(dt)
        g1.step(dt)
    assert np.array_equal(g0.structure(), g1.structure())
    assert np.array_equal(g0.download(), g1.download())
    assert g0.counters() == g1.counters()


def test_inadmissible_leaf_state_is_reported():
    """A NaN planted in one leaf cell of an adopted hierarchy: dt_cfl and step
    return EMG_ERR_INADMISSIBLE (no trap, no device fault)."""
    from emergence_b200 import EmgError
    s, cfg, lo, hi, bc, init = W.shock_bubble(dim=2, base=4, levels=3)
    o = O.OracleAmr(s, cfg, lo, hi, bc, init, mode=FluxMode.Weno)
    st, u = o.structure(), o.download()
    leaf = int(np.flatnonzero(st[:, 4] == 1)[0])
    u = u.copy()
    u[leaf, 37, 0] = float("nan")
    g = gpu_amr(s, cfg, lo, hi, bc, mode=FluxMode.Weno, blocks=(st, u))
    with pytest.raises(EmgError) as e:
        g.dt_cfl()
    assert e.value.code == 4
    with pytest.raises(EmgError) as e:
        g.step(1e-4)
    assert e.value.code == 4
