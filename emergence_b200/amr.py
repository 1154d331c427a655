"""GpuAmr: block-AMR solver on the device, mirroring compressible-cuda's
``GpuAmr`` (fluid/crates/compressible-cuda/src/amr.rs:95-858) together with
the hierarchy construction of ``compressible::amr::Amr::new``
(fluid/crates/compressible/src/amr.rs:289-344), for the Euler system or, when
``sys`` is a FiveEq, the five-equation two-phase system (GpuSystem::FiveEq)."""
import ctypes as C

import numpy as np

from ._abi import EmgAmrConfig, EmgEos, EmgOpts, INIT_FN, check, lib
from .physics import FluxMode, Precision
from .solver import _c_bcs


def _cfg(cfg):
    c = EmgAmrConfig()
    c.b, c.levels, c.eps, c.regrid_every, c.ghosts = cfg["b"], cfg["levels"], cfg["eps"], cfg["regrid_every"], cfg["ghosts"]
    for d in range(3):
        c.base_blocks[d] = cfg["base_blocks"][d]
    return c


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def init_callback(fn, nv=5):
    """Wrap init(x[n,3]) -> w[n,nv] (primitive state at cell centres)."""
    def cb(ctx, x, n, w):
        xa = np.ctypeslib.as_array(x, shape=(n, 3)).copy()
        np.ctypeslib.as_array(w, shape=(n, nv))[...] = fn(xa)
    return INIT_FN(cb)


class GpuAmr:
    """Device block-AMR solver. ``cfg`` holds the fields of AmrConfig
    (b, levels, eps, regrid_every, base_blocks, ghosts). ``autotune``: on the
    first step, time the batched sweeps with one and two block rows per CTA
    and keep the faster per axis (results are the same either way).
    ``subcycle``: ``run_to`` takes subcycled steps (Amr::subcycle,
    fluid/crates/compressible/src/amr.rs:233-236), each level with its own
    time step; ``step`` / ``dt_cfl`` stay the global step as in the
    reference, ``step_subcycled`` / ``dt_cfl_subcycled`` are the subcycled
    ones."""

    def __init__(self, sys, cfg, lo, hi, bc, init=None, cfl=0.4, mode=FluxMode.Weno, tol=1e-3, positivity=True,
                 precision=Precision.F64, blocks=None, autotune=False, subcycle=False):
        from .five import FiveEq, _c_bcs7, _c_system
        self.cfg = dict(cfg)
        self._c = _cfg(cfg)
        five = isinstance(sys, FiveEq)
        self.nv = 7 if five else 5
        if five:
            self._e = _c_system(sys)
            self._b = _c_bcs7(bc)
        else:
            self._e = EmgEos(sys.eos.gamma, sys.eos.p_inf, sys.eos.b, sys.eos.q, sys.eos.cv)
            self._b = _c_bcs(bc)
        flags = (1 if autotune else 0) | (2 if subcycle else 0)
        self._o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, precision, flags)
        self._lo = np.ascontiguousarray(lo, dtype=np.float64)
        self._hi = np.ascontiguousarray(hi, dtype=np.float64)
        self.bcells = 1
        for d in range(3):
            self.bcells *= cfg["b"] if cfg["base_blocks"][d] > 0 else 1
        h = C.c_void_p()
        L = lib()
        if blocks is not None:
            desc, data = blocks
            desc = np.ascontiguousarray(desc, dtype=np.int64)
            data = np.ascontiguousarray(data, dtype=np.float64)
            create = L.emg_amr_create_five_from_blocks if five else L.emg_amr_create_from_blocks
            check(create(C.byref(self._c), C.byref(self._e), _dptr(self._lo), _dptr(self._hi), self._b,
                         C.byref(self._o), desc.ctypes.data_as(C.POINTER(C.c_int64)), desc.shape[0], _dptr(data),
                         C.byref(h)))
        else:
            self._cb = init_callback(init, self.nv)
            create = L.emg_amr_create_five if five else L.emg_amr_create
            check(create(C.byref(self._c), C.byref(self._e), _dptr(self._lo), _dptr(self._hi), self._b,
                         C.byref(self._o), self._cb, None, C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().emg_amr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt):
        check(lib().emg_amr_step(self._h, float(dt)))

    def dt_cfl(self):
        v = C.c_double()
        check(lib().emg_amr_dt_cfl(self._h, C.byref(v)))
        return v.value

    def step_subcycled(self, dt):
        """Level lmin by dt, finer levels by dt/2^(l-lmin) (Amr::step_subcycled)."""
        check(lib().emg_amr_step_subcycled(self._h, float(dt)))

    def dt_cfl_subcycled(self):
        v = C.c_double()
        check(lib().emg_amr_dt_cfl_subcycled(self._h, C.byref(v)))
        return v.value

    def run_to(self, t_end):
        n = C.c_uint64()
        check(lib().emg_amr_run_to(self._h, float(t_end), C.byref(n)))
        return n.value

    def regrid(self):
        check(lib().emg_amr_regrid(self._h))

    def block_count(self):
        b, l = C.c_uint64(), C.c_uint64()
        check(lib().emg_amr_block_count(self._h, C.byref(b), C.byref(l)))
        return b.value, l.value

    def leaf_count(self):
        """Leaf blocks of the hierarchy (GpuAmr::leaf_count,
        fluid/crates/compressible-cuda/src/amr.rs:855-857)."""
        return self.block_count()[1]

    def structure(self):
        nb, _ = self.block_count()
        out = np.zeros((nb, 5), dtype=np.int64)
        check(lib().emg_amr_structure(self._h, out.ctypes.data_as(C.POINTER(C.c_int64)), nb))
        return out

    def download(self):
        nb, _ = self.block_count()
        out = np.zeros((nb, self.bcells, self.nv))
        check(lib().emg_amr_download(self._h, _dptr(out), nb))
        return out

    def totals(self):
        out = np.zeros(self.nv)
        check(lib().emg_amr_totals(self._h, _dptr(out)))
        return out

    def counters(self):
        out = (C.c_uint64 * 4)()
        check(lib().emg_amr_counters(self._h, out))
        return list(out)

    def phase_times(self):
        out = np.zeros(5)
        check(lib().emg_amr_phase_times(self._h, _dptr(out)))
        return dict(zip(("restrict", "ghosts", "fluxes", "reflux_update", "regrid"), out))

    def launch_count(self):
        n = C.c_uint64()
        check(lib().emg_amr_launch_count(self._h, C.byref(n)))
        return n.value

    def synchronize(self):
        check(lib().emg_amr_synchronize(self._h))

    def stream(self):
        p = C.c_void_p()
        check(lib().emg_amr_stream(self._h, C.byref(p)))
        return p.value

    @property
    def t(self):
        v = C.c_double()
        check(lib().emg_amr_get_time(self._h, C.byref(v)))
        return v.value

    @property
    def steps(self):
        v = C.c_uint64()
        check(lib().emg_amr_steps(self._h, C.byref(v)))
        return v.value
