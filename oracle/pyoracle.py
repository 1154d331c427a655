"""CPU ORACLE — test infrastructure only.

ctypes wrapper of ``liboracle.so``, the C++ restatement of the reference CPU
f64 solver (oracle.hpp). Used only by tests/, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of bench.py, as the checker and the timed CPU baseline;
the product package never imports it.

``OracleSolver`` has the same constructor and methods as
``emergence_b200.GpuSolver`` so that parity tests drive both identically.
"""
import ctypes as C
import math
import os
import subprocess

import numpy as np

from emergence_b200._abi import EmgBc, EmgBc7, EmgEos, EmgFiveSystem, EmgMesh, EmgOpts
from emergence_b200.physics import Bc, FluxMode

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_D = C.POINTER(C.c_double)
_U64 = C.POINTER(C.c_uint64)
_P = C.c_void_p
SIGS = {
    "emgo_last_error": (C.c_char_p, []),
    "emgo_num_threads": (C.c_int, []),
    "emgo_set_num_threads": (None, [C.c_int]),
    "emgo_state_hash": (C.c_int, [C.POINTER(EmgMesh), _D, C.c_size_t, C.POINTER(C.c_uint64)]),
    "emgo_uniform_create": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgEos), C.POINTER(EmgBc), C.POINTER(EmgOpts),
                                      _D, C.c_size_t, C.POINTER(_P)]),
    "emgo_uniform_destroy": (C.c_int, [_P]),
    "emgo_uniform_step": (C.c_int, [_P, C.c_double]),
    "emgo_uniform_dt_cfl": (C.c_int, [_P, _D]),
    "emgo_uniform_run_to": (C.c_int, [_P, C.c_double, _U64]),
    "emgo_uniform_download": (C.c_int, [_P, _D, C.c_size_t]),
    "emgo_uniform_upload": (C.c_int, [_P, _D, C.c_size_t]),
    "emgo_uniform_totals": (C.c_int, [_P, _D]),
    "emgo_uniform_counters": (C.c_int, [_P, _U64]),
    "emgo_uniform_get_time": (C.c_int, [_P, _D]),
    "emgo_uniform_set_time": (C.c_int, [_P, C.c_double]),
    "emgo_uniform_fill_ghosts": (C.c_int, [_P]),
    "emgo_uniform_fill_ghosts_of": (C.c_int, [_P, _D, C.c_size_t]),
    "emgo_line_fluxes": (C.c_int, [C.POINTER(EmgEos), _D, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                   _D, _D, _U64]),
    "emgo_positivity_limit": (C.c_int, [C.POINTER(EmgEos), _D, C.c_int, C.c_int, C.c_int, C.c_double, _D, _D, _U64]),
    "emgo_midpoint_flux": (C.c_int, [C.POINTER(EmgEos), _D, C.c_int, C.c_int, _D, _D, C.POINTER(C.c_int)]),
    "emgo_riemann_flux": (C.c_int, [C.POINTER(EmgEos), _D, _D, C.c_int, _D, _D]),
    "emgo_weno5z_interp": (C.c_int, [C.c_double] * 5 + [_D]),
    "emgo_to_prim": (C.c_int, [C.POINTER(EmgEos), _D, _D]),
    "emgo_to_cons": (C.c_int, [C.POINTER(EmgEos), _D, _D]),
    "emgo_eigen": (C.c_int, [C.POINTER(EmgEos), _D, C.c_int, _D, _D]),
    "emgo_max_speed": (C.c_int, [C.POINTER(EmgEos), _D, C.c_int, _D]),
    "emgo_admissible": (C.c_int, [C.POINTER(EmgEos), _D]),
    "emgo_characteristic_ghost_layer": (C.c_int, [C.POINTER(EmgEos), _D, _D, _D, C.c_int, C.c_int, C.c_double, _D]),
    "emgo_exact_star": (C.c_int, [_D, _D, C.POINTER(EmgEos), C.POINTER(EmgEos), _D]),
    "emgo_exact_sample": (C.c_int, [_D, _D, C.POINTER(EmgEos), C.POINTER(EmgEos), _D, C.c_size_t, _D]),
    "emgo_dual_run": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgEos), C.POINTER(EmgBc), C.POINTER(EmgOpts), _D, _D,
                                C.c_size_t, C.c_double, _D, C.c_size_t, C.c_int, _D, _D, _D, _D, _D, _D]),
    "emgo_box_objective": (C.c_int, [_P, C.c_int, _D, _D, _D]),
    "emgo_five_create": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgFiveSystem), C.POINTER(EmgBc7),
                                   C.POINTER(EmgOpts), _D, C.c_size_t, C.POINTER(_P)]),
    "emgo_five_destroy": (C.c_int, [_P]),
    "emgo_five_step": (C.c_int, [_P, C.c_double]),
    "emgo_five_dt_cfl": (C.c_int, [_P, _D]),
    "emgo_five_run_to": (C.c_int, [_P, C.c_double, _U64]),
    "emgo_five_download": (C.c_int, [_P, _D, C.c_size_t]),
    "emgo_five_fill_ghosts": (C.c_int, [_P]),
    "emgo_five_totals": (C.c_int, [_P, _D]),
    "emgo_five_counters": (C.c_int, [_P, _U64]),
    "emgo_five_get_time": (C.c_int, [_P, _D]),
    "emgo_five_to_cons": (C.c_int, [C.POINTER(EmgFiveSystem), _D, _D]),
    "emgo_five_props": (C.c_int, [C.POINTER(EmgFiveSystem), _D, C.c_double, _D]),
    "emgo_dual_step_cons": (C.c_int, [C.POINTER(EmgMesh), C.POINTER(EmgEos), C.POINTER(EmgBc), C.POINTER(EmgOpts), _D,
                                      _D, C.c_size_t, C.c_double, C.c_double, _D, _D]),
}

_lib = None


def build():
    """Compile liboracle.so from oracle.hpp / oracle_capi.cpp (make)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _chk(code):
    if code != 0:
        raise RuntimeError(f"oracle error {code}: {lib().emgo_last_error().decode()}")


def dptr(a):
    return a.ctypes.data_as(_D)


def c_eos(eos):
    return EmgEos(eos.gamma, eos.p_inf, eos.b, eos.q, eos.cv)


def arr(x):
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def set_threads(n):
    lib().emgo_set_num_threads(int(n))


def num_threads():
    return lib().emgo_num_threads()


class OracleSolver:
    """C++ restatement of ``compressible::Solver`` (Euler system)."""

    def __init__(self, sys, mesh, u, bc=None, cfl=0.5, mode=FluxMode.Hybrid, tol=1e-3, positivity=True,
                 precision=0):
        from emergence_b200.solver import _c_bcs, _c_mesh
        self.sys, self.mesh = sys, mesh
        self.bc = bc if bc is not None else [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
        u = arr(u)
        self._m = _c_mesh(mesh)
        self._e = c_eos(sys.eos)
        self._b = _c_bcs(self.bc)
        self._o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, 0, 0)
        h = C.c_void_p()
        _chk(lib().emgo_uniform_create(C.byref(self._m), C.byref(self._e), self._b, C.byref(self._o), dptr(u),
                                       mesh.len(), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().emgo_uniform_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt):
        _chk(lib().emgo_uniform_step(self._h, float(dt)))

    def dt_cfl(self):
        v = C.c_double()
        _chk(lib().emgo_uniform_dt_cfl(self._h, C.byref(v)))
        return v.value

    def run_to(self, t_end):
        n = C.c_uint64()
        _chk(lib().emgo_uniform_run_to(self._h, float(t_end), C.byref(n)))
        return n.value

    def advance(self, nsteps, t_end=math.inf):
        """Same stepping rule as GpuSolver.advance, on the CPU."""
        taken = 0
        for _ in range(int(nsteps)):
            t = self.t
            if math.isfinite(t_end):
                if not (t < t_end - 1e-10 * abs(t_end)):
                    break
                dt = min(self.dt_cfl(), t_end - t)
            else:
                dt = self.dt_cfl()
            self.step(dt)
            taken += 1
        return taken

    def download(self):
        out = np.empty((self.mesh.len(), 5))
        _chk(lib().emgo_uniform_download(self._h, dptr(out), self.mesh.len()))
        return out

    def upload(self, u):
        u = arr(u)
        _chk(lib().emgo_uniform_upload(self._h, dptr(u), self.mesh.len()))

    def totals(self):
        out = np.empty(5)
        _chk(lib().emgo_uniform_totals(self._h, dptr(out)))
        return out

    def counters(self):
        out = (C.c_uint64 * 4)()
        _chk(lib().emgo_uniform_counters(self._h, out))
        return list(out)

    @property
    def t(self):
        v = C.c_double()
        _chk(lib().emgo_uniform_get_time(self._h, C.byref(v)))
        return v.value

    @t.setter
    def t(self, value):
        _chk(lib().emgo_uniform_set_time(self._h, float(value)))

    def fill_ghosts(self):
        _chk(lib().emgo_uniform_fill_ghosts(self._h))

    def fill_ghosts_of(self, u):
        u = arr(u).copy()
        _chk(lib().emgo_uniform_fill_ghosts_of(self._h, dptr(u), self.mesh.len()))
        return u

    def prim(self, i, j, k):
        m = self.mesh
        u = self.download()[m.idx(i + m.g(0), j + m.g(1), k + m.g(2))]
        return to_prim(self.sys.eos, u)


# ---- unit-level helpers

OBJ_PRESSURE, OBJ_ENERGY = 0, 1


def dual_run(sys, mesh, w0, dw0, dgamma, dts, objective, box_lo, box_hi, bc, mode=FluxMode.Weno, positivity=True,
             tol=1e-3, want_state=False):
    """Forward-mode derivative of a frozen-dt run on the CPU: starts from the
    padded primitive state ``w0`` with tangent ``dw0`` (and ``dgamma`` on γ),
    takes one SSP-RK3 step per entry of ``dts`` and returns (J, dJ) of the box
    objective (OBJ_PRESSURE: Σ p·vol, OBJ_ENERGY: Σ E·vol over interior cells
    whose centre lies in [box_lo, box_hi]); with want_state also the final
    conserved state and its tangent (padded AoS)."""
    from emergence_b200.solver import _c_bcs, _c_mesh
    w0, dw0 = arr(w0).reshape(-1, 5), arr(dw0).reshape(-1, 5)
    dts = arr(dts).reshape(-1)
    m, e, b = _c_mesh(mesh), c_eos(sys.eos), _c_bcs(bc)
    o = EmgOpts(0.5, tol, mode, 1 if positivity else 0, 0, 0)
    J, dJ = C.c_double(), C.c_double()
    blo, bhi = arr(box_lo), arr(box_hi)
    uo = np.zeros_like(w0) if want_state else None
    duo = np.zeros_like(w0) if want_state else None
    _chk(lib().emgo_dual_run(C.byref(m), C.byref(e), b, C.byref(o), dptr(w0), dptr(dw0), w0.shape[0], float(dgamma),
                             dptr(dts), dts.shape[0], int(objective), dptr(blo), dptr(bhi), C.byref(J), C.byref(dJ),
                             dptr(uo) if want_state else None, dptr(duo) if want_state else None))
    if want_state:
        return J.value, dJ.value, uo, duo
    return J.value, dJ.value


def dual_step(sys, mesh, u, du, dgamma, dt, bc, mode=FluxMode.Weno, positivity=True, tol=1e-3):
    """One SSP-RK3 step of size dt in dual numbers from the padded conserved
    state u with tangent du (dgamma on γ): returns (u', du')."""
    from emergence_b200.solver import _c_bcs, _c_mesh
    u, du = arr(u).reshape(-1, 5), arr(du).reshape(-1, 5)
    m, e, b = _c_mesh(mesh), c_eos(sys.eos), _c_bcs(bc)
    o = EmgOpts(0.5, tol, mode, 1 if positivity else 0, 0, 0)
    u1, du1 = np.zeros_like(u), np.zeros_like(u)
    _chk(lib().emgo_dual_step_cons(C.byref(m), C.byref(e), b, C.byref(o), dptr(u), dptr(du), u.shape[0],
                                   float(dgamma), float(dt), dptr(u1), dptr(du1)))
    return u1, du1


def box_objective(solver, objective, box_lo, box_hi):
    """The box objective of an OracleSolver's current state."""
    J = C.c_double()
    _chk(lib().emgo_box_objective(solver._h, int(objective), dptr(arr(box_lo)), dptr(arr(box_hi)), C.byref(J)))
    return J.value


def line_fluxes(eos, w, d, ng, mode, tol=1e-3, lam=0.0):
    w = arr(w)
    n = w.shape[0] - 2 * ng
    out = np.zeros((n + 1, 5))
    uf = np.zeros(n + 1)
    st = (C.c_uint64 * 4)()
    e = c_eos(eos)
    _chk(lib().emgo_line_fluxes(C.byref(e), dptr(w), w.shape[0], d, ng, mode, tol, lam, dptr(out), dptr(uf), st))
    return out, uf, list(st)


def positivity_limit(eos, w, d, ng, lam, flux, uface):
    w, flux, uface = arr(w), arr(flux).copy(), arr(uface).copy()
    e = c_eos(eos)
    n = C.c_uint64()
    _chk(lib().emgo_positivity_limit(C.byref(e), dptr(w), w.shape[0], d, ng, lam, dptr(flux), dptr(uface),
                                     C.byref(n)))
    return flux, uface, n.value


def riemann_flux(eos, wl, wr, d):
    e = c_eos(eos)
    f = np.zeros(5)
    ss = C.c_double()
    _chk(lib().emgo_riemann_flux(C.byref(e), dptr(arr(wl)), dptr(arr(wr)), d, dptr(f), C.byref(ss)))
    return f, ss.value


def to_prim(eos, u):
    e = c_eos(eos)
    w = np.zeros(5)
    _chk(lib().emgo_to_prim(C.byref(e), dptr(arr(u)), dptr(w)))
    return w


def to_cons(eos, w):
    e = c_eos(eos)
    u = np.zeros(5)
    _chk(lib().emgo_to_cons(C.byref(e), dptr(arr(w)), dptr(u)))
    return u


def eigen(eos, w, d):
    e = c_eos(eos)
    l, r = np.zeros(25), np.zeros(25)
    _chk(lib().emgo_eigen(C.byref(e), dptr(arr(w)), d, dptr(l), dptr(r)))
    return l.reshape(5, 5), r.reshape(5, 5)


def max_speed(eos, w, d):
    e = c_eos(eos)
    s = C.c_double()
    _chk(lib().emgo_max_speed(C.byref(e), dptr(arr(w)), d, C.byref(s)))
    return s.value


def admissible(eos, w):
    e = c_eos(eos)
    return bool(lib().emgo_admissible(C.byref(e), dptr(arr(w))))


def characteristic_ghost_layer(eos, u_b, u_b1, u_far, d, side, m):
    e = c_eos(eos)
    out = np.zeros(5)
    _chk(lib().emgo_characteristic_ghost_layer(C.byref(e), dptr(arr(u_b)), dptr(arr(u_b1)), dptr(arr(u_far)), d, side,
                                               float(m), dptr(out)))
    return out


def weno5z_interp(v0, v1, v2, v3, v4):
    o = C.c_double()
    _chk(lib().emgo_weno5z_interp(v0, v1, v2, v3, v4, C.byref(o)))
    return o.value


def exact_star(left, right, eos_l, eos_r=None):
    eos_r = eos_r or eos_l
    out = np.zeros(4)
    el, er = c_eos(eos_l), c_eos(eos_r)
    _chk(lib().emgo_exact_star(dptr(arr(left)), dptr(arr(right)), C.byref(el), C.byref(er), dptr(out)))
    return out  # p*, u*, rho*_L, rho*_R


def exact_sample(left, right, xi, eos_l, eos_r=None):
    eos_r = eos_r or eos_l
    xi = arr(xi)
    out = np.zeros((xi.size, 3))
    el, er = c_eos(eos_l), c_eos(eos_r)
    _chk(lib().emgo_exact_sample(dptr(arr(left)), dptr(arr(right)), C.byref(el), C.byref(er), dptr(xi), xi.size,
                                 dptr(out)))
    return out  # rho, u, p per xi


def state_hash(mesh, u):
    """The hash of fluid/crates/compressible/examples/cpu_validate.rs:7-22 over
    the interior cells of a ghost-padded AoS state."""
    from emergence_b200.solver import _c_mesh
    u = np.ascontiguousarray(u, dtype=np.float64)
    out = C.c_uint64()
    _chk(lib().emgo_state_hash(C.byref(_c_mesh(mesh)), dptr(u), mesh.len(), C.byref(out)))
    return out.value


# ---- block AMR (amr_oracle.hpp)
from emergence_b200._abi import EmgAmrConfig, INIT_FN  # noqa: E402

SIGS_AMR = {
    "emgo_amr_create": (C.c_int, [C.POINTER(EmgAmrConfig), C.POINTER(EmgEos), _D, _D, C.POINTER(EmgBc),
                                  C.POINTER(EmgOpts), INIT_FN, C.c_void_p, C.POINTER(_P)]),
    "emgo_amr_destroy": (C.c_int, [_P]),
    "emgo_amr_step": (C.c_int, [_P, C.c_double]),
    "emgo_amr_step_subcycled": (C.c_int, [_P, C.c_double]),
    "emgo_amr_dt_cfl_subcycled": (C.c_int, [_P, _D]),
    "emgo_amr_dt_cfl": (C.c_int, [_P, _D]),
    "emgo_amr_run_to": (C.c_int, [_P, C.c_double, _U64]),
    "emgo_amr_regrid": (C.c_int, [_P]),
    "emgo_amr_block_count": (C.c_int, [_P, _U64, _U64]),
    "emgo_amr_structure": (C.c_int, [_P, C.POINTER(C.c_int64), C.c_size_t]),
    "emgo_amr_download": (C.c_int, [_P, _D, C.c_size_t]),
    "emgo_amr_totals": (C.c_int, [_P, _D]),
    "emgo_amr_counters": (C.c_int, [_P, _U64]),
    "emgo_amr_get_time": (C.c_int, [_P, _D]),
    "emgo_amr_steps": (C.c_int, [_P, _U64]),
    "emgo_amr_details": (C.c_int, [_P, _D, C.c_size_t]),
    "emgo_amr_sample": (C.c_int, [_P, C.c_int64, C.POINTER(C.c_int64), C.c_size_t, _D]),
    "emgo_amr_nv": (C.c_int, [_P, C.POINTER(C.c_int)]),
}


def _amr_lib():
    L = lib()
    if not getattr(L, "_amr_ready", False):
        from emergence_b200._abi import EmgBc7, EmgFiveSystem
        sigs = dict(SIGS_AMR)
        sigs["emgo_amr_five_create"] = (C.c_int, [C.POINTER(EmgAmrConfig), C.POINTER(EmgFiveSystem), _D, _D,
                                                  C.POINTER(EmgBc7), C.POINTER(EmgOpts), INIT_FN, C.c_void_p,
                                                  C.POINTER(_P)])
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        L._amr_ready = True
    return L


def make_init(fn, nv=5):
    """Wrap a numpy init(x[n,3]) -> w[n,nv] (primitives) as the C callback type."""
    def cb(ctx, x, n, w):
        xa = np.ctypeslib.as_array(x, shape=(n, 3)).copy()
        wa = np.ctypeslib.as_array(w, shape=(n, nv))
        wa[...] = fn(xa)
    return INIT_FN(cb)


def c_amr_config(cfg):
    c = EmgAmrConfig()
    c.b, c.levels, c.eps, c.regrid_every, c.ghosts = cfg["b"], cfg["levels"], cfg["eps"], cfg["regrid_every"], cfg["ghosts"]
    for d in range(3):
        c.base_blocks[d] = cfg["base_blocks"][d]
    return c


class OracleAmr:
    """C++ restatement of ``compressible::amr::Amr`` (global and subcycled
    steps) for the Euler system or, when ``sys`` is a FiveEq, the
    five-equation system (7 variables; ``init`` gives 7 primitives)."""

    def __init__(self, sys, cfg, lo, hi, bc, init, cfl=0.4, mode=FluxMode.Hybrid, tol=1e-3, positivity=True,
                 subcycle=False):
        L = _amr_lib()
        self.cfg = dict(cfg)
        self._c = c_amr_config(cfg)
        self._o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, 0, 2 if subcycle else 0)
        lo_, hi_ = arr(lo), arr(hi)
        h = C.c_void_p()
        from emergence_b200.five import FiveEq
        if isinstance(sys, FiveEq):
            from emergence_b200.five import _c_bcs7, _c_system
            self.nv = 7
            self._e = _c_system(sys)
            self._b = _c_bcs7(bc)
            self._cb = make_init(init, 7)
            _chk(L.emgo_amr_five_create(C.byref(self._c), C.byref(self._e), dptr(lo_), dptr(hi_), self._b,
                                        C.byref(self._o), self._cb, None, C.byref(h)))
        else:
            from emergence_b200.solver import _c_bcs
            self.nv = 5
            self._e = c_eos(sys.eos)
            self._b = _c_bcs(bc)
            self._cb = make_init(init)
            _chk(L.emgo_amr_create(C.byref(self._c), C.byref(self._e), dptr(lo_), dptr(hi_), self._b,
                                   C.byref(self._o), self._cb, None, C.byref(h)))
        self._h = h
        self.bcells = 1
        for d in range(3):
            self.bcells *= cfg["b"] if cfg["base_blocks"][d] > 0 else 1

    def close(self):
        if getattr(self, "_h", None):
            _amr_lib().emgo_amr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt):
        _chk(_amr_lib().emgo_amr_step(self._h, float(dt)))

    def dt_cfl(self):
        v = C.c_double()
        _chk(_amr_lib().emgo_amr_dt_cfl(self._h, C.byref(v)))
        return v.value

    def step_subcycled(self, dt):
        _chk(_amr_lib().emgo_amr_step_subcycled(self._h, float(dt)))

    def dt_cfl_subcycled(self):
        v = C.c_double()
        _chk(_amr_lib().emgo_amr_dt_cfl_subcycled(self._h, C.byref(v)))
        return v.value

    def run_to(self, t_end):
        n = C.c_uint64()
        _chk(_amr_lib().emgo_amr_run_to(self._h, float(t_end), C.byref(n)))
        return n.value

    def regrid(self):
        _chk(_amr_lib().emgo_amr_regrid(self._h))

    def block_count(self):
        b, l = C.c_uint64(), C.c_uint64()
        _chk(_amr_lib().emgo_amr_block_count(self._h, C.byref(b), C.byref(l)))
        return b.value, l.value

    def structure(self):
        nb, _ = self.block_count()
        out = np.zeros((nb, 5), dtype=np.int64)
        _chk(_amr_lib().emgo_amr_structure(self._h, out.ctypes.data_as(C.POINTER(C.c_int64)), nb))
        return out

    def download(self):
        nb, _ = self.block_count()
        out = np.zeros((nb, self.bcells, self.nv))
        _chk(_amr_lib().emgo_amr_download(self._h, dptr(out), nb))
        return out

    def totals(self):
        out = np.zeros(self.nv)
        _chk(_amr_lib().emgo_amr_totals(self._h, dptr(out)))
        return out

    def counters(self):
        out = (C.c_uint64 * 4)()
        _chk(_amr_lib().emgo_amr_counters(self._h, out))
        return list(out)

    def details(self):
        nb, _ = self.block_count()
        out = np.zeros(nb)
        _chk(_amr_lib().emgo_amr_details(self._h, dptr(out), nb))
        return out

    def sample(self, level, g):
        """Conserved states at level-``level`` cell coordinates g (int [n, 3]):
        the covering leaf's data or its prediction (Amr::sample)."""
        g = np.ascontiguousarray(g, dtype=np.int64).reshape(-1, 3)
        out = np.zeros((len(g), self.nv))
        _chk(_amr_lib().emgo_amr_sample(self._h, int(level), g.ctypes.data_as(C.POINTER(C.c_int64)), len(g), dptr(out)))
        return out

    @property
    def t(self):
        v = C.c_double()
        _chk(_amr_lib().emgo_amr_get_time(self._h, C.byref(v)))
        return v.value

    @property
    def steps(self):
        v = C.c_uint64()
        _chk(_amr_lib().emgo_amr_steps(self._h, C.byref(v)))
        return v.value


class FiveOracleSolver:
    """C++ restatement of ``compressible::Solver<7, FiveEq>`` (five_oracle.hpp),
    with the constructor and methods of ``emergence_b200.GpuFiveSolver``."""

    def __init__(self, sys, mesh, u, bc=None, cfl=0.5, mode=FluxMode.Weno, tol=1e-3, positivity=True):
        from emergence_b200.five import _c_bcs7, _c_system
        from emergence_b200.solver import _c_mesh
        self.sys, self.mesh = sys, mesh
        self.bc = bc if bc is not None else [[Bc.Periodic, Bc.Periodic] for _ in range(3)]
        u = arr(u)
        self._m = _c_mesh(mesh)
        self._s = _c_system(sys)
        self._b = _c_bcs7(self.bc)
        self._o = EmgOpts(cfl, tol, mode, 1 if positivity else 0, 0, 0)
        h = C.c_void_p()
        _chk(lib().emgo_five_create(C.byref(self._m), C.byref(self._s), self._b, C.byref(self._o), dptr(u),
                                    mesh.len(), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().emgo_five_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt):
        _chk(lib().emgo_five_step(self._h, float(dt)))

    def dt_cfl(self):
        v = C.c_double()
        _chk(lib().emgo_five_dt_cfl(self._h, C.byref(v)))
        return v.value

    def run_to(self, t_end):
        n = C.c_uint64()
        _chk(lib().emgo_five_run_to(self._h, float(t_end), C.byref(n)))
        return n.value

    def download(self):
        out = np.empty((self.mesh.len(), 7))
        _chk(lib().emgo_five_download(self._h, dptr(out), self.mesh.len()))
        return out

    def fill_ghosts(self):
        _chk(lib().emgo_five_fill_ghosts(self._h))

    def totals(self):
        out = np.empty(7)
        _chk(lib().emgo_five_totals(self._h, dptr(out)))
        return out

    def counters(self):
        out = (C.c_uint64 * 4)()
        _chk(lib().emgo_five_counters(self._h, out))
        return list(out)

    @property
    def t(self):
        v = C.c_double()
        _chk(lib().emgo_five_get_time(self._h, C.byref(v)))
        return v.value


def five_props(sys, w, divu=0.0):
    """(sound speed, dilatation rate, admissible, Kapila K) of one primitive state."""
    from emergence_b200.five import _c_system
    s = _c_system(sys)
    out = np.empty(4)
    _chk(lib().emgo_five_props(C.byref(s), dptr(arr(w)), float(divu), dptr(out)))
    return out
