// CPU ORACLE — test infrastructure only (see oracle.hpp).
//
// C entry points over the C++ restatement of the reference CPU solver, with
// the same argument types as the product ABI in include/emergence_b200.h, so
// the tests drive the oracle and the CUDA library through identical calls.
// Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU leg.
#include "oracle.hpp"
#include "amr_oracle.hpp"
#include "dual.hpp"
#include "five_oracle.hpp"
#include "../include/emergence_b200.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <type_traits>
#include <string>

using namespace oracle;

namespace {
thread_local std::string g_err;
int fail(int code, const char* msg) {
    g_err = msg;
    return code;
}
struct Handle {
    Solver<double> s;
    Handle(const Euler<double>& sys, const Mesh& m) : s(sys, m) {}
};
Mesh to_mesh(const emg_mesh* m) {
    Mesh r;
    for (int d = 0; d < 3; d++) {
        r.n[d] = m->n[d];
        r.lo[d] = m->lo[d];
        r.dx[d] = m->dx[d];
    }
    r.ng = m->ng;
    return r;
}
Euler<double> to_sys(const emg_eos* e) { return Euler<double>{Nasg<double>{e->gamma, e->p_inf, e->b, e->q, e->cv}}; }
}  // namespace

extern "C" {

const char* emgo_last_error(void) { return g_err.c_str(); }

// fluid/crates/compressible/examples/cpu_validate.rs:7-22: FNV-style hash of
// the interior conserved state, cells in (i, j, k) order, each value's bits
// folded in whole.
int emgo_state_hash(const emg_mesh* mesh, const double* u_aos, size_t len, uint64_t* out) {
    if (!mesh || !u_aos || !out) return fail(1, "null argument");
    const Mesh m = to_mesh(mesh);
    if ((size_t)m.len() != len) return fail(1, "state length does not match the padded mesh");
    uint64_t h = 0xcbf29ce484222325ull;
    for (int64_t i = 0; i < m.n[0]; i++)
        for (int64_t j = 0; j < m.n[1]; j++)
            for (int64_t k = 0; k < m.n[2]; k++) {
                const size_t q = (size_t)m.idx(i + m.g(0), j + m.g(1), k + m.g(2));
                for (int f = 0; f < 5; f++) {
                    uint64_t bits;
                    std::memcpy(&bits, u_aos + 5 * q + f, sizeof bits);
                    h = (h ^ bits) * 0x100000001b3ull;
                }
            }
    *out = h;
    return 0;
}

int emgo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void emgo_set_num_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int emgo_uniform_create(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                        const double* u_aos, size_t len, void** out) {
    if (!mesh || !eos || !bc || !opts || !u_aos || !out) return fail(EMG_ERR_INVALID, "null argument");
    Mesh m = to_mesh(mesh);
    if ((size_t)m.len() != len) return fail(EMG_ERR_INVALID, "state length does not match the padded mesh");
    Handle* h = new Handle(to_sys(eos), m);
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++) {
            h->s.bc[d][s].kind = bc[2 * d + s].kind;
            for (int k = 0; k < 5; k++) h->s.bc[d][s].state[k] = bc[2 * d + s].state[k];
        }
    h->s.cfl = opts->cfl;
    h->s.tol = opts->tol;
    h->s.mode = opts->mode;
    h->s.positivity = opts->positivity != 0;
    std::memcpy(h->s.u.data(), u_aos, len * 5 * sizeof(double));
    *out = h;
    return EMG_OK;
}
int emgo_uniform_destroy(void* h) {
    delete (Handle*)h;
    return EMG_OK;
}
int emgo_uniform_step(void* h, double dt) {
    ((Handle*)h)->s.step(dt);
    return EMG_OK;
}
int emgo_uniform_dt_cfl(void* h, double* dt) {
    *dt = ((Handle*)h)->s.dt_cfl();
    return EMG_OK;
}
int emgo_uniform_run_to(void* h, double t_end, uint64_t* steps) {
    int64_t n = ((Handle*)h)->s.run_to(t_end);
    if (n < 0) return fail(EMG_ERR_DT_COLLAPSED, "time step collapsed");
    if (steps) *steps = (uint64_t)n;
    return EMG_OK;
}
int emgo_uniform_download(void* h, double* u_aos, size_t len) {
    Handle* hh = (Handle*)h;
    if (len != hh->s.u.size()) return fail(EMG_ERR_INVALID, "length mismatch");
    std::memcpy(u_aos, hh->s.u.data(), len * 5 * sizeof(double));
    return EMG_OK;
}
int emgo_uniform_upload(void* h, const double* u_aos, size_t len) {
    Handle* hh = (Handle*)h;
    if (len != hh->s.u.size()) return fail(EMG_ERR_INVALID, "length mismatch");
    std::memcpy(hh->s.u.data(), u_aos, len * 5 * sizeof(double));
    return EMG_OK;
}
int emgo_uniform_totals(void* h, double out[5]) {
    V5<double> t = ((Handle*)h)->s.totals();
    for (int k = 0; k < 5; k++) out[k] = t[k];
    return EMG_OK;
}
int emgo_uniform_counters(void* h, uint64_t out[4]) {
    Stats& s = ((Handle*)h)->s.stats;
    out[0] = s.faces;
    out[1] = s.weno_faces;
    out[2] = s.fallback_faces;
    out[3] = s.limited_faces;
    return EMG_OK;
}
int emgo_uniform_get_time(void* h, double* t) {
    *t = ((Handle*)h)->s.t;
    return EMG_OK;
}
int emgo_uniform_set_time(void* h, double t) {
    ((Handle*)h)->s.t = t;
    return EMG_OK;
}
// Ghost fill of the handle's own state (C/solver.rs:252-348).
int emgo_uniform_fill_ghosts(void* h) {
    Handle* hh = (Handle*)h;
    hh->s.fill_ghosts(hh->s.u);
    return EMG_OK;
}
// Ghost fill of a caller array with the handle's mesh and boundary conditions.
int emgo_uniform_fill_ghosts_of(void* h, double* u_aos, size_t len) {
    Handle* hh = (Handle*)h;
    if (len != hh->s.u.size()) return fail(EMG_ERR_INVALID, "length mismatch");
    std::vector<V5<double>> tmp(len);
    std::memcpy(tmp.data(), u_aos, len * 5 * sizeof(double));
    hh->s.fill_ghosts(tmp);
    std::memcpy(u_aos, tmp.data(), len * 5 * sizeof(double));
    return EMG_OK;
}

// ---- unit-level entry points (scheme / boundary / physics)

// Face fluxes of one line of primitive states (C/scheme.rs:132-281).
int emgo_line_fluxes(const emg_eos* eos, const double* w, int len, int d, int ng, int mode, double tol, double lambda,
                     double* out, double* uface, uint64_t stats[4]) {
    Euler<double> sys = to_sys(eos);
    SchemeOpts o{mode, tol, lambda};
    Stats s;
    line_fluxes(sys, (const V5<double>*)w, len, d, ng, o, (V5<double>*)out, uface, s);
    stats[0] = s.faces;
    stats[1] = s.weno_faces;
    stats[2] = s.fallback_faces;
    stats[3] = s.limited_faces;
    return EMG_OK;
}

// Positivity limiter on given face fluxes (C/scheme.rs:395-464).
int emgo_positivity_limit(const emg_eos* eos, const double* w, int len, int d, int ng, double lambda, double* out,
                          double* uface, uint64_t* limited) {
    Euler<double> sys = to_sys(eos);
    Stats s;
    positivity_limit(sys, (const V5<double>*)w, len, d, ng, lambda, (V5<double>*)out, uface, s);
    *limited = s.limited_faces;
    return EMG_OK;
}

// Midpoint flux between cells j and j+1 of a primitive line (C/scheme.rs:286-333).
int emgo_midpoint_flux(const emg_eos* eos, const double* w, int j, int d, double f[5], double* us, int* fb) {
    Euler<double> sys = to_sys(eos);
    MidResult<double> m = midpoint_flux(sys, (const V5<double>*)w, j, d);
    for (int k = 0; k < 5; k++) f[k] = m.f[k];
    *us = m.us;
    *fb = m.fb;
    return EMG_OK;
}

// HLLC flux (C/system.rs:260-312).
int emgo_riemann_flux(const emg_eos* eos, const double wl[5], const double wr[5], int d, double f[5], double* ss) {
    Euler<double> sys = to_sys(eos);
    V5<double> a, b;
    for (int k = 0; k < 5; k++) {
        a[k] = wl[k];
        b[k] = wr[k];
    }
    V5<double> r = sys.riemann_flux(a, b, d, ss);
    for (int k = 0; k < 5; k++) f[k] = r[k];
    return EMG_OK;
}

int emgo_weno5z_interp(double v0, double v1, double v2, double v3, double v4, double* out) {
    *out = weno5z_interp(v0, v1, v2, v3, v4);
    return EMG_OK;
}

int emgo_to_prim(const emg_eos* eos, const double u[5], double w[5]) {
    Euler<double> sys = to_sys(eos);
    V5<double> a;
    for (int k = 0; k < 5; k++) a[k] = u[k];
    V5<double> r = sys.to_prim(a);
    for (int k = 0; k < 5; k++) w[k] = r[k];
    return EMG_OK;
}
int emgo_to_cons(const emg_eos* eos, const double w[5], double u[5]) {
    Euler<double> sys = to_sys(eos);
    V5<double> a;
    for (int k = 0; k < 5; k++) a[k] = w[k];
    V5<double> r = sys.to_cons(a);
    for (int k = 0; k < 5; k++) u[k] = r[k];
    return EMG_OK;
}
int emgo_eigen(const emg_eos* eos, const double w[5], int d, double l[25], double r[25]) {
    Euler<double> sys = to_sys(eos);
    V5<double> a;
    for (int k = 0; k < 5; k++) a[k] = w[k];
    Mat5<double> L, R;
    sys.eigen(a, d, L, R);
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) {
            l[5 * i + j] = L[i][j];
            r[5 * i + j] = R[i][j];
        }
    return EMG_OK;
}
int emgo_max_speed(const emg_eos* eos, const double w[5], int d, double* s) {
    Euler<double> sys = to_sys(eos);
    V5<double> a;
    for (int k = 0; k < 5; k++) a[k] = w[k];
    *s = sys.max_speed(a, d);
    return EMG_OK;
}
int emgo_admissible(const emg_eos* eos, const double w[5]) {
    Euler<double> sys = to_sys(eos);
    V5<double> a;
    for (int k = 0; k < 5; k++) a[k] = w[k];
    return sys.admissible(a) ? 1 : 0;
}

// Characteristic ghost layer (C/boundary.rs:34-44).
int emgo_characteristic_ghost_layer(const emg_eos* eos, const double u_b[5], const double u_b1[5],
                                    const double u_far[5], int d, int side, double m, double out[5]) {
    Euler<double> sys = to_sys(eos);
    V5<double> a, b, c;
    for (int k = 0; k < 5; k++) {
        a[k] = u_b[k];
        b[k] = u_b1[k];
        c[k] = u_far[k];
    }
    V5<double> r = characteristic_ghost_layer(sys, a, b, c, d, side, m);
    for (int k = 0; k < 5; k++) out[k] = r[k];
    return EMG_OK;
}

// Exact Riemann star state and sampling (C/exact.rs:45-109).
int emgo_exact_star(const double l[3], const double r[3], const emg_eos* eos_l, const emg_eos* eos_r, double out[4]) {
    Side L{l[0], l[1], l[2], Nasg<double>{eos_l->gamma, eos_l->p_inf, eos_l->b, eos_l->q, eos_l->cv}};
    Side R{r[0], r[1], r[2], Nasg<double>{eos_r->gamma, eos_r->p_inf, eos_r->b, eos_r->q, eos_r->cv}};
    Star s = star(L, R);
    out[0] = s.p;
    out[1] = s.u;
    out[2] = s.rho_l;
    out[3] = s.rho_r;
    return EMG_OK;
}
int emgo_exact_sample(const double l[3], const double r[3], const emg_eos* eos_l, const emg_eos* eos_r,
                      const double* xi, size_t n, double* out) {
    Side L{l[0], l[1], l[2], Nasg<double>{eos_l->gamma, eos_l->p_inf, eos_l->b, eos_l->q, eos_l->cv}};
    Side R{r[0], r[1], r[2], Nasg<double>{eos_r->gamma, eos_r->p_inf, eos_r->b, eos_r->q, eos_r->cv}};
    Star s = star(L, R);
    for (size_t i = 0; i < n; i++) sample(L, R, s, xi[i], out + 3 * i);
    return EMG_OK;
}


// ---- block AMR (amr_oracle.hpp)
namespace {
InitFn wrap_init(emg_init_fn f, void* ctx) {
    return [f, ctx](const double* x, int64_t n, double* w) { f(ctx, x, n, w); };
}
AmrConfig to_cfg(const emg_amr_config* c) {
    AmrConfig r;
    r.b = c->b;
    r.levels = c->levels;
    r.eps = c->eps;
    r.regrid_every = c->regrid_every;
    for (int d = 0; d < 3; d++) r.base_blocks[d] = c->base_blocks[d];
    r.ghosts = c->ghosts;
    return r;
}
}  // namespace

}  // extern "C"

// An oracle hierarchy of either system: Euler (5 variables) or the
// five-equation model (7 variables).
struct AmrHandle {
    int nv = 5;
    std::unique_ptr<Amr> e;
    std::unique_ptr<AmrFiveEq> f;
    template <class Fn> auto with(Fn fn) { return nv == 5 ? fn(*e) : fn(*f); }
};
static AmrHandle* H(void* h) { return (AmrHandle*)h; }

template <class A> static void amr_opts(A& a, const emg_opts* opts) {
    a.cfl = opts->cfl;
    a.tol = opts->tol;
    a.mode = opts->mode;
    a.positivity = opts->positivity != 0;
    a.subcycle = (opts->flags & EMG_OPT_SUBCYCLE) != 0;
}

extern "C" {

int emgo_amr_create(const emg_amr_config* cfg, const emg_eos* eos, const double lo[3], const double hi[3],
                    const emg_bc bc[6], const emg_opts* opts, emg_init_fn init, void* ctx, void** out) {
    if (!cfg || !eos || !lo || !hi || !bc || !opts || !init || !out) return fail(EMG_ERR_INVALID, "null argument");
    Bc<double> b[3][2];
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++) {
            b[d][s].kind = bc[2 * d + s].kind;
            for (int k = 0; k < 5; k++) b[d][s].state[k] = bc[2 * d + s].state[k];
        }
    AmrHandle* h = new AmrHandle();
    h->e.reset(new Amr(to_sys(eos), to_cfg(cfg), lo, hi, b, wrap_init(init, ctx)));
    amr_opts(*h->e, opts);
    *out = h;
    return EMG_OK;
}
// the five-equation system on the block hierarchy; init fills 7 primitives per cell
int emgo_amr_five_create(const emg_amr_config* cfg, const emg_five_system* sys, const double lo[3], const double hi[3],
                         const emg_bc7 bc[6], const emg_opts* opts, emg_init_fn init, void* ctx, void** out) {
    if (!cfg || !sys || !lo || !hi || !bc || !opts || !init || !out) return fail(EMG_ERR_INVALID, "null argument");
    FiveEq<double> f;
    for (int k = 0; k < 2; k++)
        f.eos[k] = Nasg<double>{sys->eos[k].gamma, sys->eos[k].p_inf, sys->eos[k].b, sys->eos[k].q, sys->eos[k].cv};
    f.kapila = sys->kapila != 0;
    Bc7<double> b[3][2];
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++) {
            b[d][s].kind = bc[2 * d + s].kind;
            for (int k = 0; k < 7; k++) b[d][s].state[k] = bc[2 * d + s].state[k];
        }
    AmrHandle* h = new AmrHandle();
    h->nv = 7;
    h->f.reset(new AmrFiveEq(f, to_cfg(cfg), lo, hi, b, wrap_init(init, ctx)));
    amr_opts(*h->f, opts);
    *out = h;
    return EMG_OK;
}
int emgo_amr_step_subcycled(void* h, double dt) {
    H(h)->with([&](auto& a) { a.step_subcycled(dt); });
    return EMG_OK;
}
int emgo_amr_dt_cfl_subcycled(void* h, double* dt) {
    *dt = H(h)->with([&](auto& a) { return a.dt_cfl_subcycled(); });
    return EMG_OK;
}
int emgo_amr_destroy(void* h) {
    delete H(h);
    return EMG_OK;
}
int emgo_amr_step(void* h, double dt) {
    H(h)->with([&](auto& a) { a.step(dt); });
    return EMG_OK;
}
int emgo_amr_dt_cfl(void* h, double* dt) {
    *dt = H(h)->with([&](auto& a) { return a.dt_cfl(); });
    return EMG_OK;
}
int emgo_amr_run_to(void* h, double t_end, uint64_t* steps) {
    int64_t n = H(h)->with([&](auto& a) { return a.run_to(t_end); });
    if (n < 0) return fail(EMG_ERR_DT_COLLAPSED, "time step collapsed");
    if (steps) *steps = (uint64_t)n;
    return EMG_OK;
}
int emgo_amr_regrid(void* h) {
    H(h)->with([&](auto& a) { a.regrid(); });
    return EMG_OK;
}
int emgo_amr_nv(void* h, int* nv) {
    *nv = H(h)->nv;
    return EMG_OK;
}
int emgo_amr_block_count(void* h, uint64_t* blocks, uint64_t* leaves) {
    return H(h)->with([&](auto& a) {
        if (blocks) *blocks = a.blocks.size();
        if (leaves) *leaves = (uint64_t)a.leaf_count();
        return (int)EMG_OK;
    });
}
int emgo_amr_structure(void* h, int64_t* desc, size_t cap) {
    return H(h)->with([&](auto& a) {
        if (cap < a.blocks.size()) return fail(EMG_ERR_INVALID, "structure buffer too small");
        for (size_t i = 0; i < a.blocks.size(); i++) {
            desc[5 * i] = a.blocks[i].level;
            for (int d = 0; d < 3; d++) desc[5 * i + 1 + d] = a.blocks[i].idx[d];
            desc[5 * i + 4] = a.blocks[i].leaf ? 1 : 0;
        }
        return (int)EMG_OK;
    });
}
// block data u[id][cell][nv]
int emgo_amr_download(void* h, double* u, size_t nblocks) {
    return H(h)->with([&](auto& a) {
        using A = std::decay_t<decltype(a)>;
        if (nblocks < a.blocks.size()) return fail(EMG_ERR_INVALID, "buffer too small");
        size_t bc_ = (size_t)a.bcells();
        for (size_t i = 0; i < a.blocks.size(); i++)
            std::memcpy(u + i * bc_ * A::N, a.blocks[i].u.data(), bc_ * A::N * sizeof(double));
        return (int)EMG_OK;
    });
}
int emgo_amr_totals(void* h, double* out) {
    H(h)->with([&](auto& a) {
        auto t = a.totals();
        for (size_t k = 0; k < t.size(); k++) out[k] = t[k];
    });
    return EMG_OK;
}
int emgo_amr_counters(void* h, uint64_t out[4]) {
    H(h)->with([&](auto& a) {
        Stats& s = a.stats;
        out[0] = s.faces;
        out[1] = s.weno_faces;
        out[2] = s.fallback_faces;
        out[3] = s.limited_faces;
    });
    return EMG_OK;
}
int emgo_amr_get_time(void* h, double* t) {
    *t = H(h)->with([&](auto& a) { return a.t; });
    return EMG_OK;
}
int emgo_amr_steps(void* h, uint64_t* s) {
    *s = H(h)->with([&](auto& a) { return (uint64_t)a.steps; });
    return EMG_OK;
}
// per-leaf wavelet details in block id order (ancestors 0), C/amr.rs:823-867
int emgo_amr_details(void* h, double* out, size_t cap) {
    return H(h)->with([&](auto& a) {
        if (cap < a.blocks.size()) return fail(EMG_ERR_INVALID, "buffer too small");
        a.restrict_all();
        std::vector<double> d = a.details();
        for (size_t i = 0; i < d.size(); i++) out[i] = d[i];
        return (int)EMG_OK;
    });
}

// conserved state at level-l cell coordinates g[3*i..] (Amr::sample, amr.rs:384-439):
// the covering block's data, or the prediction from coarser levels; nv values per cell
int emgo_amr_sample(void* h, int64_t l, const int64_t* g, size_t n, double* out) {
    return H(h)->with([&](auto& a) {
        using A = std::decay_t<decltype(a)>;
        if (l < 0 || l >= a.cfg.levels) return fail(EMG_ERR_INVALID, "level out of range");
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < (int64_t)n; i++) {
            auto v = a.sample(l, {g[3 * i], g[3 * i + 1], g[3 * i + 2]});
            for (int q = 0; q < A::N; q++) out[A::N * i + q] = v[q];
        }
        return (int)EMG_OK;
    });
}

}  // extern "C"

// ---- forward-mode derivative of a frozen-dt run (dual-number instantiation)

namespace {
// Objective over the interior cells whose centre lo + (i+½)dx lies in
// [box_lo, box_hi] on every active axis: kind 0 = Σ p·vol, kind 1 = Σ E·vol.
template <class T>
T box_objective(const Solver<T>& s, int kind, const double* box_lo, const double* box_hi) {
    const Mesh& m = s.mesh;
    T vol = T(1.0);
    for (int d = 0; d < 3; d++)
        if (m.active(d)) vol = vol * T(m.dx[d]);
    T acc = T(0.0);
    for (int64_t i = 0; i < m.n[0]; i++)
        for (int64_t j = 0; j < m.n[1]; j++)
            for (int64_t k = 0; k < m.n[2]; k++) {
                const int64_t ijk[3] = {i, j, k};
                bool in = true;
                for (int d = 0; d < 3; d++) {
                    if (!m.active(d)) continue;
                    const double x = m.lo[d] + ((double)ijk[d] + 0.5) * m.dx[d];
                    in = in && x >= box_lo[d] && x <= box_hi[d];
                }
                if (!in) continue;
                const V5<T>& u = s.u[m.idx(i + m.g(0), j + m.g(1), k + m.g(2))];
                T v = kind == 0 ? s.sys.to_prim(u)[4] : u[4];
                acc = acc + v * vol;
            }
    return acc;
}
}  // namespace

extern "C" {

// Runs `nsteps` SSP-RK3 steps with the given time steps from the initial
// primitive state w0 (padded AoS, ghosts ignored) in dual numbers, with the
// tangent dw0 on the initial primitives and dgamma on γ; returns the box
// objective J and its directional derivative dJ. Optional u_out / du_out
// receive the final conserved state and its tangent (padded AoS).
int emgo_dual_run(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                  const double* w0, const double* dw0, size_t len, double dgamma, const double* dts, size_t nsteps,
                  int objective, const double box_lo[3], const double box_hi[3], double* J, double* dJ,
                  double* u_out, double* du_out) {
    if (!mesh || !eos || !bc || !opts || !w0 || !dw0 || (nsteps && !dts) || !J || !dJ)
        return fail(EMG_ERR_INVALID, "null argument");
    Mesh m = to_mesh(mesh);
    if ((size_t)m.len() != len) return fail(EMG_ERR_INVALID, "state length does not match the padded mesh");
    Euler<Dual> sys{Nasg<Dual>{Dual(eos->gamma, dgamma), Dual(eos->p_inf), Dual(eos->b), Dual(eos->q), Dual(eos->cv)}};
    Solver<Dual> s(sys, m);
    for (int d = 0; d < 3; d++)
        for (int q = 0; q < 2; q++) {
            s.bc[d][q].kind = bc[2 * d + q].kind;
            for (int k = 0; k < 5; k++) s.bc[d][q].state[k] = Dual(bc[2 * d + q].state[k]);
        }
    s.cfl = opts->cfl;
    s.tol = opts->tol;
    s.mode = opts->mode;
    s.positivity = opts->positivity != 0;
    for (size_t c = 0; c < len; c++) {
        V5<Dual> w;
        for (int k = 0; k < 5; k++) w[k] = Dual(w0[5 * c + k], dw0[5 * c + k]);
        s.u[c] = sys.to_cons(w);
    }
    for (size_t n = 0; n < nsteps; n++) s.step(dts[n]);
    Dual j = box_objective(s, objective, box_lo, box_hi);
    *J = j.v;
    *dJ = j.d;
    if (u_out)
        for (size_t c = 0; c < len; c++)
            for (int k = 0; k < 5; k++) u_out[5 * c + k] = s.u[c][k].v;
    if (du_out)
        for (size_t c = 0; c < len; c++)
            for (int k = 0; k < 5; k++) du_out[5 * c + k] = s.u[c][k].d;
    return EMG_OK;
}

// The same objective of a plain f64 state held by a uniform oracle handle.
int emgo_box_objective(void* h, int objective, const double box_lo[3], const double box_hi[3], double* J) {
    Handle* hh = (Handle*)h;
    *J = box_objective(hh->s, objective, box_lo, box_hi);
    return EMG_OK;
}

}  // extern "C"

extern "C" {
// One SSP-RK3 step of size dt in dual numbers from the padded conserved state
// u with tangent du (and dgamma on γ); writes the new state and its tangent.
int emgo_dual_step_cons(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                        const double* u, const double* du, size_t len, double dgamma, double dt, double* u_out,
                        double* du_out) {
    Mesh m = to_mesh(mesh);
    if ((size_t)m.len() != len) return fail(EMG_ERR_INVALID, "state length does not match the padded mesh");
    Euler<Dual> sys{Nasg<Dual>{Dual(eos->gamma, dgamma), Dual(eos->p_inf), Dual(eos->b), Dual(eos->q), Dual(eos->cv)}};
    Solver<Dual> s(sys, m);
    for (int d = 0; d < 3; d++)
        for (int q = 0; q < 2; q++) {
            s.bc[d][q].kind = bc[2 * d + q].kind;
            for (int k = 0; k < 5; k++) s.bc[d][q].state[k] = Dual(bc[2 * d + q].state[k]);
        }
    s.tol = opts->tol;
    s.mode = opts->mode;
    s.positivity = opts->positivity != 0;
    for (size_t c = 0; c < len; c++)
        for (int k = 0; k < 5; k++) s.u[c][k] = Dual(u[5 * c + k], du[5 * c + k]);
    s.step(dt);
    for (size_t c = 0; c < len; c++)
        for (int k = 0; k < 5; k++) {
            u_out[5 * c + k] = s.u[c][k].v;
            du_out[5 * c + k] = s.u[c][k].d;
        }
    return EMG_OK;
}
}  // extern "C"

// ---------------------------------------------------------------- five-equation system
// (five_oracle.hpp: multiphase.rs and the system-generic step it runs)
namespace {
struct FiveHandle {
    SolverFive<double> s;
    FiveHandle(const FiveEq<double>& sys, const Mesh& m) : s(sys, m) {}
};
}  // namespace

extern "C" {
int emgo_five_create(const emg_mesh* mesh, const emg_five_system* sys, const emg_bc7 bc[6], const emg_opts* opts,
                     const double* u_aos, size_t len, void** out) {
    if (!mesh || !sys || !bc || !opts || !u_aos || !out) return fail(EMG_ERR_INVALID, "null argument");
    Mesh m = to_mesh(mesh);
    if ((size_t)m.len() != len) return fail(EMG_ERR_INVALID, "state length does not match the padded mesh");
    FiveEq<double> f;
    for (int k = 0; k < 2; k++)
        f.eos[k] = Nasg<double>{sys->eos[k].gamma, sys->eos[k].p_inf, sys->eos[k].b, sys->eos[k].q, sys->eos[k].cv};
    f.kapila = sys->kapila != 0;
    FiveHandle* h = new FiveHandle(f, m);
    for (int d = 0; d < 3; d++)
        for (int q = 0; q < 2; q++) {
            h->s.bc[d][q].kind = bc[2 * d + q].kind;
            for (int k = 0; k < 7; k++) h->s.bc[d][q].state[k] = bc[2 * d + q].state[k];
        }
    h->s.cfl = opts->cfl;
    h->s.tol = opts->tol;
    h->s.mode = opts->mode;
    h->s.positivity = opts->positivity != 0;
    std::memcpy(h->s.u.data(), u_aos, len * 7 * sizeof(double));
    *out = h;
    return EMG_OK;
}
int emgo_five_destroy(void* h) {
    delete (FiveHandle*)h;
    return EMG_OK;
}
int emgo_five_step(void* h, double dt) {
    ((FiveHandle*)h)->s.step(dt);
    return EMG_OK;
}
int emgo_five_dt_cfl(void* h, double* dt) {
    *dt = ((FiveHandle*)h)->s.dt_cfl();
    return EMG_OK;
}
// solver.rs:758-768
int emgo_five_run_to(void* h, double t_end, uint64_t* steps) {
    SolverFive<double>& s = ((FiveHandle*)h)->s;
    uint64_t n = 0;
    while (s.t < t_end - 1e-10 * std::fabs(t_end)) {
        double dt = std::fmin(s.dt_cfl(), t_end - s.t);
        if (!(std::isfinite(dt) && dt > 1e-12 * std::fmax(std::fabs(t_end), 1e-300)))
            return fail(EMG_ERR_DT_COLLAPSED, "time step collapsed");
        s.step(dt);
        n++;
    }
    if (steps) *steps = n;
    return EMG_OK;
}
int emgo_five_download(void* h, double* u_aos, size_t len) {
    FiveHandle* hh = (FiveHandle*)h;
    if (len != hh->s.u.size()) return fail(EMG_ERR_INVALID, "length mismatch");
    std::memcpy(u_aos, hh->s.u.data(), len * 7 * sizeof(double));
    return EMG_OK;
}
int emgo_five_fill_ghosts(void* h) {
    FiveHandle* hh = (FiveHandle*)h;
    hh->s.fill_ghosts(hh->s.u);
    return EMG_OK;
}
int emgo_five_totals(void* h, double out[7]) {
    V7<double> t = ((FiveHandle*)h)->s.totals();
    for (int k = 0; k < 7; k++) out[k] = t[k];
    return EMG_OK;
}
int emgo_five_counters(void* h, uint64_t out[4]) {
    Stats& s = ((FiveHandle*)h)->s.stats;
    out[0] = s.faces;
    out[1] = s.weno_faces;
    out[2] = s.fallback_faces;
    out[3] = s.limited_faces;
    return EMG_OK;
}
int emgo_five_get_time(void* h, double* t) {
    *t = ((FiveHandle*)h)->s.t;
    return EMG_OK;
}
// system-level pieces for the known-answer tests: primitive → conserved,
// conserved → primitive, sound speed, dilatation rate, admissibility
int emgo_five_to_cons(const emg_five_system* sys, const double* w, double* u) {
    FiveEq<double> f;
    for (int k = 0; k < 2; k++)
        f.eos[k] = Nasg<double>{sys->eos[k].gamma, sys->eos[k].p_inf, sys->eos[k].b, sys->eos[k].q, sys->eos[k].cv};
    f.kapila = sys->kapila != 0;
    V7<double> ww;
    for (int k = 0; k < 7; k++) ww[k] = w[k];
    V7<double> uu = f.to_cons(ww);
    for (int k = 0; k < 7; k++) u[k] = uu[k];
    return EMG_OK;
}
int emgo_five_props(const emg_five_system* sys, const double* w, double divu, double out[4]) {
    FiveEq<double> f;
    for (int k = 0; k < 2; k++)
        f.eos[k] = Nasg<double>{sys->eos[k].gamma, sys->eos[k].p_inf, sys->eos[k].b, sys->eos[k].q, sys->eos[k].cv};
    f.kapila = sys->kapila != 0;
    V7<double> ww;
    for (int k = 0; k < 7; k++) ww[k] = w[k];
    out[0] = f.sound_speed(ww);
    out[1] = f.dilatation_rate(ww, divu);
    out[2] = f.admissible(ww) ? 1.0 : 0.0;
    out[3] = f.kapila_k(ww);
    return EMG_OK;
}
}  // extern "C"
