// Test-only host build of the device adjoint functions (emergence_b200/csrc/
// adjoint.cuh, compiled here by g++ as plain host code) next to the
// dual-number instantiation of the CPU oracle, so the hand-written
// vector–Jacobian products can be checked on the CPU: for any direction dw and
// cotangent fb, <fb, J·dw> (dual numbers) must equal <J^T·fb, dw> (adjoint).
#include "../../emergence_b200/csrc/adjoint.cuh"
#include "../../oracle/oracle.hpp"
#include "../../oracle/dual.hpp"
#include "../../include/emergence_b200.h"

using oracle::Dual;
namespace {
emg::Eos<double> deos(const emg_eos* e) { return emg::Eos<double>{e->gamma, e->p_inf, e->b, e->q}; }
oracle::Euler<Dual> dsys(const emg_eos* e, double dg) {
    return oracle::Euler<Dual>{oracle::Nasg<Dual>{Dual(e->gamma, dg), Dual(e->p_inf), Dual(e->b), Dual(e->q), Dual(e->cv)}};
}
oracle::V5<Dual> dv(const double* w, const double* dw) {
    oracle::V5<Dual> r;
    for (int k = 0; k < 5; k++) r[k] = Dual(w[k], dw[k]);
    return r;
}
}  // namespace

extern "C" {

int adjh_midpoint_vjp(const emg_eos* eos, const double* w6, int d, const double* fb, double* wb6, double* gb) {
    emg::Eos<double> e = deos(eos);
    auto W = reinterpret_cast<const double(*)[5]>(w6);
    auto B = reinterpret_cast<double(*)[5]>(wb6);
    double g = 0.0;
    if (d == 0) emg::adj::midpoint_vjp<0>(e, W, fb, B, g);
    if (d == 1) emg::adj::midpoint_vjp<1>(e, W, fb, B, g);
    if (d == 2) emg::adj::midpoint_vjp<2>(e, W, fb, B, g);
    *gb = g;
    return 0;
}

// Forward-mode: the oracle's midpoint_flux in dual numbers.
int adjh_midpoint_jvp(const emg_eos* eos, const double* w6, const double* dw6, double dg, int d, double* f,
                      double* df, int* fallback) {
    auto sys = dsys(eos, dg);
    oracle::V5<Dual> w[6];
    for (int s = 0; s < 6; s++) w[s] = dv(w6 + 5 * s, dw6 + 5 * s);
    oracle::MidResult<Dual> m = oracle::midpoint_flux(sys, w, 2, d);
    for (int k = 0; k < 5; k++) {
        f[k] = m.f[k].v;
        df[k] = m.f[k].d;
    }
    *fallback = m.fb ? 1 : 0;
    return 0;
}

int adjh_hllc_vjp(const emg_eos* eos, const double* wl, const double* wr, int d, const double* fb, double* wlb,
                  double* wrb, double* gb) {
    emg::Eos<double> e = deos(eos);
    double g = 0.0;
    if (d == 0) emg::adj::hllc_vjp<1>(e, wl, wr, fb, wlb, wrb, g);
    if (d == 1) emg::adj::hllc_vjp<2>(e, wl, wr, fb, wlb, wrb, g);
    if (d == 2) emg::adj::hllc_vjp<3>(e, wl, wr, fb, wlb, wrb, g);
    *gb = g;
    return 0;
}

int adjh_hllc_jvp(const emg_eos* eos, const double* wl, const double* dwl, const double* wr, const double* dwr,
                  double dg, int d, double* f, double* df) {
    auto sys = dsys(eos, dg);
    Dual ss;
    oracle::V5<Dual> r = sys.riemann_flux(dv(wl, dwl), dv(wr, dwr), d, &ss);
    for (int k = 0; k < 5; k++) {
        f[k] = r[k].v;
        df[k] = r[k].d;
    }
    return 0;
}

int adjh_weno_grad(const double* v, double* g) {
    emg::adj::weno5z_grad(v[0], v[1], v[2], v[3], v[4], g);
    return 0;
}

int adjh_weno_jvp(const double* v, const double* dvv, double* y, double* dy) {
    Dual r = oracle::weno5z_interp(Dual(v[0], dvv[0]), Dual(v[1], dvv[1]), Dual(v[2], dvv[2]), Dual(v[3], dvv[3]),
                                   Dual(v[4], dvv[4]));
    *y = r.v;
    *dy = r.d;
    return 0;
}

int adjh_prim_vjp(const emg_eos* eos, const double* u, const double* wb, double* ub, double* gb) {
    double g = 0.0;
    for (int k = 0; k < 5; k++) ub[k] = 0.0;
    emg::adj::to_prim_vjp(deos(eos), u, wb, ub, g);
    *gb = g;
    return 0;
}

int adjh_prim_jvp(const emg_eos* eos, const double* u, const double* du, double dg, double* w, double* dw) {
    auto r = dsys(eos, dg).to_prim(dv(u, du));
    for (int k = 0; k < 5; k++) {
        w[k] = r[k].v;
        dw[k] = r[k].d;
    }
    return 0;
}

int adjh_cons_vjp(const emg_eos* eos, const double* w, const double* qb, double* wb, double* gb) {
    double g = 0.0;
    for (int k = 0; k < 5; k++) wb[k] = 0.0;
    emg::adj::to_cons_vjp(deos(eos), w, qb, wb, g);
    *gb = g;
    return 0;
}

int adjh_cons_jvp(const emg_eos* eos, const double* w, const double* dw, double dg, double* q, double* dq) {
    auto r = dsys(eos, dg).to_cons(dv(w, dw));
    for (int k = 0; k < 5; k++) {
        q[k] = r[k].v;
        dq[k] = r[k].d;
    }
    return 0;
}

// Lax–Friedrichs part (1 − θ)·F_LF of a limited face (scheme.rs:419-423).
int adjh_lf_vjp(const emg_eos* eos, const double* wi, const double* wj, int d, double theta, const double* Fb,
                double* wib, double* wjb, double* gb) {
    emg::Eos<double> e = deos(eos);
    double g = 0.0;
    for (int k = 0; k < 5; k++) wib[k] = wjb[k] = 0.0;
    if (d == 0) emg::adj::lf_vjp<0>(e, wi, wj, theta, Fb, wib, wjb, g);
    if (d == 1) emg::adj::lf_vjp<1>(e, wi, wj, theta, Fb, wib, wjb, g);
    if (d == 2) emg::adj::lf_vjp<2>(e, wi, wj, theta, Fb, wib, wjb, g);
    *gb = g;
    return 0;
}

int adjh_lf_jvp(const emg_eos* eos, const double* wi, const double* dwi, const double* wj, const double* dwj,
                double dg, int d, double theta, double* F, double* dF) {
    auto sys = dsys(eos, dg);
    auto a = dv(wi, dwi), b = dv(wj, dwj);
    auto ul = sys.to_cons(a), ur = sys.to_cons(b);
    auto fl = sys.flux(a, d), fr = sys.flux(b, d);
    Dual alpha = oracle::fmax_(sys.max_speed(a, d), sys.max_speed(b, d));
    for (int k = 0; k < 5; k++) {
        Dual flf = Dual(0.5) * (fl[k] + fr[k]) - Dual(0.5) * alpha * (ur[k] - ul[k]);
        Dual v = Dual(1.0 - theta) * flf;
        F[k] = v.v;
        dF[k] = v.d;
    }
    return 0;
}

}  // extern "C"

// ---- whole-step reverse on the CPU, built from the same device functions ----
//
// A plain-loop restatement of what adjoint.cu does on the GPU (stage recompute
// with the oracle, limiter blend weights, RK reverse, per-line sweep reverse,
// ghost reverse), so that the device adjoint's structure can be checked on
// the CPU against dual numbers.
namespace {

using V5d = oracle::V5<double>;

// Blend weight θ of every face of a line (1: untouched), following the
// oracle's positivity_limit (scheme.rs:395-464) on high-order fluxes `fh`.
void limiter_theta(const oracle::Euler<double>& sys, const V5d* w, int len, int d, int ng, double lambda,
                   const V5d* fh_all, double* theta) {
    int n = len - 2 * ng;
    for (int f = 0; f <= n; f++) {
        int i = ng - 1 + f;
        theta[f] = 1.0;
        if (!(lambda > 0.0)) continue;
        V5d ul = sys.to_cons(w[i]), ur = sys.to_cons(w[i + 1]);
        V5d fl = sys.flux(w[i], d), fr = sys.flux(w[i + 1], d);
        auto ok = [&](const V5d& fx) {
            V5d a, b;
            for (int k = 0; k < 5; k++) {
                a[k] = ul[k] - 2.0 * lambda * (fx[k] - fl[k]);
                b[k] = ur[k] + 2.0 * lambda * (fx[k] - fr[k]);
            }
            return sys.admissible(sys.to_prim(a)) && sys.admissible(sys.to_prim(b));
        };
        V5d fh = fh_all[f];
        bool fin = true;
        for (int k = 0; k < 5; k++) fin = fin && std::isfinite(fh[k]);
        if (fin && ok(fh)) continue;
        double alpha = std::fmax(sys.max_speed(w[i], d), sys.max_speed(w[i + 1], d));
        V5d flf;
        for (int k = 0; k < 5; k++) flf[k] = 0.5 * (fl[k] + fr[k]) - 0.5 * alpha * (ur[k] - ul[k]);
        double lo = 0.0, hi = 1.0;
        for (int it = 0; it < 30; it++) {
            double mid = 0.5 * (lo + hi);
            V5d v;
            for (int k = 0; k < 5; k++) v[k] = std::isfinite(fh[k]) ? mid * fh[k] + (1.0 - mid) * flf[k] : flf[k];
            if (ok(v))
                lo = mid;
            else
                hi = mid;
        }
        theta[f] = lo;
    }
}

template <int D>
void midpoint_vjp_d(const emg::Eos<double>& e, const double (*w6)[5], const double* fb, double (*wb6)[5], double& g) {
    emg::adj::midpoint_vjp<D>(e, w6, fb, wb6, g);
}
template <int D>
void lf_vjp_d(const emg::Eos<double>& e, const double* wi, const double* wj, double th, const double* fb, double* wib,
              double* wjb, double& g) {
    emg::adj::lf_vjp<D>(e, wi, wj, th, fb, wib, wjb, g);
}

struct CpuAdj {
    oracle::Solver<double>& s;
    emg::Eos<double> e;
    double lam_dt;
    // x̄ += (∂R/∂X)ᵀ(coef·ȳ), γ̄ += ...
    void sweeps(const std::vector<V5d>& X, const std::vector<V5d>& ybar, double coef, double dt, std::vector<V5d>& xbar,
                double& gb) {
        const oracle::Mesh& m = s.mesh;
        const double ndim = (double)m.ndim();
        for (int d = 0; d < 3; d++) {
            if (!m.active(d)) continue;
            int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            const int ng = (int)m.ng, n = (int)m.n[d], len = (int)m.m(d);
            const double lambda = s.positivity ? ndim * dt / m.dx[d] : 0.0;
            const double inv = 1.0 / m.dx[d];
            for (int64_t a = 0; a < m.n[e0]; a++)
                for (int64_t b = 0; b < m.n[e1]; b++) {
                    auto at = [&](int64_t c) {
                        int64_t ijk[3];
                        ijk[d] = c;
                        ijk[e0] = a + m.g(e0);
                        ijk[e1] = b + m.g(e1);
                        return m.idx(ijk[0], ijk[1], ijk[2]);
                    };
                    std::vector<V5d> w(len), fh(n + 1);
                    for (int c = 0; c < len; c++) w[c] = s.sys.to_prim(X[at(c)]);
                    oracle::Stats st;
                    oracle::SchemeOpts o{oracle::WENO, s.tol, 0.0};
                    oracle::line_fluxes(s.sys, w.data(), len, d, ng, o, fh.data(), (double*)nullptr, st);
                    std::vector<double> th(n + 1);
                    limiter_theta(s.sys, w.data(), len, d, ng, lambda, fh.data(), th.data());
                    std::vector<V5d> wb(len, V5d{0, 0, 0, 0, 0}), aft(len, V5d{0, 0, 0, 0, 0});
                    for (int f = 0; f <= n; f++) {
                        int i = ng - 1 + f;
                        double fb[5];
                        for (int k = 0; k < 5; k++) {
                            double rl = (i >= ng) ? coef * ybar[at(i)][k] : 0.0;
                            double rr = (i + 1 <= ng + n - 1) ? coef * ybar[at(i + 1)][k] : 0.0;
                            fb[k] = (rr - rl) * inv;
                        }
                        for (int k = 0; k < 5; k++) aft[i][k] = th[f] * fb[k];
                        if (th[f] < 1.0) {
                            double wib[5] = {0}, wjb[5] = {0};
                            if (d == 0) lf_vjp_d<0>(e, w[i].data(), w[i + 1].data(), th[f], fb, wib, wjb, gb);
                            if (d == 1) lf_vjp_d<1>(e, w[i].data(), w[i + 1].data(), th[f], fb, wib, wjb, gb);
                            if (d == 2) lf_vjp_d<2>(e, w[i].data(), w[i + 1].data(), th[f], fb, wib, wjb, gb);
                            for (int k = 0; k < 5; k++) {
                                wb[i][k] += wib[k];
                                wb[i + 1][k] += wjb[k];
                            }
                        }
                    }
                    for (int j = ng - 3; j <= ng + n + 1; j++) {
                        double fb[5];
                        auto A = [&](int i, int k) { return (i >= ng - 1 && i <= ng + n - 1) ? aft[i][k] : 0.0; };
                        for (int k = 0; k < 5; k++)
                            fb[k] = oracle::S6[0] * A(j, k) + oracle::S6[1] * (A(j - 1, k) + A(j + 1, k)) +
                                    oracle::S6[2] * (A(j - 2, k) + A(j + 2, k));
                        double w6[6][5], wb6[6][5] = {{0}};
                        for (int q = 0; q < 6; q++)
                            for (int k = 0; k < 5; k++) w6[q][k] = w[j - 2 + q][k];
                        if (d == 0) midpoint_vjp_d<0>(e, w6, fb, wb6, gb);
                        if (d == 1) midpoint_vjp_d<1>(e, w6, fb, wb6, gb);
                        if (d == 2) midpoint_vjp_d<2>(e, w6, fb, wb6, gb);
                        for (int q = 0; q < 6; q++)
                            for (int k = 0; k < 5; k++) wb[j - 2 + q][k] += wb6[q][k];
                    }
                    for (int c = 0; c < len; c++) {
                        double ub[5] = {0, 0, 0, 0, 0};
                        emg::adj::to_prim_vjp(e, X[at(c)].data(), wb[c].data(), ub, gb);
                        for (int k = 0; k < 5; k++) xbar[at(c)][k] += ub[k];
                    }
                }
        }
    }
    void ghosts_rev(std::vector<V5d>& xb) {
        const oracle::Mesh& m = s.mesh;
        for (int d = 2; d >= 0; d--) {
            if (!m.active(d)) continue;
            int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            int64_t n = m.n[d], ng = m.ng;
            for (int64_t a = 0; a < m.m(e0); a++)
                for (int64_t b = 0; b < m.m(e1); b++) {
                    auto at = [&](int64_t c) {
                        int64_t ijk[3];
                        ijk[d] = c;
                        ijk[e0] = a;
                        ijk[e1] = b;
                        return m.idx(ijk[0], ijk[1], ijk[2]);
                    };
                    for (int64_t gi = 0; gi < ng; gi++)
                        for (int side = 0; side < 2; side++) {
                            int kind = s.bc[d][side].kind;
                            int64_t dst = side == 0 ? at(gi) : at(n + ng + gi), src = -1;
                            if (kind == oracle::BC_OUTFLOW) src = side == 0 ? at(ng) : at(n + ng - 1);
                            if (kind == oracle::BC_PERIODIC) src = side == 0 ? at(n + gi) : at(ng + gi);
                            if (kind == oracle::BC_REFLECT) src = side == 0 ? at(2 * ng - 1 - gi) : at(n + ng - 1 - gi);
                            for (int k = 0; k < 5; k++) {
                                double v = xb[dst][k];
                                xb[dst][k] = 0.0;
                                if (src >= 0) xb[src][k] += (kind == oracle::BC_REFLECT && k == 1 + d) ? -v : v;
                            }
                        }
                }
        }
    }
};

}  // namespace

extern "C" {

// Reverse of one SSP-RK3 step of size dt from the padded AoS state u with
// output cotangent ybar; writes ubar and *gb (γ̄ at fixed u).
int adjh_step_vjp(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], int positivity, const double* u,
                  double dt, const double* ybar, double* ubar, double* gb) {
    oracle::Mesh m;
    for (int d = 0; d < 3; d++) {
        m.n[d] = mesh->n[d];
        m.lo[d] = mesh->lo[d];
        m.dx[d] = mesh->dx[d];
    }
    m.ng = mesh->ng;
    oracle::Euler<double> sys{oracle::Nasg<double>{eos->gamma, eos->p_inf, eos->b, eos->q, eos->cv}};
    oracle::Solver<double> s(sys, m);
    for (int d = 0; d < 3; d++)
        for (int q = 0; q < 2; q++) {
            s.bc[d][q].kind = bc[2 * d + q].kind;
            for (int k = 0; k < 5; k++) s.bc[d][q].state[k] = bc[2 * d + q].state[k];
        }
    s.mode = oracle::WENO;
    s.positivity = positivity != 0;
    s.stage_dt = dt;
    const size_t len = m.len();
    std::vector<V5d> X1(len), X2, X3, Y(len), an(len, V5d{0, 0, 0, 0, 0}), ax(len, V5d{0, 0, 0, 0, 0}),
        ay(len, V5d{0, 0, 0, 0, 0});
    std::memcpy(X1.data(), u, len * 5 * sizeof(double));
    std::memcpy(Y.data(), ybar, len * 5 * sizeof(double));
    // forward stages (the oracle's step, keeping the stage inputs)
    s.u = X1;
    s.rhs(s.u);
    X1 = s.u;  // ghost-filled
    s.stage = s.u;
    s.rk_combine<1>(s.stage, s.u, dt);
    s.rhs(s.stage);
    X2 = s.stage;
    s.rk_combine<2>(s.stage, s.u, dt);
    s.rhs(s.stage);
    X3 = s.stage;
    CpuAdj A{s, emg::Eos<double>{eos->gamma, eos->p_inf, eos->b, eos->q}, dt};
    double g = 0.0;
    auto interior = [&](auto fn) {
        for (int64_t i = m.g(0); i < m.g(0) + m.n[0]; i++)
            for (int64_t j = m.g(1); j < m.g(1) + m.n[1]; j++)
                for (int64_t k = m.g(2); k < m.g(2) + m.n[2]; k++) fn(m.idx(i, j, k));
    };
    interior([&](int64_t c) {
        for (int k = 0; k < 5; k++) {
            an[c][k] = (1.0 / 3.0) * Y[c][k];
            ax[c][k] = (2.0 / 3.0) * Y[c][k];
        }
    });
    A.sweeps(X3, Y, (2.0 / 3.0) * dt, dt, ax, g);
    A.ghosts_rev(ax);
    interior([&](int64_t c) {
        for (int k = 0; k < 5; k++) {
            an[c][k] = an[c][k] + 0.75 * ax[c][k];
            ay[c][k] = 0.25 * ax[c][k];
        }
    });
    A.sweeps(X2, ax, 0.25 * dt, dt, ay, g);
    A.ghosts_rev(ay);
    interior([&](int64_t c) {
        for (int k = 0; k < 5; k++) an[c][k] = an[c][k] + ay[c][k];
    });
    A.sweeps(X1, ay, dt, dt, an, g);
    A.ghosts_rev(an);
    std::memcpy(ubar, an.data(), len * 5 * sizeof(double));
    *gb = g;
    return 0;
}

}  // extern "C"

extern "C" {
// The three (ghost-filled) stage inputs of one step, as adjh_step_vjp forms them.
int adjh_stage_inputs(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], int positivity, const double* u,
                      double dt, double* x1, double* x2, double* x3) {
    oracle::Mesh m;
    for (int d = 0; d < 3; d++) {
        m.n[d] = mesh->n[d];
        m.lo[d] = mesh->lo[d];
        m.dx[d] = mesh->dx[d];
    }
    m.ng = mesh->ng;
    oracle::Euler<double> sys{oracle::Nasg<double>{eos->gamma, eos->p_inf, eos->b, eos->q, eos->cv}};
    oracle::Solver<double> s(sys, m);
    for (int d = 0; d < 3; d++)
        for (int q = 0; q < 2; q++) {
            s.bc[d][q].kind = bc[2 * d + q].kind;
            for (int k = 0; k < 5; k++) s.bc[d][q].state[k] = bc[2 * d + q].state[k];
        }
    s.mode = oracle::WENO;
    s.positivity = positivity != 0;
    s.stage_dt = dt;
    const size_t len = m.len();
    std::memcpy(s.u.data(), u, len * 5 * sizeof(double));
    s.rhs(s.u);
    std::memcpy(x1, s.u.data(), len * 5 * sizeof(double));
    s.stage = s.u;
    s.rk_combine<1>(s.stage, s.u, dt);
    s.rhs(s.stage);
    std::memcpy(x2, s.stage.data(), len * 5 * sizeof(double));
    s.rk_combine<2>(s.stage, s.u, dt);
    s.rhs(s.stage);
    std::memcpy(x3, s.stage.data(), len * 5 * sizeof(double));
    return 0;
}
}  // extern "C"

extern "C" {
// Face fluxes of a primitive line (no limiter) in dual numbers.
int adjh_line_jvp(const emg_eos* eos, const double* w, const double* dw, int len, int d, int ng, double* f,
                  double* df) {
    auto sys = dsys(eos, 0.0);
    std::vector<oracle::V5<Dual>> wl(len), out(len - 2 * ng + 1);
    for (int c = 0; c < len; c++) wl[c] = dv(w + 5 * c, dw + 5 * c);
    oracle::Stats st;
    oracle::SchemeOpts o{oracle::WENO, 1e-3, 0.0};
    oracle::line_fluxes(sys, wl.data(), len, d, ng, o, out.data(), (Dual*)nullptr, st);
    for (size_t i = 0; i < out.size(); i++)
        for (int k = 0; k < 5; k++) {
            f[5 * i + k] = out[i][k].v;
            df[5 * i + k] = out[i][k].d;
        }
    return 0;
}
// Its reverse: face-flux cotangents Fb (n+1 faces) → primitive cotangents wb.
int adjh_line_vjp(const emg_eos* eos, const double* w, int len, int d, int ng, const double* Fb, double* wb) {
    emg::Eos<double> e = deos(eos);
    const int n = len - 2 * ng;
    double g = 0.0;
    for (int c = 0; c < 5 * len; c++) wb[c] = 0.0;
    auto A = [&](int i, int k) { return (i >= ng - 1 && i <= ng + n - 1) ? Fb[5 * (i - ng + 1) + k] : 0.0; };
    for (int j = ng - 3; j <= ng + n + 1; j++) {
        double fb[5];
        for (int k = 0; k < 5; k++)
            fb[k] = oracle::S6[0] * A(j, k) + oracle::S6[1] * (A(j - 1, k) + A(j + 1, k)) +
                    oracle::S6[2] * (A(j - 2, k) + A(j + 2, k));
        double w6[6][5], wb6[6][5] = {{0}};
        for (int q = 0; q < 6; q++)
            for (int k = 0; k < 5; k++) w6[q][k] = w[5 * (j - 2 + q) + k];
        if (d == 0) emg::adj::midpoint_vjp<0>(e, w6, fb, wb6, g);
        if (d == 1) emg::adj::midpoint_vjp<1>(e, w6, fb, wb6, g);
        if (d == 2) emg::adj::midpoint_vjp<2>(e, w6, fb, wb6, g);
        for (int q = 0; q < 6; q++)
            for (int k = 0; k < 5; k++) wb[5 * (j - 2 + q) + k] += wb6[q][k];
    }
    return 0;
}
}  // extern "C"

// ---- (study aid) the mixed form's midpoint flux on the host, variants ----
namespace {
// variant 0: as the device mixed sweep (FP32 avg, eigenvectors, projection,
// WENO-Z, back-projection, HLLC); variant 1: characteristic deviations from
// the FP64 value at row j (WENO is translation invariant), FP32 WENO on the
// deviations, back-projection + HLLC in FP32; variant 2: as 1 with the
// back-projection and HLLC in FP64.
template <int D>
void mixed_midpoint(const emg::Eos<double>& ed, const double (*w6)[5], int variant, double* f) {
    using emg::Eos;
    const Eos<float> ef = Eos<float>::from(emg::EosD{ed.gamma, ed.p_inf, ed.b, ed.q});
    constexpr int un = 1 + D, t1 = 1 + (D + 1) % 3, t2 = 1 + (D + 2) % 3;
    if (variant == 0) {
        float w[6][5];
        for (int s = 0; s < 6; s++)
            for (int k = 0; k < 5; k++) w[s][k] = (float)w6[s][k];
        float avg0 = 0.5f * (w[2][0] + w[3][0]), avg4 = 0.5f * (w[2][4] + w[3][4]);
        float rho = avg0, c = emg::sound_speed(ef, avg0, avg4);
        float l4un = rho / (2.f * c), l0un = -l4un, l04 = 1.f / (2.f * c * c), l14 = -1.f / (c * c);
        float run4 = c / rho, run0 = -run4, r40 = c * c;
        float ch[5][6];
        for (int s = 0; s < 6; s++) {
            ch[0][s] = l0un * w[s][un] + l04 * w[s][4];
            ch[1][s] = w[s][0] + l14 * w[s][4];
            ch[2][s] = w[s][t1];
            ch[3][s] = w[s][t2];
            ch[4][s] = l4un * w[s][un] + l04 * w[s][4];
        }
        float cl[5], cr[5];
        for (int a = 0; a < 5; a++) {
            cl[a] = emg::weno5z_interp(ch[a][0], ch[a][1], ch[a][2], ch[a][3], ch[a][4]);
            cr[a] = emg::weno5z_interp(ch[a][5], ch[a][4], ch[a][3], ch[a][2], ch[a][1]);
        }
        float wl[5], wr[5];
        wl[0] = (cl[0] + cl[1]) + cl[4];
        wr[0] = (cr[0] + cr[1]) + cr[4];
        wl[un] = run0 * cl[0] + run4 * cl[4];
        wr[un] = run0 * cr[0] + run4 * cr[4];
        wl[t1] = cl[2]; wr[t1] = cr[2]; wl[t2] = cl[3]; wr[t2] = cr[3];
        wl[4] = r40 * cl[0] + r40 * cl[4];
        wr[4] = r40 * cr[0] + r40 * cr[4];
        if (!emg::admissible(ef, wl[0], wl[4]) || !emg::admissible(ef, wr[0], wr[4]))
            for (int k = 0; k < 5; k++) { wl[k] = w[2][k]; wr[k] = w[3][k]; }
        float ff[5];
        emg::hllc(ef, wl, wr, un, ff);
        for (int k = 0; k < 5; k++) f[k] = ff[k];
        return;
    }
    // characteristic projection in FP64, deviations from row 2 (left) / row 3 (right)
    double avg0 = 0.5 * (w6[2][0] + w6[3][0]), avg4 = 0.5 * (w6[2][4] + w6[3][4]);
    double rho = avg0, c = emg::sound_speed(ed, avg0, avg4);
    double l4un = rho / (2.0 * c), l0un = -l4un, l04 = 1.0 / (2.0 * c * c), l14 = -1.0 / (c * c);
    double run4 = c / rho, run0 = -run4, r40 = c * c;
    double ch[5][6];
    for (int s = 0; s < 6; s++) {
        ch[0][s] = l0un * w6[s][un] + l04 * w6[s][4];
        ch[1][s] = w6[s][0] + l14 * w6[s][4];
        ch[2][s] = w6[s][t1];
        ch[3][s] = w6[s][t2];
        ch[4][s] = l4un * w6[s][un] + l04 * w6[s][4];
    }
    double cl[5], cr[5];
    for (int a = 0; a < 5; a++) {
        const double bl = variant == 3 ? 0.0 : ch[a][2], br = variant == 3 ? 0.0 : ch[a][3];
        float v[6];
        for (int s = 0; s < 6; s++) v[s] = (float)(ch[a][s] - bl);
        cl[a] = bl + (double)emg::weno5z_interp(v[0], v[1], v[2], v[3], v[4]);
        for (int s = 0; s < 6; s++) v[s] = (float)(ch[a][s] - br);
        cr[a] = br + (double)emg::weno5z_interp(v[5], v[4], v[3], v[2], v[1]);
    }
    double wl[5], wr[5];
    wl[0] = (cl[0] + cl[1]) + cl[4];
    wr[0] = (cr[0] + cr[1]) + cr[4];
    wl[un] = run0 * cl[0] + run4 * cl[4];
    wr[un] = run0 * cr[0] + run4 * cr[4];
    wl[t1] = cl[2]; wr[t1] = cr[2]; wl[t2] = cl[3]; wr[t2] = cr[3];
    wl[4] = r40 * cl[0] + r40 * cl[4];
    wr[4] = r40 * cr[0] + r40 * cr[4];
    if (!emg::admissible(ed, wl[0], wl[4]) || !emg::admissible(ed, wr[0], wr[4]))
        for (int k = 0; k < 5; k++) { wl[k] = w6[2][k]; wr[k] = w6[3][k]; }
    if (variant == 2 || variant == 3) {
        emg::hllc(ed, wl, wr, un, f);
        return;
    }
    float wlf[5], wrf[5], ff[5];
    for (int k = 0; k < 5; k++) { wlf[k] = (float)wl[k]; wrf[k] = (float)wr[k]; }
    emg::hllc(ef, wlf, wrf, un, ff);
    for (int k = 0; k < 5; k++) f[k] = ff[k];
}
}  // namespace

extern "C" {
// Face fluxes (S6 of midpoint fluxes, no limiter) of a primitive line with the
// midpoint flux in a mixed-precision variant (variant < 0: plain FP64).
int adjh_mixed_line_fluxes(const emg_eos* eos, const double* w, int len, int d, int ng, int variant, double* out) {
    emg::Eos<double> e = deos(eos);
    const int n = len - 2 * ng;
    std::vector<double> mf(5 * len, 0.0);
    for (int j = ng - 3; j <= ng + n + 1; j++) {
        const double(*w6)[5] = reinterpret_cast<const double(*)[5]>(w + 5 * (j - 2));
        double f[5];
        if (variant < 0) {
            oracle::Euler<double> sys{oracle::Nasg<double>{eos->gamma, eos->p_inf, eos->b, eos->q, eos->cv}};
            std::vector<oracle::V5<double>> wl(len);
            for (int c = 0; c < len; c++)
                for (int k = 0; k < 5; k++) wl[c][k] = w[5 * c + k];
            auto m = oracle::midpoint_flux(sys, wl.data(), j, d);
            for (int k = 0; k < 5; k++) f[k] = m.f[k];
        } else if (d == 0) mixed_midpoint<0>(e, w6, variant, f);
        else if (d == 1) mixed_midpoint<1>(e, w6, variant, f);
        else mixed_midpoint<2>(e, w6, variant, f);
        for (int k = 0; k < 5; k++) mf[5 * j + k] = f[k];
    }
    for (int fc = 0; fc <= n; fc++) {
        const int i = ng - 1 + fc;
        for (int k = 0; k < 5; k++) {
            double acc = 0.0;
            acc = acc + oracle::S6[0] * mf[5 * i + k];
            acc = acc + oracle::S6[1] * mf[5 * (i + 1) + k];
            acc = acc + oracle::S6[1] * mf[5 * (i - 1) + k];
            acc = acc + oracle::S6[2] * mf[5 * (i + 2) + k];
            acc = acc + oracle::S6[2] * mf[5 * (i - 2) + k];
            out[5 * fc + k] = acc;
        }
    }
    return 0;
}
}  // extern "C"
