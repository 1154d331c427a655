// CPU ORACLE — test infrastructure only.
//
// C++ restatement of the reference's five-equation two-phase system (Kapila's
// model, fluid/crates/compressible/src/multiphase.rs:1-392) and of the
// system-generic parts of its explicit uniform-grid step that this system
// exercises: the hybrid / WCNS line fluxes with face velocities
// (fluid/crates/compressible/src/scheme.rs:132-333), the positivity limiter
// (scheme.rs:395-464), ghost fill (solver.rs:278-348, boundary.rs), the
// residual with the non-conservative α term (solver.rs:351-475), SSP-RK3
// (solver.rs:97-137, 659-738) and the CFL step with the dilatation limit
// (solver.rs:478-523, neighbour states as solver.rs:565-640). Only the test
// suite loads it, as the checker of the five-equation device path; the
// product library never links, loads or calls it.
//
// Every formula keeps the reference's operation order (build with
// -ffp-contract=off). The scheme loops are dense over the N = 7 variables as
// in the reference (zero entries of the eigenvectors included).
#pragma once
#include "oracle.hpp"

namespace oracle {

template <class T> using V7 = std::array<T, 7>;
template <class T> using Mat7 = std::array<std::array<T, 7>, 7>;

// Rust f64::clamp (NaN stays NaN)
inline double clamp_(double x, double lo, double hi) {
    if (x < lo) return lo;
    if (x > hi) return hi;
    return x;
}

// ---------------------------------------------------------------- system
// multiphase.rs: conserved (a1, a2, ρu, ρv, ρw, E, α1), primitive (a1, a2, u, v, w, p, α1)
template <class T> struct FiveEq {
    static constexpr int N = 7;
    static constexpr int IA = 6, IP = 5, IU = 2;
    Nasg<T> eos[2];
    bool kapila = true;

    // multiphase.rs:58-69
    void db(const V7<T>& w, T& d, T& b) const {
        T al[2] = {w[IA], T(1.0) - w[IA]};
        d = T(0.0);
        b = T(0.0);
        for (int k = 0; k < 2; k++) {
            const Nasg<T>& e = eos[k];
            T vol = al[k] - e.b * w[k];
            d = d + vol / (e.gamma - T(1.0));
            b = b + e.gamma * e.p_inf * vol / (e.gamma - T(1.0)) + e.q * w[k];
        }
    }
    // multiphase.rs:71-75
    T rho_e(const V7<T>& w) const {
        T d, b;
        db(w, d, b);
        return w[IP] * d + b;
    }
    // multiphase.rs:77-84
    T rho_c2_phase(const V7<T>& w, int k) const {
        T al = k == 0 ? w[IA] : T(1.0) - w[IA];
        const Nasg<T>& e = eos[k];
        T rho_k = (al > T(1e-12) && w[k] > T(0.0)) ? w[k] / al : T(0.0);
        return e.gamma * (w[IP] + e.p_inf) / fmax_(T(1.0) - e.b * rho_k, T(1e-12));
    }
    // multiphase.rs:86-97
    T kapila_k(const V7<T>& w) const {
        if (!kapila) return T(0.0);
        T a = clamp_(w[IA], 0.0, 1.0);
        T al[2] = {a, T(1.0) - a};
        T z1 = rho_c2_phase(w, 0), z2 = rho_c2_phase(w, 1);
        T den = al[1] * z1 + al[0] * z2;
        if (den <= T(0.0)) return T(0.0);
        return al[0] * al[1] * (z2 - z1) / den;
    }
    // multiphase.rs:113-117
    T drhoe_dalpha(T p) const {
        const Nasg<T>&e1 = eos[0], &e2 = eos[1];
        return (p + e1.gamma * e1.p_inf) / (e1.gamma - T(1.0)) - (p + e2.gamma * e2.p_inf) / (e2.gamma - T(1.0));
    }
    // multiphase.rs:100-110
    T rho_c2(const V7<T>& w) const {
        T d, bb;
        db(w, d, bb);
        T p = w[IP];
        T num = rho_e(w) + p;
        for (int k = 0; k < 2; k++) {
            const Nasg<T>& e = eos[k];
            num = num + w[k] * (e.b * (p + e.gamma * e.p_inf) / (e.gamma - T(1.0)) - e.q);
        }
        num = num + kapila_k(w) * drhoe_dalpha(p);
        return num / d;
    }
    static T rho(const V7<T>& w) { return w[0] + w[1]; }
    // multiphase.rs:127-130
    T p_inf_mix(const V7<T>& w) const {
        T a = clamp_(w[IA], 0.0, 1.0);
        return a * eos[0].p_inf + (T(1.0) - a) * eos[1].p_inf;
    }
    // multiphase.rs:131-146
    V7<T> to_prim(const V7<T>& u) const {
        T r = u[0] + u[1];
        T vx = u[2] / r, vy = u[3] / r, vz = u[4] / r;
        V7<T> w{};
        w[0] = u[0];
        w[1] = u[1];
        w[2] = vx;
        w[3] = vy;
        w[4] = vz;
        w[IA] = u[6];
        T rhoe = u[5] - T(0.5) * r * (vx * vx + vy * vy + vz * vz);
        T d, b;
        db(w, d, b);
        w[IP] = (rhoe - b) / d;
        return w;
    }
    // multiphase.rs:152-163
    V7<T> to_cons(const V7<T>& w) const {
        T r = w[0] + w[1];
        V7<T> u{};
        u[0] = w[0];
        u[1] = w[1];
        u[2] = r * w[2];
        u[3] = r * w[3];
        u[4] = r * w[4];
        u[5] = rho_e(w) + T(0.5) * r * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
        u[6] = w[IA];
        return u;
    }
    // multiphase.rs:165-167
    T sound_speed(const V7<T>& w) const { return std::sqrt(fmax_(rho_c2(w), T(0.0)) / rho(w)); }
    int momentum_index(int d) const { return 2 + d; }
    // multiphase.rs:202-236
    void eigen(const V7<T>& w, int d, Mat7<T>& l, Mat7<T>& r) const {
        T rh = rho(w);
        T c = sound_speed(w);
        T kk = kapila_k(w);
        int un = IU + d, t1 = IU + (d + 1) % 3, t2 = IU + (d + 2) % 3;
        for (auto& row : l) row.fill(T(0.0));
        for (auto& row : r) row.fill(T(0.0));
        T c2 = c * c;
        l[0][0] = T(1.0);
        l[0][IP] = -w[0] / rh / c2;
        l[1][1] = T(1.0);
        l[1][IP] = -w[1] / rh / c2;
        l[2][un] = -rh / (T(2.0) * c);
        l[2][IP] = T(1.0) / (T(2.0) * c2);
        l[3][t1] = T(1.0);
        l[4][t2] = T(1.0);
        l[5][un] = rh / (T(2.0) * c);
        l[5][IP] = T(1.0) / (T(2.0) * c2);
        l[6][IA] = T(1.0);
        l[6][IP] = kk / rh / c2;
        r[0][0] = T(1.0);
        r[1][1] = T(1.0);
        r[t1][3] = T(1.0);
        r[t2][4] = T(1.0);
        r[IA][6] = T(1.0);
        const int cols[2] = {2, 5};
        const double sg[2] = {-1.0, 1.0};
        for (int m = 0; m < 2; m++) {
            int col = cols[m];
            r[0][col] = w[0] / rh;
            r[1][col] = w[1] / rh;
            r[un][col] = T(sg[m]) * c / rh;
            r[IP][col] = c2;
            r[IA][col] = -kk / rh;
        }
    }
    // multiphase.rs:238-243
    V7<T> eigenvalues(const V7<T>& w, int d) const {
        T u = w[IU + d], c = sound_speed(w);
        return {u, u, u - c, u, u, u + c, u};
    }
    // multiphase.rs:331-343
    V7<T> flux(const V7<T>& w, int d) const {
        int un = IU + d;
        V7<T> q = to_cons(w);
        T u = w[un];
        V7<T> f{};
        for (int k = 0; k < 5; k++) f[k] = q[k] * u;
        f[un] = f[un] + w[IP];
        f[5] = (q[5] + w[IP]) * u;
        f[6] = w[IA] * u;
        return f;
    }
    // multiphase.rs:245-289 (HLLC, Davis bounds); *ss the contact speed
    V7<T> riemann_flux(const V7<T>& wl, const V7<T>& wr, int d, T* ss_out) const {
        int un = IU + d;
        T cl = sound_speed(wl), cr = sound_speed(wr);
        T ul = wl[un], ur = wr[un];
        T sl = fmin_(ul - cl, ur - cr);
        T sr = fmax_(ul + cl, ur + cr);
        V7<T> ql = to_cons(wl), qr = to_cons(wr);
        if (sl >= T(0.0)) {
            *ss_out = ul;
            return flux(wl, d);
        }
        if (sr <= T(0.0)) {
            *ss_out = ur;
            return flux(wr, d);
        }
        T rl = rho(wl), rr = rho(wr);
        T pl = wl[IP], pr = wr[IP];
        T ss = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) / (rl * (sl - ul) - rr * (sr - ur));
        auto star = [&](const V7<T>& w, const V7<T>& q, T s) {
            T rh = rho(w), u = w[un];
            T fac = (s - u) / (s - ss);
            V7<T> qs{};
            qs[0] = w[0] * fac;
            qs[1] = w[1] * fac;
            for (int k = IU; k < IU + 3; k++) qs[k] = rh * fac * w[k];
            qs[un] = rh * fac * ss;
            qs[5] = rh * fac * (q[5] / rh + (ss - u) * (ss + w[IP] / (rh * (s - u))));
            qs[6] = w[IA] * fac;
            return qs;
        };
        V7<T> f{};
        if (ss >= T(0.0)) {
            V7<T> fl = flux(wl, d), qs = star(wl, ql, sl);
            for (int k = 0; k < 7; k++) f[k] = fl[k] + sl * (qs[k] - ql[k]);
        } else {
            V7<T> fr = flux(wr, d), qs = star(wr, qr, sr);
            for (int k = 0; k < 7; k++) f[k] = fr[k] + sr * (qs[k] - qr[k]);
        }
        *ss_out = ss;
        return f;
    }
    // multiphase.rs:291-309
    V7<T> split_flux(const V7<T>& a, const V7<T>& b, int d) const {
        int un = IU + d;
        T u = T(0.5) * (a[un] + b[un]);
        T rh = T(0.5) * (rho(a) + rho(b));
        T c = rh * u;
        V7<T> f{};
        f[0] = T(0.5) * (a[0] + b[0]) * u;
        f[1] = T(0.5) * (a[1] + b[1]) * u;
        for (int k = IU; k < IU + 3; k++) f[k] = c * T(0.5) * (a[k] + b[k]);
        f[un] = f[un] + T(0.5) * (a[IP] + b[IP]);
        T kin = c * T(0.5) * (a[2] * b[2] + a[3] * b[3] + a[4] * b[4]);
        T rhoe = T(0.5) * (rho_e(a) + rho_e(b));
        T pw = T(0.5) * (a[un] * b[IP] + b[un] * a[IP]);
        f[5] = kin + u * rhoe + pw;
        f[6] = T(0.5) * (a[IA] + b[IA]) * u;
        return f;
    }
    // multiphase.rs:345-350
    bool admissible(const V7<T>& w) const {
        for (int k = 0; k < 7; k++)
            if (!std::isfinite(w[k])) return false;
        return rho(w) > T(0.0) && w[IA] >= T(-0.05) && w[IA] <= T(1.05) && rho_c2(w) > T(0.0);
    }
    T nc_coef(const V7<T>& w) const { return w[IA] + kapila_k(w); }  // multiphase.rs:356-358
    // multiphase.rs:363-377
    T dilatation_rate(const V7<T>& w, T divu) const {
        T a = w[IA];
        T pmin_inf = T(INFINITY);
        if (a > T(1e-6)) pmin_inf = fmin_(pmin_inf, eos[0].p_inf);
        if (T(1.0) - a > T(1e-6)) pmin_inf = fmin_(pmin_inf, eos[1].p_inf);
        T floor = T(1e-6) * fmax_(eos[0].p_inf, eos[1].p_inf);
        T head = fmax_(fmax_(w[IP] + pmin_inf, floor), T(1e-300));
        return fmax_(rho_c2(w), T(0.0)) * std::fabs(divu) / head;
    }
    // multiphase.rs:379-384
    int sensor(const V7<T>& w, T* out) const {
        out[0] = std::log(fmax_(rho(w), T(1e-300)));
        out[1] = std::log(fmax_(w[IP] + p_inf_mix(w), T(1e-300)));
        out[2] = w[IA];
        return 3;
    }
    // system.rs:185-187
    T max_speed(const V7<T>& w, int d) const { return std::fabs(w[IU + d]) + sound_speed(w); }
    // multiphase.rs:148-150
    T velocity_conserved(const V7<T>& u, int d) const { return u[2 + d] / (u[0] + u[1]); }
};

// ---------------------------------------------------------------- scheme (dense N = 7)
template <class T> struct MidResult7 {
    V7<T> f;
    T us;
    bool fb;
};

// scheme.rs:286-333
template <class T>
MidResult7<T> midpoint_flux7(const FiveEq<T>& sys, const V7<T>* w, int j, int d) {
    V7<T> avg;
    for (int k = 0; k < 7; k++) avg[k] = T(0.5) * (w[j][k] + w[j + 1][k]);
    Mat7<T> l, r;
    sys.eigen(avg, d, l, r);
    T ch[6][7];
    for (int s = 0; s < 6; s++) {
        const V7<T>& ws = w[j - 2 + s];
        for (int a = 0; a < 7; a++) {
            T acc = T(0.0);
            for (int k = 0; k < 7; k++) acc = acc + l[a][k] * ws[k];
            ch[s][a] = acc;
        }
    }
    T cl[7], cr[7];
    for (int a = 0; a < 7; a++) {
        cl[a] = weno5z_interp(ch[0][a], ch[1][a], ch[2][a], ch[3][a], ch[4][a]);
        cr[a] = weno5z_interp(ch[5][a], ch[4][a], ch[3][a], ch[2][a], ch[1][a]);
    }
    V7<T> wl, wr;
    for (int k = 0; k < 7; k++) {
        T sl = T(0.0), sr = T(0.0);
        for (int a = 0; a < 7; a++) {
            sl = sl + r[k][a] * cl[a];
            sr = sr + r[k][a] * cr[a];
        }
        wl[k] = sl;
        wr[k] = sr;
    }
    bool fb = false;
    if (!sys.admissible(wl) || !sys.admissible(wr)) {
        fb = true;
        wl = w[j];
        wr = w[j + 1];
    }
    MidResult7<T> m;
    m.f = sys.riemann_flux(wl, wr, d, &m.us);
    m.fb = fb;
    return m;
}

// scheme.rs:395-464 (face velocities blended with the mean velocity)
template <class T>
void positivity_limit7(const FiveEq<T>& sys, const V7<T>* w, int len, int d, int ng, double lambda, V7<T>* out,
                       T* uface, Stats& stats) {
    int n = len - 2 * ng;
    V7<T> previous_cons = sys.to_cons(w[ng - 1]);
    V7<T> previous_flux = sys.flux(w[ng - 1], d);
    for (int f = 0; f <= n; f++) {
        int i = ng - 1 + f;
        V7<T> ul = previous_cons, fl_phys = previous_flux;
        V7<T> ur = sys.to_cons(w[i + 1]);
        V7<T> fr_phys = sys.flux(w[i + 1], d);
        previous_cons = ur;
        previous_flux = fr_phys;
        auto ok = [&](const V7<T>& fx) {
            V7<T> a, b;
            for (int k = 0; k < 7; k++) {
                a[k] = ul[k] - T(2.0) * T(lambda) * (fx[k] - fl_phys[k]);
                b[k] = ur[k] + T(2.0) * T(lambda) * (fx[k] - fr_phys[k]);
            }
            return sys.admissible(sys.to_prim(a)) && sys.admissible(sys.to_prim(b));
        };
        V7<T> fh = out[f];
        bool all_finite = true;
        for (int k = 0; k < 7; k++) all_finite = all_finite && std::isfinite(fh[k]);
        if (all_finite && ok(fh)) continue;
        T alpha = fmax_(sys.max_speed(w[i], d), sys.max_speed(w[i + 1], d));
        V7<T> flf;
        for (int k = 0; k < 7; k++) flf[k] = T(0.5) * (fl_phys[k] + fr_phys[k]) - T(0.5) * alpha * (ur[k] - ul[k]);
        stats.limited_faces += 1;
        auto blend = [&](T t) {
            V7<T> v;
            for (int k = 0; k < 7; k++) v[k] = std::isfinite(fh[k]) ? t * fh[k] + (T(1.0) - t) * flf[k] : flf[k];
            return v;
        };
        T lo = T(0.0), hi = T(1.0);
        for (int it = 0; it < 30; it++) {
            T mid = T(0.5) * (lo + hi);
            if (ok(blend(mid)))
                lo = mid;
            else
                hi = mid;
        }
        out[f] = blend(lo);
        int un = 2 + d;
        T um = T(0.5) * (w[i][un] + w[i + 1][un]);
        uface[f] = std::isfinite(uface[f]) ? lo * uface[f] + (T(1.0) - lo) * um : um;
    }
}

// scheme.rs:132-281 (Wcns shock path), faces and face velocities
template <class T>
void line_fluxes7(const FiveEq<T>& sys, const V7<T>* w, int len, int d, int ng, const SchemeOpts& o, V7<T>* out,
                  T* uface, Stats& stats) {
    int n = len - 2 * ng;
    int un = 2 + d;
    int ns = 0;
    std::vector<std::array<T, 3>> sens;
    if (o.mode == HYBRID) {
        sens.resize(len);
        for (int c = 0; c < len; c++) {
            T v[8];
            ns = sys.sensor(w[c], v);
            sens[c] = {v[0], v[1], v[2]};
        }
    }
    std::vector<MidResult7<T>> mid;
    std::vector<char> have;
    if (o.mode != CENTRAL) {
        mid.resize(len);
        have.assign(len, 0);
    }
    for (int f = 0; f <= n; f++) {
        int i = ng - 1 + f;
        T theta;
        if (o.mode == CENTRAL) {
            theta = T(0.0);
        } else if (o.mode == WENO) {
            theta = T(1.0);
        } else {
            T r = T(0.0);
            for (int k = 0; k < ns; k++) {
                auto s = [&](int j) { return sens[j][k]; };
                r = fmax_(fmax_(r, d4(s(i - 2), s(i - 1), s(i), s(i + 1), s(i + 2))),
                          d4(s(i - 1), s(i), s(i + 1), s(i + 2), s(i + 3)));
            }
            T x = (r / T(o.tol) - T(0.5)) / T(0.5);
            if (x < T(0.0)) x = T(0.0);
            if (x > T(1.0)) x = T(1.0);
            theta = std::isfinite(r) ? x * x * (T(3.0) - T(2.0) * x) : T(1.0);
        }
        stats.faces += 1;
        V7<T> central{};
        T uf_c = T(0.0);
        if (theta < T(1.0)) {
            for (int li = 0; li < 3; li++) {
                int lag = li + 1;
                for (int m = 0; m < lag; m++) {
                    const V7<T>& wa = w[i - m];
                    const V7<T>& wb = w[i - m + lag];
                    V7<T> ft = sys.split_flux(wa, wb, d);
                    for (int k = 0; k < 7; k++) central[k] = central[k] + T(2.0) * T(A6[li]) * ft[k];
                    uf_c = uf_c + T(A6[li]) * (wa[un] + wb[un]);
                }
            }
            if (theta == T(0.0)) {
                out[f] = central;
                uface[f] = uf_c;
                continue;
            }
        }
        stats.weno_faces += 1;
        V7<T> fl{};
        T uf = T(0.0);
        for (int s = 0; s < 3; s++) {
            T c = T(S6[s]);
            int js[2] = {i + s, i - s};
            int nj = s == 0 ? 1 : 2;
            for (int q = 0; q < nj; q++) {
                int j = js[q];
                if (!have[j]) {
                    mid[j] = midpoint_flux7(sys, w, j, d);
                    stats.fallback_faces += mid[j].fb ? 1 : 0;
                    have[j] = 1;
                }
                for (int k = 0; k < 7; k++) fl[k] = fl[k] + c * mid[j].f[k];
                uf = uf + c * mid[j].us;
            }
        }
        out[f] = fl;
        uface[f] = uf;
        if (theta < T(1.0)) {
            for (int k = 0; k < 7; k++) out[f][k] = theta * out[f][k] + (T(1.0) - theta) * central[k];
            uface[f] = theta * uface[f] + (T(1.0) - theta) * uf_c;
        }
    }
    if (o.lambda > 0.0) positivity_limit7(sys, w, len, d, ng, o.lambda, out, uface, stats);
}

// ---------------------------------------------------------------- boundary (N = 7)
template <class T> struct Bc7 {
    int kind = BC_PERIODIC;
    V7<T> state{};  // conserved Dirichlet / far-field state
};

// boundary.rs:48-96 with the five-equation eigenvectors
template <class T> struct CharStencil7 {
    V7<T> wi, wf, w1;
    Mat7<T> l, r;
    bool outgoing[7];
    CharStencil7() = default;
    CharStencil7(const FiveEq<T>& sys, const V7<T>& u_b, const V7<T>& u_b1, const V7<T>& u_far, int d, int side) {
        wi = sys.to_prim(u_b);
        wf = sys.to_prim(u_far);
        w1 = sys.to_prim(u_b1);
        sys.eigen(wi, d, l, r);
        V7<T> lam = sys.eigenvalues(wi, d);
        double outward = side == 1 ? 1.0 : -1.0;
        for (int k = 0; k < 7; k++) outgoing[k] = lam[k] * T(outward) > T(0.0);
    }
    V7<T> conserved(const FiveEq<T>& sys, double m) const {
        V7<T> dw;
        for (int k = 0; k < 7; k++) dw[k] = wi[k] - wf[k] + T(m) * (wi[k] - w1[k]);
        V7<T> wg = wf;
        for (int kf = 0; kf < 7; kf++) {
            if (outgoing[kf]) {
                T amp = T(-0.0);  // Rust (0..N).map(..).sum() folds from -0.0
                for (int q = 0; q < 7; q++) amp = amp + l[kf][q] * dw[q];
                for (int q = 0; q < 7; q++) wg[q] = wg[q] + r[q][kf] * amp;
            }
        }
        return sys.to_cons(wg);
    }
};

// ---------------------------------------------------------------- solver (uniform grid, N = 7)
template <class T> struct SolverFive {
    FiveEq<T> sys;
    Mesh mesh;
    std::vector<V7<T>> u;
    Bc7<T> bc[3][2];
    double cfl = 0.5;
    int mode = HYBRID;
    double tol = 1e-3;
    double t = 0.0;
    Stats stats;
    bool positivity = true;
    double stage_dt = 0.0;
    std::vector<V7<T>> rhs_buf, stage;

    SolverFive(const FiveEq<T>& s, const Mesh& m) : sys(s), mesh(m) {
        u.assign(mesh.len(), V7<T>{});
        rhs_buf = u;
        stage = u;
    }

    // solver.rs:278-348 (n >= ng on reflecting axes: no deep images)
    void fill_ghosts(std::vector<V7<T>>& uu) const {
        const Mesh& m = mesh;
        for (int d = 0; d < 3; d++) {
            if (!m.active(d)) continue;
            int64_t n = m.n[d], ng = m.ng;
            int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            const int mom = sys.momentum_index(d);
            for (int64_t a = 0; a < m.m(e0); a++) {
                for (int64_t bb = 0; bb < m.m(e1); bb++) {
                    auto at = [&](int64_t c) {
                        int64_t ijk[3];
                        ijk[d] = c;
                        ijk[e0] = a;
                        ijk[e1] = bb;
                        return m.idx(ijk[0], ijk[1], ijk[2]);
                    };
                    CharStencil7<T> chars[2];
                    if (bc[d][0].kind == BC_CHARACTERISTIC)
                        chars[0] = CharStencil7<T>(sys, uu[at(ng)], uu[at(ng + 1)], bc[d][0].state, d, 0);
                    if (bc[d][1].kind == BC_CHARACTERISTIC)
                        chars[1] = CharStencil7<T>(sys, uu[at(n + ng - 1)], uu[at(n + ng - 2)], bc[d][1].state, d, 1);
                    for (int64_t gi = 0; gi < ng; gi++) {
                        int64_t lo_s, hi_s;
                        m.periodic_ghost_sources(d, gi, lo_s, hi_s);
                        V7<T> vl, vh;
                        switch (bc[d][0].kind) {
                            case BC_PERIODIC: vl = uu[at(lo_s)]; break;
                            case BC_OUTFLOW: vl = uu[at(ng)]; break;
                            case BC_DIRICHLET: vl = bc[d][0].state; break;
                            case BC_CHARACTERISTIC: vl = chars[0].conserved(sys, (double)(ng - gi)); break;
                            default:
                                vl = uu[at(2 * ng - 1 - gi)];
                                vl[mom] = -vl[mom];
                        }
                        uu[at(gi)] = vl;
                        switch (bc[d][1].kind) {
                            case BC_PERIODIC: vh = uu[at(hi_s)]; break;
                            case BC_OUTFLOW: vh = uu[at(n + ng - 1)]; break;
                            case BC_DIRICHLET: vh = bc[d][1].state; break;
                            case BC_CHARACTERISTIC: vh = chars[1].conserved(sys, (double)(gi + 1)); break;
                            default:
                                vh = uu[at(n + ng - 1 - gi)];
                                vh[mom] = -vh[mom];
                        }
                        uu[at(n + ng + gi)] = vh;
                    }
                }
            }
        }
    }

    // solver.rs:351-475: −∇·F plus the non-conservative (α + K)∇·u term
    Stats rhs(std::vector<V7<T>>& uu) {
        fill_ghosts(uu);
        const Mesh& m = mesh;
        for (auto& v : rhs_buf) v = V7<T>{};
        Stats total;
        double ndim = (double)m.ndim();
        for (int d = 0; d < 3; d++) {
            if (!m.active(d)) continue;
            int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            SchemeOpts opts{mode, tol, positivity ? ndim * stage_dt / m.dx[d] : 0.0};
            int64_t ne0 = m.n[e0], ne1 = m.n[e1];
            int64_t npen = ne0 * ne1;
            int64_t len = m.m(d);
            uint64_t f0 = 0, f1 = 0, f2 = 0, f3 = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : f0, f1, f2, f3)
            for (int64_t p = 0; p < npen; p++) {
                int64_t a = p / ne1, b = p % ne1;
                auto at = [&](int64_t c) {
                    int64_t ijk[3];
                    ijk[d] = c;
                    ijk[e0] = a + m.g(e0);
                    ijk[e1] = b + m.g(e1);
                    return m.idx(ijk[0], ijk[1], ijk[2]);
                };
                std::vector<V7<T>> w(len);
                for (int64_t c = 0; c < len; c++) w[c] = sys.to_prim(uu[at(c)]);
                std::vector<V7<T>> fl(m.n[d] + 1);
                std::vector<T> uf(m.n[d] + 1);
                Stats s;
                line_fluxes7(sys, w.data(), (int)len, d, (int)m.ng, opts, fl.data(), uf.data(), s);
                T inv = T(1.0) / T(m.dx[d]);
                for (int64_t c = 0; c < m.n[d]; c++) {
                    V7<T>& o = rhs_buf[at(c + m.ng)];
                    for (int k = 0; k < 7; k++) o[k] = o[k] - (fl[c + 1][k] - fl[c][k]) * inv;
                    o[6] = o[6] + sys.nc_coef(w[c + m.ng]) * (uf[c + 1] - uf[c]) * inv;
                }
                f0 += s.faces;
                f1 += s.weno_faces;
                f2 += s.fallback_faces;
                f3 += s.limited_faces;
            }
            total.faces += f0;
            total.weno_faces += f1;
            total.fallback_faces += f2;
            total.limited_faces += f3;
        }
        return total;
    }

    template <int STAGE>
    void rk_combine(std::vector<V7<T>>& dest, const std::vector<V7<T>>& old, double dt) const {
        const Mesh& m = mesh;
#pragma omp parallel for schedule(static)
        for (int64_t i = m.g(0); i < m.g(0) + m.n[0]; i++)
            for (int64_t j = m.g(1); j < m.g(1) + m.n[1]; j++)
                for (int64_t k = m.g(2); k < m.g(2) + m.n[2]; k++) {
                    int64_t q = m.idx(i, j, k);
                    for (int v = 0; v < 7; v++) {
                        T r = rhs_buf[q][v];
                        if (STAGE == 1)
                            dest[q][v] = old[q][v] + T(dt) * r;
                        else if (STAGE == 2)
                            dest[q][v] = T(0.75) * old[q][v] + T(0.25) * (dest[q][v] + T(dt) * r);
                        else
                            dest[q][v] = dest[q][v] / T(3.0) + T(2.0 / 3.0) * (old[q][v] + T(dt) * r);
                    }
                }
    }

    void step(double dt) {
        stage_dt = dt;
        Stats s1 = rhs(u);
        stage = u;
        rk_combine<1>(stage, u, dt);
        Stats s2 = rhs(stage);
        rk_combine<2>(stage, u, dt);
        Stats s3 = rhs(stage);
        rk_combine<3>(u, stage, dt);
        stats.add(s1);
        stats.add(s2);
        stats.add(s3);
        t += dt;
    }

    // solver.rs:592-640: the state next to interior cell c along d (boundary
    // neighbours from the boundary condition, first ghost layer semantics)
    V7<T> neighbor_conserved(const int64_t c[3], int d, bool high) const {
        const Mesh& m = mesh;
        bool boundary = high ? c[d] == m.g(d) + m.n[d] - 1 : c[d] == m.g(d);
        int64_t q[3] = {c[0], c[1], c[2]};
        if (!boundary) {
            q[d] += high ? 1 : -1;
            return u[m.idx(q[0], q[1], q[2])];
        }
        V7<T> center = u[m.idx(c[0], c[1], c[2])];
        const Bc7<T>& b = bc[d][high ? 1 : 0];
        switch (b.kind) {
            case BC_PERIODIC:
                q[d] = high ? m.g(d) : m.g(d) + m.n[d] - 1;
                return u[m.idx(q[0], q[1], q[2])];
            case BC_OUTFLOW: return center;
            case BC_DIRICHLET: return b.state;
            case BC_REFLECT: {
                V7<T> v = center;
                v[sys.momentum_index(d)] = v[sys.momentum_index(d)] * T(-1.0);
                return v;
            }
            default: {
                q[d] += high ? -1 : 1;
                return CharStencil7<T>(sys, center, u[m.idx(q[0], q[1], q[2])], b.state, d, high ? 1 : 0)
                    .conserved(sys, 1.0);
            }
        }
    }

    // solver.rs:478-523 with the dilatation limit (need_source: the system has an α term)
    double dt_cfl() const {
        const Mesh& m = mesh;
        double rate = 0.0, source = 0.0;
#pragma omp parallel for reduction(max : rate, source) schedule(static)
        for (int64_t i = 0; i < m.n[0]; i++)
            for (int64_t j = 0; j < m.n[1]; j++)
                for (int64_t k = 0; k < m.n[2]; k++) {
                    const int64_t c[3] = {i + m.g(0), j + m.g(1), k + m.g(2)};
                    V7<T> w = sys.to_prim(u[m.idx(c[0], c[1], c[2])]);
                    T acoustic = T(-0.0);
                    for (int d = 0; d < 3; d++)
                        if (m.active(d)) acoustic = acoustic + sys.max_speed(w, d) / T(m.dx[d]);
                    rate = fmax_(rate, acoustic);
                    T divu = T(0.0);
                    for (int d = 0; d < 3; d++) {
                        if (!m.active(d)) continue;
                        T va = sys.velocity_conserved(neighbor_conserved(c, d, false), d);
                        T vb = sys.velocity_conserved(neighbor_conserved(c, d, true), d);
                        divu = divu + std::fabs(vb - va) / (T(2.0) * T(m.dx[d]));
                    }
                    source = fmax_(source, sys.dilatation_rate(w, divu));
                }
        double dt = cfl / rate;
        if (source > 0.0) dt = std::fmin(dt, 0.5 / source);
        return dt;
    }

    V7<T> totals() const {
        const Mesh& m = mesh;
        T vol = T(1.0);
        for (int d = 0; d < 3; d++)
            if (m.active(d)) vol = vol * T(m.dx[d]);
        V7<T> s{};
        for (int64_t i = 0; i < m.n[0]; i++)
            for (int64_t j = 0; j < m.n[1]; j++)
                for (int64_t k = 0; k < m.n[2]; k++) {
                    int64_t q = m.idx(i + m.g(0), j + m.g(1), k + m.g(2));
                    for (int v = 0; v < 7; v++) s[v] = s[v] + u[q][v] * vol;
                }
        return s;
    }
};

}  // namespace oracle
