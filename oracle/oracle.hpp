// CPU ORACLE — test infrastructure only.
//
// A C++ restatement of the reference CPU f64 solver for the compressible
// Euler hot path (anthony-firn/emergence, crate `fluid/crates/compressible`).
// Only the test suite, `__graft_entry__.smoke()` and the CPU-baseline leg of
// `bench.py` load it, and only as the checker / the timed CPU baseline. The
// product library (`emergence_b200/`) never links, loads or calls it.
//
// Pinning: the reference is Rust and no Rust toolchain exists here, so the
// reference itself cannot be built. This restatement is pinned instead by the
// reference's own known-answer tests, restated in `tests/test_oracle_*.py`
// (Toro star states, ghost-fill images, characteristic layers, uniform-flow
// preservation, limiter activation, CFL limit, thread-count reproducibility).
//
// Every function follows the reference's formula and operation order so that
// it is bit-compatible with it; build with `-ffp-contract=off` and without
// fast-math (FMA contraction would change roundings).
//
// Templated on the scalar type T so that the same code runs in f64 and, for
// derivative checks, in a forward-mode dual-number type.
#pragma once
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <limits>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace oracle {

// ---------------------------------------------------------------- scalar helpers
// Rust f64::max/min (maxNum/minNum: a NaN operand yields the other one).
inline double fmax_(double a, double b) { return std::fmax(a, b); }
inline double fmin_(double a, double b) { return std::fmin(a, b); }
inline bool finite_(double a) { return std::isfinite(a); }
inline double value_(double a) { return a; }

template <class T> using V5 = std::array<T, 5>;
template <class T> using Mat5 = std::array<std::array<T, 5>, 5>;

// ---------------------------------------------------------------- EOS
// fluid/crates/compressible/src/eos.rs:12-80 (Nasg)
template <class T> struct Nasg {
    T gamma, p_inf, b, q, cv;
    static Nasg ideal(T g) { return Nasg{g, T(0.0), T(0.0), T(0.0), T(1.0)}; }  // eos.rs:27-29
    // eos.rs:37-41
    T pressure(T rho, T e) const {
        T v = T(1.0) / rho;
        return (gamma - T(1.0)) * (e - q) / (v - b) - gamma * p_inf;
    }
    // eos.rs:44-48
    T energy(T rho, T p) const {
        T v = T(1.0) / rho;
        return (p + gamma * p_inf) * (v - b) / (gamma - T(1.0)) + q;
    }
    // eos.rs:51-54
    T rho_e(T rho, T p) const { return rho * energy(rho, p); }
    // eos.rs:56-60
    T sound_speed_sq(T rho, T p) const {
        T v = T(1.0) / rho;
        return gamma * (p + p_inf) * v * v / (v - b);
    }
    // eos.rs:75-79
    bool admissible(T rho, T p) const {
        return value_(rho) > 0.0 && value_(T(1.0) / rho) > value_(b) && value_(p + p_inf) > 0.0;
    }
};

// ---------------------------------------------------------------- Euler system
// fluid/crates/compressible/src/system.rs:190-414; w = (ρ,u,v,w,p), u = (ρ,ρu,ρv,ρw,E)
template <class T> struct Euler {
    Nasg<T> eos;
    static constexpr int N = 5;
    // system.rs:197-203
    V5<T> to_prim(const V5<T>& u) const {
        T rho = u[0];
        T vx = u[1] / rho, vy = u[2] / rho, vz = u[3] / rho;
        T e = u[4] / rho - T(0.5) * (vx * vx + vy * vy + vz * vz);
        return {rho, vx, vy, vz, eos.pressure(rho, e)};
    }
    // system.rs:210-217
    V5<T> to_cons(const V5<T>& w) const {
        T rho = w[0];
        T ke = T(0.5) * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
        return {rho, rho * w[1], rho * w[2], rho * w[3], eos.rho_e(rho, w[4]) + ke};
    }
    // system.rs:219-222
    T sound_speed(const V5<T>& w) const {
        using std::sqrt;
        T c2 = eos.sound_speed_sq(w[0], w[4]);
        return sqrt(fmax_(c2, T(0.0)));
    }
    int momentum_index(int d) const { return 1 + d; }  // system.rs:228-230
    // system.rs:232-258 (waves 0 = u−c, 1 entropy, 2,3 shear, 4 = u+c)
    void eigen(const V5<T>& w, int d, Mat5<T>& l, Mat5<T>& r) const {
        T rho = w[0], c = sound_speed(w);
        int un = 1 + d, t1 = 1 + (d + 1) % 3, t2 = 1 + (d + 2) % 3;
        for (auto& row : l) row.fill(T(0.0));
        for (auto& row : r) row.fill(T(0.0));
        l[0][un] = -rho / (T(2.0) * c);
        l[0][4] = T(1.0) / (T(2.0) * c * c);
        l[1][0] = T(1.0);
        l[1][4] = -T(1.0) / (c * c);
        l[2][t1] = T(1.0);
        l[3][t2] = T(1.0);
        l[4][un] = rho / (T(2.0) * c);
        l[4][4] = T(1.0) / (T(2.0) * c * c);
        r[0][0] = T(1.0);
        r[un][0] = -c / rho;
        r[4][0] = c * c;
        r[0][1] = T(1.0);
        r[t1][2] = T(1.0);
        r[t2][3] = T(1.0);
        r[0][4] = T(1.0);
        r[un][4] = c / rho;
        r[4][4] = c * c;
    }
    // physical flux of primitive w with conserved q, system.rs:268-278
    static V5<T> flux_wq(const V5<T>& w, const V5<T>& q, int un) {
        T u = w[un];
        V5<T> f;
        f[0] = q[0] * u;
        f[1] = q[1] * u;
        f[2] = q[2] * u;
        f[3] = q[3] * u;
        f[un] = f[un] + w[4];
        f[4] = (q[4] + w[4]) * u;
        return f;
    }
    // HLLC with Davis bounds, system.rs:260-312. Returns the flux; *ss the contact speed.
    V5<T> riemann_flux(const V5<T>& wl, const V5<T>& wr, int d, T* ss_out) const {
        int un = 1 + d;
        T cl = sound_speed(wl), cr = sound_speed(wr);
        T ul = wl[un], ur = wr[un];
        T sl = fmin_(ul - cl, ur - cr);
        T sr = fmax_(ul + cl, ur + cr);
        V5<T> ql = to_cons(wl), qr = to_cons(wr);
        if (value_(sl) >= 0.0) {
            if (ss_out) *ss_out = ul;
            return flux_wq(wl, ql, un);
        }
        if (value_(sr) <= 0.0) {
            if (ss_out) *ss_out = ur;
            return flux_wq(wr, qr, un);
        }
        T rl = wl[0], rr = wr[0], pl = wl[4], pr = wr[4];
        T ss = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) / (rl * (sl - ul) - rr * (sr - ur));
        auto star = [&](const V5<T>& w, const V5<T>& q, T s) {
            T rho = w[0], u = w[un];
            T fac = rho * (s - u) / (s - ss);
            V5<T> qs;
            qs[0] = fac;
            for (int k = 1; k < 4; k++) qs[k] = fac * w[k];
            qs[un] = fac * ss;
            qs[4] = fac * (q[4] / rho + (ss - u) * (ss + w[4] / (rho * (s - u))));
            return qs;
        };
        V5<T> f;
        if (value_(ss) >= 0.0) {
            V5<T> fl = flux_wq(wl, ql, un), qs = star(wl, ql, sl);
            for (int k = 0; k < 5; k++) f[k] = fl[k] + sl * (qs[k] - ql[k]);
        } else {
            V5<T> fr = flux_wq(wr, qr, un), qs = star(wr, qr, sr);
            for (int k = 0; k < 5; k++) f[k] = fr[k] + sr * (qs[k] - qr[k]);
        }
        if (ss_out) *ss_out = ss;
        return f;
    }
    // KEEP-PE two-point flux, system.rs:317-334
    V5<T> split_flux(const V5<T>& a, const V5<T>& b, int d) const {
        int un = 1 + d;
        T rho = T(0.5) * (a[0] + b[0]);
        T u = T(0.5) * (a[un] + b[un]);
        T c = rho * u;
        V5<T> f;
        f[0] = c;
        for (int k = 1; k < 4; k++) f[k] = c * T(0.5) * (a[k] + b[k]);
        f[4] = T(0.0);
        f[un] = f[un] + T(0.5) * (a[4] + b[4]);
        T kin = c * T(0.5) * (a[1] * b[1] + a[2] * b[2] + a[3] * b[3]);
        T rhoe = T(0.5) * (eos.rho_e(a[0], a[4]) + eos.rho_e(b[0], b[4]));
        T pw = T(0.5) * (a[un] * b[4] + b[un] * a[4]);
        f[4] = kin + u * rhoe + pw;
        return f;
    }
    // system.rs:336-348
    V5<T> flux(const V5<T>& w, int d) const {
        int un = 1 + d;
        V5<T> q = to_cons(w);
        T u = w[un];
        V5<T> f;
        for (int k = 0; k < 4; k++) f[k] = q[k] * u;
        f[un] = f[un] + w[4];
        f[4] = (q[4] + w[4]) * u;
        return f;
    }
    // system.rs:379-384
    V5<T> eigenvalues(const V5<T>& w, int d) const {
        T u = w[1 + d], c = sound_speed(w);
        return {u - c, u, u, u, u + c};
    }
    // system.rs:185-187
    T max_speed(const V5<T>& w, int d) const {
        using std::fabs;
        return fabs(w[1 + d]) + sound_speed(w);
    }
    // system.rs:404-407
    bool admissible(const V5<T>& w) const {
        return finite_(w[0]) && finite_(w[4]) && eos.admissible(w[0], w[4]);
    }
    // system.rs:409-413
    int sensor(const V5<T>& w, T* out) const {
        using std::log;
        out[0] = log(fmax_(w[0], T(1e-300)));
        out[1] = log(fmax_(w[4] + eos.p_inf, T(1e-300)));
        return 2;
    }
};

// ---------------------------------------------------------------- scheme
// fluid/crates/compressible/src/scheme.rs
enum FluxMode { HYBRID = 0, WENO = 1, CENTRAL = 2 };

constexpr double WENO_EPS = 1e-40;  // scheme.rs:55
// scheme.rs:89 and :92
constexpr double A6[3] = {0.75, -0.15, 1.0 / 60.0};
constexpr double S6[3] = {75.0 / 64.0 - 25.0 / 384.0 + 3.0 / 640.0, -25.0 / 384.0 + 3.0 / 640.0, 3.0 / 640.0};

// scheme.rs:76-86
template <class T>
inline T weno_z_combine(const T q[3], const double dw[3], T v0, T v1, T v2, T v3, T v4) {
    using std::fabs;
    auto sq = [](T x) { return x * x; };
    T b0 = T(13.0 / 12.0) * sq(v0 - T(2.0) * v1 + v2) + T(0.25) * sq(v0 - T(4.0) * v1 + T(3.0) * v2);
    T b1 = T(13.0 / 12.0) * sq(v1 - T(2.0) * v2 + v3) + T(0.25) * sq(v1 - v3);
    T b2 = T(13.0 / 12.0) * sq(v2 - T(2.0) * v3 + v4) + T(0.25) * sq(T(3.0) * v2 - T(4.0) * v3 + v4);
    T tau = fabs(b0 - b2);
    T a0 = T(dw[0]) * (T(1.0) + sq(tau / (b0 + T(WENO_EPS))));
    T a1 = T(dw[1]) * (T(1.0) + sq(tau / (b1 + T(WENO_EPS))));
    T a2 = T(dw[2]) * (T(1.0) + sq(tau / (b2 + T(WENO_EPS))));
    return (a0 * q[0] + a1 * q[1] + a2 * q[2]) / (a0 + a1 + a2);
}

// scheme.rs:67-74 (WENO5-Z interpolation of point values to x_{2+1/2})
template <class T> inline T weno5z_interp(T v0, T v1, T v2, T v3, T v4) {
    T q[3] = {(T(3.0) * v0 - T(10.0) * v1 + T(15.0) * v2) / T(8.0), (-v1 + T(6.0) * v2 + T(3.0) * v3) / T(8.0),
              (T(3.0) * v2 + T(6.0) * v3 - v4) / T(8.0)};
    static constexpr double dw[3] = {1.0 / 16.0, 10.0 / 16.0, 5.0 / 16.0};
    return weno_z_combine(q, dw, v0, v1, v2, v3, v4);
}

// scheme.rs:97-99
template <class T> inline T d4(T q0, T q1, T q2, T q3, T q4) {
    using std::fabs;
    return fabs(q0 - T(4.0) * q1 + T(6.0) * q2 - T(4.0) * q3 + q4);
}

struct Stats {
    uint64_t faces = 0, weno_faces = 0, fallback_faces = 0, limited_faces = 0;  // scheme.rs:101-117
    void add(const Stats& o) {
        faces += o.faces;
        weno_faces += o.weno_faces;
        fallback_faces += o.fallback_faces;
        limited_faces += o.limited_faces;
    }
};

struct SchemeOpts {
    int mode;
    double tol;
    double lambda;  // D·Δt/Δx for the positivity limiter; 0 disables (scheme.rs:119-127)
};

template <class T> struct MidResult {
    V5<T> f;
    T us;
    bool fb;
};

// Characteristic WENO5-Z interpolation to the midpoint between cells j and
// j+1, and the HLLC flux there: scheme.rs:286-333.
template <class T>
MidResult<T> midpoint_flux(const Euler<T>& sys, const V5<T>* w, int j, int d) {
    V5<T> avg;
    for (int k = 0; k < 5; k++) avg[k] = T(0.5) * (w[j][k] + w[j + 1][k]);
    Mat5<T> l, r;
    sys.eigen(avg, d, l, r);
    T ch[6][5];
    for (int s = 0; s < 6; s++) {
        const V5<T>& ws = w[j - 2 + s];
        for (int a = 0; a < 5; a++) {
            T acc = T(0.0);
            for (int k = 0; k < 5; k++) acc = acc + l[a][k] * ws[k];
            ch[s][a] = acc;
        }
    }
    T cl[5], cr[5];
    for (int a = 0; a < 5; a++) {
        cl[a] = weno5z_interp(ch[0][a], ch[1][a], ch[2][a], ch[3][a], ch[4][a]);
        cr[a] = weno5z_interp(ch[5][a], ch[4][a], ch[3][a], ch[2][a], ch[1][a]);
    }
    V5<T> wl, wr;
    for (int k = 0; k < 5; k++) {
        T sl = T(0.0), sr = T(0.0);
        for (int a = 0; a < 5; a++) {
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
    MidResult<T> m;
    m.f = sys.riemann_flux(wl, wr, d, &m.us);
    m.fb = fb;
    return m;
}

// Hu–Adams–Shu positivity limiter on the n+1 faces of a line: scheme.rs:395-464.
template <class T>
void positivity_limit(const Euler<T>& sys, const V5<T>* w, int len, int d, int ng, double lambda, V5<T>* out,
                      T* uface, Stats& stats) {
    int n = len - 2 * ng;
    V5<T> previous_cons = sys.to_cons(w[ng - 1]);
    V5<T> previous_flux = sys.flux(w[ng - 1], d);
    for (int f = 0; f <= n; f++) {
        int i = ng - 1 + f;
        V5<T> ul = previous_cons, fl_phys = previous_flux;
        V5<T> ur = sys.to_cons(w[i + 1]);
        V5<T> fr_phys = sys.flux(w[i + 1], d);
        previous_cons = ur;
        previous_flux = fr_phys;
        auto ok = [&](const V5<T>& fx) {
            V5<T> a, b;
            for (int k = 0; k < 5; k++) {
                a[k] = ul[k] - T(2.0) * T(lambda) * (fx[k] - fl_phys[k]);
                b[k] = ur[k] + T(2.0) * T(lambda) * (fx[k] - fr_phys[k]);
            }
            return sys.admissible(sys.to_prim(a)) && sys.admissible(sys.to_prim(b));
        };
        V5<T> fh = out[f];
        bool all_finite = true;
        for (int k = 0; k < 5; k++) all_finite = all_finite && finite_(fh[k]);
        if (all_finite && ok(fh)) continue;
        T alpha = fmax_(sys.max_speed(w[i], d), sys.max_speed(w[i + 1], d));
        V5<T> flf;
        for (int k = 0; k < 5; k++) flf[k] = T(0.5) * (fl_phys[k] + fr_phys[k]) - T(0.5) * alpha * (ur[k] - ul[k]);
        stats.limited_faces += 1;
        auto blend = [&](T t) {
            V5<T> v;
            for (int k = 0; k < 5; k++) v[k] = finite_(fh[k]) ? t * fh[k] + (T(1.0) - t) * flf[k] : flf[k];
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
        int un = 1 + d;
        T um = T(0.5) * (w[i][un] + w[i + 1][un]);
        if (uface) uface[f] = finite_(uface[f]) ? lo * uface[f] + (T(1.0) - lo) * um : um;
    }
}

// Face fluxes of the n+1 faces bounding the n interior cells of a line of
// primitive states (length n + 2 ng): scheme.rs:132-281 (Wcns shock path).
template <class T>
void line_fluxes(const Euler<T>& sys, const V5<T>* w, int len, int d, int ng, const SchemeOpts& o, V5<T>* out,
                 T* uface, Stats& stats) {
    int n = len - 2 * ng;
    int un = 1 + d;
    std::vector<std::array<T, 2>> sens;
    if (o.mode == HYBRID) {
        sens.resize(len);
        for (int c = 0; c < len; c++) {
            T v[8];
            sys.sensor(w[c], v);
            sens[c] = {v[0], v[1]};
        }
    }
    std::vector<MidResult<T>> mid;
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
        } else {  // scheme.rs:174-182
            T r = T(0.0);
            for (int k = 0; k < 2; k++) {
                auto s = [&](int j) { return sens[j][k]; };
                r = fmax_(fmax_(r, d4(s(i - 2), s(i - 1), s(i), s(i + 1), s(i + 2))),
                          d4(s(i - 1), s(i), s(i + 1), s(i + 2), s(i + 3)));
            }
            T x = (r / T(o.tol) - T(0.5)) / T(0.5);
            // Rust clamp(0, 1): NaN stays NaN
            if (value_(x) < 0.0) x = T(0.0);
            if (value_(x) > 1.0) x = T(1.0);
            theta = finite_(r) ? x * x * (T(3.0) - T(2.0) * x) : T(1.0);
        }
        stats.faces += 1;
        V5<T> central{T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
        T uf_c = T(0.0);
        if (value_(theta) < 1.0) {  // scheme.rs:188-223
            for (int li = 0; li < 3; li++) {
                int lag = li + 1;
                for (int m = 0; m < lag; m++) {
                    const V5<T>& wa = w[i - m];
                    const V5<T>& wb = w[i - m + lag];
                    V5<T> ft = sys.split_flux(wa, wb, d);
                    for (int k = 0; k < 5; k++) central[k] = central[k] + T(2.0) * T(A6[li]) * ft[k];
                    uf_c = uf_c + T(A6[li]) * (wa[un] + wb[un]);
                }
            }
            if (value_(theta) == 0.0) {
                out[f] = central;
                if (uface) uface[f] = uf_c;
                continue;
            }
        }
        stats.weno_faces += 1;
        // WCNS combination, scheme.rs:226-250
        V5<T> fl{T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
        T uf = T(0.0);
        for (int s = 0; s < 3; s++) {
            T c = T(S6[s]);
            int js[2] = {i + s, i - s};
            int nj = s == 0 ? 1 : 2;
            for (int q = 0; q < nj; q++) {
                int j = js[q];
                if (!have[j]) {
                    mid[j] = midpoint_flux(sys, w, j, d);
                    stats.fallback_faces += mid[j].fb ? 1 : 0;
                    have[j] = 1;
                }
                for (int k = 0; k < 5; k++) fl[k] = fl[k] + c * mid[j].f[k];
                uf = uf + c * mid[j].us;
            }
        }
        out[f] = fl;
        if (uface) uface[f] = uf;
        if (value_(theta) < 1.0) {  // scheme.rs:270-276
            for (int k = 0; k < 5; k++) out[f][k] = theta * out[f][k] + (T(1.0) - theta) * central[k];
            if (uface) uface[f] = theta * uface[f] + (T(1.0) - theta) * uf_c;
        }
    }
    if (o.lambda > 0.0) positivity_limit(sys, w, len, d, ng, o.lambda, out, uface, stats);
}

// ---------------------------------------------------------------- boundary
// fluid/crates/compressible/src/solver.rs:8-20 (Bc)
enum BcKind { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECT = 2, BC_DIRICHLET = 3, BC_CHARACTERISTIC = 4 };
template <class T> struct Bc {
    int kind = BC_PERIODIC;
    V5<T> state{};  // conserved Dirichlet / far-field state
};

// Characteristic (non-reflecting) ghost stencil: boundary.rs:48-96
template <class T> struct CharStencil {
    V5<T> wi, wf, w1;
    Mat5<T> l, r;
    bool outgoing[5];
    CharStencil() = default;
    CharStencil(const Euler<T>& sys, const V5<T>& u_b, const V5<T>& u_b1, const V5<T>& u_far, int d, int side) {
        wi = sys.to_prim(u_b);
        wf = sys.to_prim(u_far);
        w1 = sys.to_prim(u_b1);
        sys.eigen(wi, d, l, r);
        V5<T> lam = sys.eigenvalues(wi, d);
        double outward = side == 1 ? 1.0 : -1.0;
        for (int k = 0; k < 5; k++) outgoing[k] = value_(lam[k] * T(outward)) > 0.0;
    }
    V5<T> conserved(const Euler<T>& sys, double m) const {
        V5<T> dw;
        for (int k = 0; k < 5; k++) dw[k] = wi[k] - wf[k] + T(m) * (wi[k] - w1[k]);
        V5<T> wg = wf;
        for (int kf = 0; kf < 5; kf++) {
            if (outgoing[kf]) {
                // Rust `(0..N).map(..).sum()` folds from -0.0
                T amp = T(-0.0);
                for (int q = 0; q < 5; q++) amp = amp + l[kf][q] * dw[q];
                for (int q = 0; q < 5; q++) wg[q] = wg[q] + r[q][kf] * amp;
            }
        }
        return sys.to_cons(wg);
    }
};

// boundary.rs:34-44
template <class T>
V5<T> characteristic_ghost_layer(const Euler<T>& sys, const V5<T>& u_b, const V5<T>& u_b1, const V5<T>& u_far, int d,
                                 int side, double m) {
    return CharStencil<T>(sys, u_b, u_b1, u_far, d, side).conserved(sys, m);
}

// ---------------------------------------------------------------- mesh
// solver.rs:22-86
struct Mesh {
    int64_t n[3];
    double lo[3];
    double dx[3];
    int64_t ng;
    bool active(int d) const { return n[d] > 1; }
    int64_t m(int d) const { return active(d) ? n[d] + 2 * ng : 1; }
    int64_t g(int d) const { return active(d) ? ng : 0; }
    // solver.rs:62-70
    void periodic_ghost_sources(int d, int64_t gi, int64_t& lo_src, int64_t& hi_src) const {
        int64_t nn = n[d];
        if (nn >= ng) {
            lo_src = nn + gi;
            hi_src = ng + gi;
        } else {
            lo_src = ng + (gi + nn - ng % nn) % nn;
            hi_src = ng + gi % nn;
        }
    }
    int64_t idx(int64_t i, int64_t j, int64_t k) const { return (i * m(1) + j) * m(2) + k; }
    int64_t len() const { return m(0) * m(1) * m(2); }
    int64_t cells() const { return n[0] * n[1] * n[2]; }
    int ndim() const { return (int)active(0) + (int)active(1) + (int)active(2); }
};

inline int64_t rem_euclid(int64_t a, int64_t b) {
    int64_t r = a % b;
    return r < 0 ? r + b : r;
}

// Deep reflected image on a short axis: boundary.rs:98-145
template <class T, class At>
V5<T> reflected_ghost(const Euler<T>& sys, const V5<T>* states, const At& at, int64_t x, int64_t n, int64_t ng, int d,
                      const Bc<T>* bc, const CharStencil<T>* chars) {
    bool flip = false;
    V5<T> v;
    for (;;) {
        if (x >= 0 && x < n) {
            v = states[at(ng + x)];
            break;
        }
        int side = x >= n ? 1 : 0;
        int kind = bc[side].kind;
        if (kind == BC_REFLECT) {
            x = side == 0 ? -1 - x : 2 * n - 1 - x;
            flip = !flip;
        } else if (kind == BC_PERIODIC) {
            v = states[at(ng + rem_euclid(x, n))];
            break;
        } else if (kind == BC_OUTFLOW) {
            v = states[at(ng + (side == 0 ? 0 : n - 1))];
            break;
        } else if (kind == BC_DIRICHLET) {
            v = bc[side].state;
            break;
        } else {
            int64_t layer = side == 0 ? -x : x - n + 1;
            v = chars[side].conserved(sys, (double)layer);
            break;
        }
    }
    if (flip) v[sys.momentum_index(d)] = -v[sys.momentum_index(d)];
    return v;
}

// ---------------------------------------------------------------- solver
// solver.rs:139-795 (Solver, Euler system, explicit SSP-RK3 path)
template <class T> struct Solver {
    Euler<T> sys;
    Mesh mesh;
    std::vector<V5<T>> u;
    Bc<T> bc[3][2];
    double cfl = 0.5;       // solver.rs:215
    int mode = HYBRID;      // solver.rs:216
    double tol = 1e-3;      // solver.rs:218
    double t = 0.0;
    Stats stats;
    bool positivity = true;  // solver.rs:223
    double stage_dt = 0.0;
    std::vector<V5<T>> rhs_buf, stage;

    Solver(const Euler<T>& s, const Mesh& m) : sys(s), mesh(m) {
        u.assign(mesh.len(), V5<T>{T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)});
        rhs_buf = u;
        stage = u;
    }

    V5<T> prim(int64_t i, int64_t j, int64_t k) const {  // solver.rs:247-250
        const Mesh& m = mesh;
        return sys.to_prim(u[m.idx(i + m.g(0), j + m.g(1), k + m.g(2))]);
    }

    // solver.rs:259-268
    void fill_ghosts(std::vector<V5<T>>& uu) const { fill_ghosts_with(uu, bc); }
    void fill_ghosts_with(std::vector<V5<T>>& uu, const Bc<T> (&b)[3][2]) const {
        const Mesh& m = mesh;
        bool deep = false;
        for (int d = 0; d < 3; d++)
            if (m.active(d) && m.n[d] < m.ng && (b[d][0].kind == BC_REFLECT || b[d][1].kind == BC_REFLECT)) deep = true;
        fill_ghosts_impl(uu, b, deep);
    }
    // solver.rs:278-348
    void fill_ghosts_impl(std::vector<V5<T>>& uu, const Bc<T> (&b)[3][2], bool DEEP) const {
        const Mesh& m = mesh;
        for (int d = 0; d < 3; d++) {
            if (!m.active(d)) continue;
            int64_t n = m.n[d], ng = m.ng;
            int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            for (int64_t a = 0; a < m.m(e0); a++) {
                for (int64_t bb = 0; bb < m.m(e1); bb++) {
                    auto at = [&](int64_t c) {
                        int64_t ijk[3];
                        ijk[d] = c;
                        ijk[e0] = a;
                        ijk[e1] = bb;
                        return m.idx(ijk[0], ijk[1], ijk[2]);
                    };
                    CharStencil<T> chars[2];
                    if (b[d][0].kind == BC_CHARACTERISTIC)
                        chars[0] = CharStencil<T>(sys, uu[at(ng)], uu[at(ng + 1)], b[d][0].state, d, 0);
                    if (b[d][1].kind == BC_CHARACTERISTIC)
                        chars[1] = CharStencil<T>(sys, uu[at(n + ng - 1)], uu[at(n + ng - 2)], b[d][1].state, d, 1);
                    for (int64_t gi = 0; gi < ng; gi++) {
                        int64_t lo_dst = at(gi), hi_dst = at(n + ng + gi);
                        int64_t lo_s, hi_s;
                        m.periodic_ghost_sources(d, gi, lo_s, hi_s);
                        int64_t lo_src = at(lo_s), hi_src = at(hi_s);
                        int64_t lo_ref = at(2 * ng - 1 - gi), hi_ref = at(n + ng - 1 - gi);
                        V5<T> vl, vh;
                        switch (b[d][0].kind) {
                            case BC_PERIODIC: vl = uu[lo_src]; break;
                            case BC_OUTFLOW: vl = uu[at(ng)]; break;
                            case BC_DIRICHLET: vl = b[d][0].state; break;
                            case BC_CHARACTERISTIC: vl = chars[0].conserved(sys, (double)(ng - gi)); break;
                            default:
                                if (DEEP && n < ng) {
                                    vl = reflected_ghost(sys, uu.data(), at, gi - ng, n, ng, d, b[d], chars);
                                } else {
                                    vl = uu[lo_ref];
                                    vl[1 + d] = -vl[1 + d];
                                }
                        }
                        uu[lo_dst] = vl;
                        switch (b[d][1].kind) {
                            case BC_PERIODIC: vh = uu[hi_src]; break;
                            case BC_OUTFLOW: vh = uu[at(n + ng - 1)]; break;
                            case BC_DIRICHLET: vh = b[d][1].state; break;
                            case BC_CHARACTERISTIC: vh = chars[1].conserved(sys, (double)(gi + 1)); break;
                            default:
                                if (DEEP && n < ng) {
                                    vh = reflected_ghost(sys, uu.data(), at, n + gi, n, ng, d, b[d], chars);
                                } else {
                                    vh = uu[hi_ref];
                                    vh[1 + d] = -vh[1 + d];
                                }
                        }
                        uu[hi_dst] = vh;
                    }
                }
            }
        }
    }

    // Spatial residual −∇·F of `uu` (ghosts refreshed), solver.rs:351-475.
    Stats rhs(std::vector<V5<T>>& uu) {
        fill_ghosts(uu);
        const Mesh& m = mesh;
        for (auto& v : rhs_buf) v = V5<T>{T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
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
                std::vector<V5<T>> w(len);
                for (int64_t c = 0; c < len; c++) w[c] = sys.to_prim(uu[at(c)]);
                std::vector<V5<T>> fl(m.n[d] + 1);
                Stats s;
                line_fluxes(sys, w.data(), (int)len, d, (int)m.ng, opts, fl.data(), (T*)nullptr, s);
                T inv = T(1.0) / T(m.dx[d]);
                for (int64_t c = 0; c < m.n[d]; c++) {
                    V5<T>& o = rhs_buf[at(c + m.ng)];
                    for (int k = 0; k < 5; k++) o[k] = o[k] - (fl[c + 1][k] - fl[c][k]) * inv;
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

    // solver.rs:97-137
    template <int STAGE>
    void rk_combine(std::vector<V5<T>>& dest, const std::vector<V5<T>>& old, double dt) const {
        const Mesh& m = mesh;
#pragma omp parallel for schedule(static)
        for (int64_t i = m.g(0); i < m.g(0) + m.n[0]; i++)
            for (int64_t j = m.g(1); j < m.g(1) + m.n[1]; j++)
                for (int64_t k = m.g(2); k < m.g(2) + m.n[2]; k++) {
                    int64_t q = m.idx(i, j, k);
                    for (int v = 0; v < 5; v++) {
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

    // One SSP-RK3 step (Shu–Osher form), solver.rs:659-738 (Euler path).
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

    // CFL rate max_cells Σ_d max_speed/dx_d over interior cells (solver.rs:478-523)
    double cfl_rate() const {
        const Mesh& m = mesh;
        double rate = 0.0;
#pragma omp parallel for reduction(max : rate) schedule(static)
        for (int64_t i = 0; i < m.n[0]; i++)
            for (int64_t j = 0; j < m.n[1]; j++)
                for (int64_t k = 0; k < m.n[2]; k++) {
                    V5<T> w = sys.to_prim(u[m.idx(i + m.g(0), j + m.g(1), k + m.g(2))]);
                    T acoustic = T(-0.0);
                    for (int d = 0; d < 3; d++)
                        if (m.active(d)) acoustic = acoustic + sys.max_speed(w, d) / T(m.dx[d]);
                    rate = fmax_(rate, value_(acoustic));
                }
        return rate;
    }
    double dt_cfl() const { return cfl / cfl_rate(); }

    // solver.rs:758-768; returns the number of steps, or -1 when dt collapsed
    int64_t run_to(double t_end) {
        int64_t steps = 0;
        while (t < t_end - 1e-10 * std::fabs(t_end)) {
            double dt = std::fmin(dt_cfl(), t_end - t);
            if (!(std::isfinite(dt) && dt > 1e-12 * std::fmax(std::fabs(t_end), 1e-300))) return -1;
            step(dt);
            steps += 1;
        }
        return steps;
    }

    // solver.rs:784-794
    V5<T> totals() const {
        const Mesh& m = mesh;
        T vol = T(1.0);
        for (int d = 0; d < 3; d++)
            if (m.active(d)) vol = vol * T(m.dx[d]);
        V5<T> s{T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
        for (int64_t i = 0; i < m.n[0]; i++)
            for (int64_t j = 0; j < m.n[1]; j++)
                for (int64_t k = 0; k < m.n[2]; k++) {
                    int64_t q = m.idx(i + m.g(0), j + m.g(1), k + m.g(2));
                    for (int v = 0; v < 5; v++) s[v] = s[v] + u[q][v] * vol;
                }
        return s;
    }
};

// ---------------------------------------------------------------- exact Riemann solver
// fluid/crates/compressible/src/exact.rs:9-109 (stiffened gas per side, Toro ch. 4)
struct Side {
    double rho, u, p;
    Nasg<double> eos;
};
struct Star {
    double p, u, rho_l, rho_r;
};
inline void f_k(double p, const Side& s, double& f, double& df) {  // exact.rs:26-42
    double g = s.eos.gamma, pi = s.eos.p_inf;
    double c = std::sqrt(g * (s.p + pi) / s.rho);
    double pk = s.p + pi, ps = p + pi;
    if (p > s.p) {
        double a = 2.0 / ((g + 1.0) * s.rho);
        double b = (g - 1.0) / (g + 1.0) * pk;
        double q = std::sqrt(a / (ps + b));
        f = (p - s.p) * q;
        df = q * (1.0 - 0.5 * (p - s.p) / (ps + b));
    } else {
        double r = ps / pk;
        f = 2.0 * c / (g - 1.0) * (std::pow(r, (g - 1.0) / (2.0 * g)) - 1.0);
        df = 1.0 / (s.rho * c) * std::pow(r, -(g + 1.0) / (2.0 * g));
    }
}
inline Star star(const Side& l, const Side& r) {  // exact.rs:45-76
    double du = r.u - l.u;
    double pmin = -(std::fmin(l.eos.p_inf, r.eos.p_inf)) + 1e-12 * (1.0 + std::fabs(l.p) + std::fabs(r.p));
    double p = std::fmax(0.5 * (l.p + r.p), pmin + 1e-8);
    for (int it = 0; it < 200; it++) {
        double fl, dl, fr, dr;
        f_k(p, l, fl, dl);
        f_k(p, r, fr, dr);
        double pn = p - (fl + fr + du) / (dl + dr);
        if (pn <= pmin) pn = 0.5 * (p + pmin);
        if (std::fabs(pn - p) <= 1e-14 * (std::fabs(pn) + std::fmax(l.eos.p_inf, r.eos.p_inf))) {
            p = pn;
            break;
        }
        p = pn;
    }
    double fl, dl, fr, dr;
    f_k(p, l, fl, dl);
    f_k(p, r, fr, dr);
    double u = 0.5 * (l.u + r.u) + 0.5 * (fr - fl);
    auto rho_star = [&](const Side& s) {
        double g = s.eos.gamma, pi = s.eos.p_inf;
        double ratio = (p + pi) / (s.p + pi);
        if (p > s.p) {
            double gr = (g - 1.0) / (g + 1.0);
            return s.rho * (ratio + gr) / (gr * ratio + 1.0);
        }
        return s.rho * std::pow(ratio, 1.0 / g);
    };
    return Star{p, u, rho_star(l), rho_star(r)};
}
// exact.rs:80-109: (rho, u, p) at xi = x/t; returns the side (0 left of the contact)
inline int sample(const Side& l, const Side& r, const Star& st, double xi, double out[3]) {
    bool left = xi <= st.u;
    const Side& s = left ? l : r;
    double sign = left ? 1.0 : -1.0;
    double rho_s = left ? st.rho_l : st.rho_r;
    double g = s.eos.gamma, pi = s.eos.p_inf;
    double c = std::sqrt(g * (s.p + pi) / s.rho);
    double u = sign * s.u, x = sign * xi, us = sign * st.u;
    int side = left ? 0 : 1;
    if (st.p > s.p) {
        double ratio = (st.p + pi) / (s.p + pi);
        double sh = u - c * std::sqrt((g + 1.0) / (2.0 * g) * ratio + (g - 1.0) / (2.0 * g));
        if (x <= sh) {
            out[0] = s.rho; out[1] = s.u; out[2] = s.p;
        } else {
            out[0] = rho_s; out[1] = st.u; out[2] = st.p;
        }
        return side;
    }
    double cs = c * std::pow((st.p + pi) / (s.p + pi), (g - 1.0) / (2.0 * g));
    double head = u - c, tail = us - cs;
    if (x <= head) {
        out[0] = s.rho; out[1] = s.u; out[2] = s.p;
    } else if (x >= tail) {
        out[0] = rho_s; out[1] = st.u; out[2] = st.p;
    } else {
        double k = 2.0 / (g + 1.0) + (g - 1.0) / ((g + 1.0) * c) * (u - x);
        out[0] = s.rho * std::pow(k, 2.0 / (g - 1.0));
        double uu = 2.0 / (g + 1.0) * (c + (g - 1.0) / 2.0 * u + x);
        out[1] = sign * uu;
        out[2] = (s.p + pi) * std::pow(k, 2.0 * g / (g - 1.0)) - pi;
    }
    return side;
}

}  // namespace oracle
