// Device physics of the two-phase five-equation system (Kapila's model):
// conserved (α1ρ1, α2ρ2, ρu, ρv, ρw, E, α1), primitive (α1ρ1, α2ρ2, u, v, w,
// p, α1), one NASG equation of state per phase.
//
// Formulas and operation order follow fluid/crates/compressible/src/
// multiphase.rs so that, compiled without FMA contraction, every value rounds
// as the reference CPU solver's does. The eigenvector products of the
// characteristic projection skip the zero entries but keep the order of the
// non-zero terms of the reference's dense loops.
#pragma once
#include "physics.cuh"

namespace emg {

constexpr int NF = 7;  // variables of the five-equation system
constexpr int F_IP = 5, F_IA = 6, F_IU = 2;

struct FiveSysD {
    EosD e[2];
    int kapila;
};

// a/b: correctly rounded in the plain form, a·(1/b) with the one-ulp
// reciprocal of physics.cuh in the fast FP64 form (F)
template <bool F> __device__ __forceinline__ double fdiv(double a, double b) {
    if constexpr (F)
        return a * rcp_f(b);
    else
        return a / b;
}
template <bool F> __device__ __forceinline__ double fsqrt(double x) {
    if constexpr (F)
        return sqrt_f(x);
    else
        return sqrt(x);
}

// Methods templated on F: the plain form (F false, the reference's operation
// order, bit-exact without FMA contraction) or the fast FP64 form (F true,
// one-ulp reciprocals and square roots, 1/(γ − 1) of each phase precomputed).
struct Five {
    Eos<double> e1, e2;
    bool kapila;
    double igm[2];  // 1/(γ − 1) of each phase (fast form)
    __device__ static Five from(const FiveSysD& s) {
        return Five{Eos<double>::from(s.e[0]), Eos<double>::from(s.e[1]), s.kapila != 0,
                    {1.0 / (s.e[0].gamma - 1.0), 1.0 / (s.e[1].gamma - 1.0)}};
    }
    __device__ __forceinline__ const Eos<double>& eos(int k) const { return k == 0 ? e1 : e2; }

    // multiphase.rs:58-69
    template <bool F = false> __device__ __forceinline__ void db(const double* w, double& d, double& b) const {
        const double al[2] = {w[F_IA], 1.0 - w[F_IA]};
        d = 0.0;
        b = 0.0;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const Eos<double>& e = eos(k);
            const double vol = al[k] - e.b * w[k];
            if constexpr (F) {
                d = d + vol * igm[k];
                b = b + e.gamma * e.p_inf * vol * igm[k] + e.q * w[k];
            } else {
                d = d + vol / (e.gamma - 1.0);
                b = b + e.gamma * e.p_inf * vol / (e.gamma - 1.0) + e.q * w[k];
            }
        }
    }
    __device__ __forceinline__ double rho_e(const double* w) const {
        double d, b;
        db(w, d, b);
        return w[F_IP] * d + b;
    }
    // multiphase.rs:77-84
    template <bool F = false> __device__ __forceinline__ double rho_c2_phase(const double* w, int k) const {
        const double al = k == 0 ? w[F_IA] : 1.0 - w[F_IA];
        const Eos<double>& e = eos(k);
        if (F && e.b == 0.0) return e.gamma * (w[F_IP] + e.p_inf);  // fmax(1 − 0, 1e-12) = 1
        const double rk = (al > 1e-12 && w[k] > 0.0) ? fdiv<F>(w[k], al) : 0.0;
        return fdiv<F>(e.gamma * (w[F_IP] + e.p_inf), fmax(1.0 - e.b * rk, 1e-12));
    }
    // multiphase.rs:86-97 (Rust clamp: NaN stays NaN)
    template <bool F = false> __device__ __forceinline__ double kapila_k(const double* w) const {
        if (!kapila) return 0.0;
        double a = w[F_IA];
        if (a < 0.0) a = 0.0;
        if (a > 1.0) a = 1.0;
        const double al0 = a, al1 = 1.0 - a;
        const double z1 = rho_c2_phase<F>(w, 0), z2 = rho_c2_phase<F>(w, 1);
        const double den = al1 * z1 + al0 * z2;
        if (den <= 0.0) return 0.0;
        return fdiv<F>(al0 * al1 * (z2 - z1), den);
    }
    // multiphase.rs:113-117
    template <bool F = false> __device__ __forceinline__ double drhoe_dalpha(double p) const {
        if constexpr (F)
            return (p + e1.gamma * e1.p_inf) * igm[0] - (p + e2.gamma * e2.p_inf) * igm[1];
        else
            return (p + e1.gamma * e1.p_inf) / (e1.gamma - 1.0) - (p + e2.gamma * e2.p_inf) / (e2.gamma - 1.0);
    }
    // multiphase.rs:100-110, from the closure values d, b of w and K = kapila_k(w)
    // (every term as the reference evaluates it; the reference recomputes d and
    // b inside rho_e, which gives the same values)
    template <bool F = false>
    __device__ __forceinline__ double rho_c2_db(const double* w, double d, double b, double kk) const {
        const double p = w[F_IP];
        double num = (w[F_IP] * d + b) + p;
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const Eos<double>& e = eos(k);
            if constexpr (F)
                num = num + w[k] * (e.b * (p + e.gamma * e.p_inf) * igm[k] - e.q);
            else
                num = num + w[k] * (e.b * (p + e.gamma * e.p_inf) / (e.gamma - 1.0) - e.q);
        }
        num = num + kk * drhoe_dalpha<F>(p);
        return fdiv<F>(num, d);
    }
    __device__ __forceinline__ double rho_c2(const double* w) const {
        double d, b;
        db(w, d, b);
        return rho_c2_db(w, d, b, kapila_k(w));
    }
    // closure values of a primitive state, computed once where a state is
    // tested, given a sound speed and converted to conserved variables
    struct St {
        double d, b, rc2;
    };
    template <bool F = false> __device__ __forceinline__ St state(const double* w) const {
        St st;
        db<F>(w, st.d, st.b);
        st.rc2 = rho_c2_db<F>(w, st.d, st.b, kapila_k<F>(w));
        return st;
    }
    __device__ __forceinline__ static double rho(const double* w) { return w[0] + w[1]; }
    // multiphase.rs:127-130
    __device__ __forceinline__ double p_inf_mix(const double* w) const {
        double a = w[F_IA];
        if (a < 0.0) a = 0.0;
        if (a > 1.0) a = 1.0;
        return a * e1.p_inf + (1.0 - a) * e2.p_inf;
    }
    // multiphase.rs:131-146; d, b: the closure values of the result (db does
    // not read the pressure)
    template <bool F = false>
    __device__ __forceinline__ void to_prim_db(const double* u, double* w, double& d, double& b) const {
        const double r = u[0] + u[1];
        double vx, vy, vz;
        if constexpr (F) {
            const double ir = rcp_f(r);
            vx = u[2] * ir;
            vy = u[3] * ir;
            vz = u[4] * ir;
        } else {
            vx = u[2] / r;
            vy = u[3] / r;
            vz = u[4] / r;
        }
        w[0] = u[0];
        w[1] = u[1];
        w[2] = vx;
        w[3] = vy;
        w[4] = vz;
        w[F_IA] = u[6];
        const double rhoe = u[5] - 0.5 * r * (vx * vx + vy * vy + vz * vz);
        db<F>(w, d, b);
        w[F_IP] = fdiv<F>(rhoe - b, d);
    }
    __device__ __forceinline__ void to_prim(const double* u, double* w) const {
        double d, b;
        to_prim_db(u, w, d, b);
    }
    // multiphase.rs:152-163
    __device__ __forceinline__ void to_cons_db(const double* w, double d, double b, double* u) const {
        const double r = w[0] + w[1];
        u[0] = w[0];
        u[1] = w[1];
        u[2] = r * w[2];
        u[3] = r * w[3];
        u[4] = r * w[4];
        u[5] = (w[F_IP] * d + b) + 0.5 * r * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
        u[6] = w[F_IA];
    }
    template <bool F = false> __device__ __forceinline__ void to_cons(const double* w, double* u) const {
        double d, b;
        db<F>(w, d, b);
        to_cons_db(w, d, b, u);
    }
    template <bool F = false> __device__ __forceinline__ static double sound_speed_rc2(const double* w, double rc2) {
        return fsqrt<F>(fdiv<F>(fmax(rc2, 0.0), rho(w)));
    }
    __device__ __forceinline__ double sound_speed(const double* w) const { return sound_speed_rc2(w, rho_c2(w)); }
    // multiphase.rs:345-350, with ρc² of w
    __device__ __forceinline__ static bool admissible_rc2(const double* w, double rc2) {
#pragma unroll
        for (int k = 0; k < NF; k++)
            if (!isfinite(w[k])) return false;
        return rho(w) > 0.0 && w[F_IA] >= -0.05 && w[F_IA] <= 1.05 && rc2 > 0.0;
    }
    __device__ __forceinline__ bool admissible(const double* w) const { return admissible_rc2(w, rho_c2(w)); }
    // multiphase.rs:331-343, from primitive w and its conserved q
    __device__ __forceinline__ static void flux_wq(const double* w, const double* q, int un, double* f) {
        const double u = w[un];
#pragma unroll
        for (int k = 0; k < 5; k++) f[k] = q[k] * u;
        f[un] = f[un] + w[F_IP];
        f[5] = (q[5] + w[F_IP]) * u;
        f[6] = w[F_IA] * u;
    }
    // multiphase.rs:245-289 (HLLC, Davis bounds) with the closure values of
    // both states; returns the contact speed
    template <bool F = false>
    __device__ __forceinline__ double riemann_st(const double* wl, const double* wr, const St& stl, const St& str_,
                                                 int un, double* f) const {
        const double cl = sound_speed_rc2<F>(wl, stl.rc2), cr = sound_speed_rc2<F>(wr, str_.rc2);
        const double ul = wl[un], ur = wr[un];
        const double sl = fmin(ul - cl, ur - cr);
        const double sr = fmax(ul + cl, ur + cr);
        double ql[NF], qr[NF];
        to_cons_db(wl, stl.d, stl.b, ql);
        to_cons_db(wr, str_.d, str_.b, qr);
        if (sl >= 0.0) {
            flux_wq(wl, ql, un, f);
            return ul;
        }
        if (sr <= 0.0) {
            flux_wq(wr, qr, un, f);
            return ur;
        }
        const double rl = rho(wl), rr = rho(wr);
        const double pl = wl[F_IP], pr = wr[F_IP];
        const double ss = fdiv<F>(pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur), rl * (sl - ul) - rr * (sr - ur));
        const bool left = ss >= 0.0;
        const double* w = left ? wl : wr;
        const double* q = left ? ql : qr;
        const double s = left ? sl : sr;
        double fx[NF];
        flux_wq(w, q, un, fx);
        const double rh = rho(w), u = w[un];
        const double fac = fdiv<F>(s - u, s - ss);
        double qs[NF];
        qs[0] = w[0] * fac;
        qs[1] = w[1] * fac;
        qs[2] = rh * fac * w[2];
        qs[3] = rh * fac * w[3];
        qs[4] = rh * fac * w[4];
        qs[un] = rh * fac * ss;
        qs[5] = rh * fac * (fdiv<F>(q[5], rh) + (ss - u) * (ss + fdiv<F>(w[F_IP], rh * (s - u))));
        qs[6] = w[F_IA] * fac;
#pragma unroll
        for (int k = 0; k < NF; k++) f[k] = fx[k] + s * (qs[k] - q[k]);
        return ss;
    }
    __device__ __forceinline__ double riemann(const double* wl, const double* wr, int un, double* f) const {
        return riemann_st(wl, wr, state(wl), state(wr), un, f);
    }
    template <bool F = false> __device__ __forceinline__ double nc_coef(const double* w) const {
        return w[F_IA] + kapila_k<F>(w);
    }
    // multiphase.rs:363-377, with ρc² of w
    __device__ __forceinline__ double dilatation_rate_rc2(const double* w, double divu, double rc2) const {
        const double a = w[F_IA];
        double pmin = INFINITY;
        if (a > 1e-6) pmin = fmin(pmin, e1.p_inf);
        if (1.0 - a > 1e-6) pmin = fmin(pmin, e2.p_inf);
        const double floor_ = 1e-6 * fmax(e1.p_inf, e2.p_inf);
        const double head = fmax(fmax(w[F_IP] + pmin, floor_), 1e-300);
        return fmax(rc2, 0.0) * fabs(divu) / head;
    }
    __device__ __forceinline__ double dilatation_rate(const double* w, double divu) const {
        return dilatation_rate_rc2(w, divu, rho_c2(w));
    }
    // velocity component from a conserved state (multiphase.rs:148-150)
    __device__ __forceinline__ static double velocity_conserved(const double* u, int d) { return u[2 + d] / (u[0] + u[1]); }
};

// Dense characteristic stencil of the five-equation system for the
// non-reflecting ghost layers (boundary.rs:48-96 with multiphase.rs:202-243).
struct CharStencil7D {
    double wi[NF], wf[NF], w1[NF];
    double l[NF][NF], r[NF][NF];
    bool outgoing[NF];
    __device__ void init(const Five& s, const double* ub, const double* ub1, const double* uf, int d, int side) {
        s.to_prim(ub, wi);
        s.to_prim(uf, wf);
        s.to_prim(ub1, w1);
        const double rh = Five::rho(wi), c = s.sound_speed(wi), kk = s.kapila_k(wi);
        const int un = F_IU + d, t1 = F_IU + (d + 1) % 3, t2 = F_IU + (d + 2) % 3;
        for (int i = 0; i < NF; i++)
            for (int j = 0; j < NF; j++) l[i][j] = r[i][j] = 0.0;
        const double c2 = c * c;
        l[0][0] = 1.0;
        l[0][F_IP] = -wi[0] / rh / c2;
        l[1][1] = 1.0;
        l[1][F_IP] = -wi[1] / rh / c2;
        l[2][un] = -rh / (2.0 * c);
        l[2][F_IP] = 1.0 / (2.0 * c2);
        l[3][t1] = 1.0;
        l[4][t2] = 1.0;
        l[5][un] = rh / (2.0 * c);
        l[5][F_IP] = 1.0 / (2.0 * c2);
        l[6][F_IA] = 1.0;
        l[6][F_IP] = kk / rh / c2;
        r[0][0] = 1.0;
        r[1][1] = 1.0;
        r[t1][3] = 1.0;
        r[t2][4] = 1.0;
        r[F_IA][6] = 1.0;
        const int cols[2] = {2, 5};
        const double sg[2] = {-1.0, 1.0};
        for (int m = 0; m < 2; m++) {
            const int col = cols[m];
            r[0][col] = wi[0] / rh;
            r[1][col] = wi[1] / rh;
            r[un][col] = sg[m] * c / rh;
            r[F_IP][col] = c2;
            r[F_IA][col] = -kk / rh;
        }
        const double u = wi[un];
        const double lam[NF] = {u, u, u - c, u, u, u + c, u};
        const double outward = side == 1 ? 1.0 : -1.0;
        for (int k = 0; k < NF; k++) outgoing[k] = lam[k] * outward > 0.0;
    }
    __device__ void conserved(const Five& s, double m, double* out) const {
        double dw[NF], wg[NF];
        for (int k = 0; k < NF; k++) dw[k] = wi[k] - wf[k] + m * (wi[k] - w1[k]);
        for (int k = 0; k < NF; k++) wg[k] = wf[k];
        for (int kf = 0; kf < NF; kf++) {
            if (outgoing[kf]) {
                double amp = -0.0;
                for (int q = 0; q < NF; q++) amp = amp + l[kf][q] * dw[q];
                for (int q = 0; q < NF; q++) wg[q] = wg[q] + r[q][kf] * amp;
            }
        }
        s.to_cons(wg, out);
    }
};

}  // namespace emg
