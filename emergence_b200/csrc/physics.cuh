// Device-side physics of the compressible Euler step: NASG equation of state,
// Euler conserved/primitive maps, primitive characteristic eigenvectors,
// WENO5-Z interpolation and the HLLC flux.
//
// Formulas and their operation order follow the reference CPU solver
// (fluid/crates/compressible/src/{eos,system,scheme}.rs) so that the plain FP64
// instantiation, compiled without FMA contraction, rounds exactly as the CPU
// does. The same templates instantiated with R = float give the FP32 flux
// arithmetic of the mixed-precision form.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace emg {

// Bounds-check build (compiled with -DEMG_BOUNDS_CHECK into
// libemergence_b200_bc.so): every global index of the sweeps, the uniform
// ghost fill and the AMR pool loads and RK update is checked against its
// array before the access; an index out of range skips the access and raises
// EMG_ERR_BOUNDS in the control block (or bit 4 of the AMR error word),
// which the host reports after the call. Nothing traps. In the product build
// the checks compile to nothing.
#ifdef EMG_BOUNDS_CHECK
constexpr bool BOUNDS_CHECK = true;
#else
constexpr bool BOUNDS_CHECK = false;
#endif
constexpr int STATUS_BOUNDS = 6;  // EMG_ERR_BOUNDS

// NASG parameters (fluid/crates/compressible/src/eos.rs:12-25).
struct EosD {
    double gamma, p_inf, b, q;
};

template <typename R> struct Eos {
    R gamma, p_inf, b, q;
    __host__ __device__ static Eos from(const EosD& e) { return Eos{R(e.gamma), R(e.p_inf), R(e.b), R(e.q)}; }
    // eos.rs:37-41
    __device__ __forceinline__ R pressure(R rho, R e) const {
        R v = R(1) / rho;
        return (gamma - R(1)) * (e - q) / (v - b) - gamma * p_inf;
    }
    // eos.rs:44-54 (ρe = ρ·energy(ρ, p))
    __device__ __forceinline__ R rho_e(R rho, R p) const {
        R v = R(1) / rho;
        return rho * ((p + gamma * p_inf) * (v - b) / (gamma - R(1)) + q);
    }
    // eos.rs:56-60
    __device__ __forceinline__ R sound_speed_sq(R rho, R p) const {
        R v = R(1) / rho;
        return gamma * (p + p_inf) * v * v / (v - b);
    }
};

template <typename R> __device__ __forceinline__ R rmax(R a, R b) { return fmax(a, b); }
template <typename R> __device__ __forceinline__ R rmin(R a, R b) { return fmin(a, b); }
__device__ __forceinline__ float rmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float rmin(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double rsqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float rsqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double rabs(double x) { return fabs(x); }
__device__ __forceinline__ float rabs(float x) { return fabsf(x); }

// Euler system, w = (ρ,u,v,w,p), u = (ρ,ρu,ρv,ρw,E): system.rs:196-217.
template <typename R> __device__ __forceinline__ void to_prim(const Eos<R>& e, const R* u, R* w) {
    R rho = u[0];
    R vx = u[1] / rho, vy = u[2] / rho, vz = u[3] / rho;
    R ein = u[4] / rho - R(0.5) * (vx * vx + vy * vy + vz * vz);
    w[0] = rho;
    w[1] = vx;
    w[2] = vy;
    w[3] = vz;
    w[4] = e.pressure(rho, ein);
}
template <typename R> __device__ __forceinline__ void to_cons(const Eos<R>& e, const R* w, R* u) {
    R rho = w[0];
    R ke = R(0.5) * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
    u[0] = rho;
    u[1] = rho * w[1];
    u[2] = rho * w[2];
    u[3] = rho * w[3];
    u[4] = e.rho_e(rho, w[4]) + ke;
}
// system.rs:219-222
template <typename R> __device__ __forceinline__ R sound_speed(const Eos<R>& e, R rho, R p) {
    return rsqrt_(rmax(e.sound_speed_sq(rho, p), R(0)));
}
// system.rs:404-407 with eos.rs:75-79
template <typename R> __device__ __forceinline__ bool admissible(const Eos<R>& e, R rho, R p) {
    return isfinite(rho) && isfinite(p) && rho > R(0) && R(1) / rho > e.b && p + e.p_inf > R(0);
}
// physical flux from primitive w and its conserved q along normal index un (system.rs:268-278)
template <typename R> __device__ __forceinline__ void flux_wq(const R* w, const R* q, int un, R* f) {
    R u = w[un];
    f[0] = q[0] * u;
    f[1] = q[1] * u;
    f[2] = q[2] * u;
    f[3] = q[3] * u;
    f[un] = f[un] + w[4];
    f[4] = (q[4] + w[4]) * u;
}

// HLLC with Davis wave-speed bounds (system.rs:260-312). Returns the contact speed.
template <typename R>
__device__ __forceinline__ R hllc(const Eos<R>& e, const R* wl, const R* wr, int un, R* f) {
    R cl = sound_speed(e, wl[0], wl[4]), cr = sound_speed(e, wr[0], wr[4]);
    R ul = wl[un], ur = wr[un];
    R sl = rmin(ul - cl, ur - cr);
    R sr = rmax(ul + cl, ur + cr);
    R ql[5], qr[5];
    to_cons(e, wl, ql);
    to_cons(e, wr, qr);
    if (sl >= R(0)) {
        flux_wq(wl, ql, un, f);
        return ul;
    }
    if (sr <= R(0)) {
        flux_wq(wr, qr, un, f);
        return ur;
    }
    R rl = wl[0], rr = wr[0], pl = wl[4], pr = wr[4];
    R ss = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) / (rl * (sl - ul) - rr * (sr - ur));
    const bool left = ss >= R(0);
    const R* w = left ? wl : wr;
    const R* q = left ? ql : qr;
    R s = left ? sl : sr;
    R fx[5];
    flux_wq(w, q, un, fx);
    R rho = w[0], u = w[un];
    R fac = rho * (s - u) / (s - ss);
    R qs[5];
    qs[0] = fac;
    qs[1] = fac * w[1];
    qs[2] = fac * w[2];
    qs[3] = fac * w[3];
    qs[un] = fac * ss;
    qs[4] = fac * (q[4] / rho + (ss - u) * (ss + w[4] / (rho * (s - u))));
#pragma unroll
    for (int k = 0; k < 5; k++) f[k] = fx[k] + s * (qs[k] - q[k]);
    return ss;
}

// Reciprocal and reciprocal square root of the mixed form, FP64 to about
// 1e-12 relative instead of correctly rounded: the PTX estimate
// (rcp.approx.ftz.f64 / rsqrt.approx.ftz.f64, good to about 2^-20) refined by
// one Newton–Raphson step, which squares the estimate's relative error
// (measured on a B200: at most 9.7e-13 and 1.24e-12 over 2^20 inputs). For 1/y, Newton's method
// on g(r) = 1/r − y gives r ← r + r·(1 − y·r); for 1/√x, on g(r) = 1/r² − x it
// gives r ← r + (r/2)·(1 − x·r²). Zero, infinite and NaN inputs give
// non-finite results, which the admissibility tests and the limiter treat as
// they treat the correctly rounded quotients' infinities. Subnormal inputs are
// flushed to zero. Only the mixed form uses these: the plain FP64 form keeps
// IEEE division and square root for bitwise parity with the CPU solver.
__device__ __forceinline__ double rcp_nr(double y) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
    const double h = fma(-y, r, 1.0);
    return fma(r, h, r);
}
__device__ __forceinline__ double rsqrt_nr(double x) {
    double r;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double xr = x * r;
    const double h = fma(-xr, r, 1.0);
    return fma(0.5 * r, h, r);
}

// Conserved state of the mixed form with 1/ρ and 1/(γ−1) given (eos.rs:44-54).
__device__ __forceinline__ void to_cons_nr(const Eos<double>& e, const double* w, double irho, double igm1, double* u) {
    const double rho = w[0];
    const double ke = 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
    u[0] = rho;
    u[1] = rho * w[1];
    u[2] = rho * w[2];
    u[3] = rho * w[3];
    u[4] = rho * ((w[4] + e.gamma * e.p_inf) * (irho - e.b) * igm1 + e.q) + ke;
}

// Admissibility of the mixed form (system.rs:404-407 with eos.rs:75-79).
__device__ __forceinline__ bool admissible_nr(const Eos<double>& e, double rho, double p) {
    return isfinite(rho) && isfinite(p) && rho > 0.0 && rcp_nr(rho) > e.b && p + e.p_inf > 0.0;
}

// HLLC of the mixed form: the Davis wave-speed bounds from FP32 sound speeds,
// the conserved states, physical fluxes, contact speed and star states in
// FP64 with the Newton-refined reciprocals above in place of divisions. An
// error in a wave speed enters the flux multiplied by a jump of the state
// across the midpoint, so it vanishes where the data are smooth; the
// reciprocals' 1e-12 stays far below the FP32 interpolation error.
__device__ __forceinline__ double hllc_fs(const Eos<double>& e, const double* wl, const double* wr, int un, double* f) {
    const Eos<float> ef{(float)e.gamma, (float)e.p_inf, (float)e.b, (float)e.q};
    const double cl = (double)sound_speed(ef, (float)wl[0], (float)wl[4]);
    const double cr = (double)sound_speed(ef, (float)wr[0], (float)wr[4]);
    double ul = wl[un], ur = wr[un];
    double sl = fmin(ul - cl, ur - cr);
    double sr = fmax(ul + cl, ur + cr);
    const double igm1 = rcp_nr(e.gamma - 1.0);
    const double irl = rcp_nr(wl[0]), irr = rcp_nr(wr[0]);
    double ql[5], qr[5];
    to_cons_nr(e, wl, irl, igm1, ql);
    to_cons_nr(e, wr, irr, igm1, qr);
    if (sl >= 0.0) {
        flux_wq(wl, ql, un, f);
        return ul;
    }
    if (sr <= 0.0) {
        flux_wq(wr, qr, un, f);
        return ur;
    }
    double rl = wl[0], rr = wr[0], pl = wl[4], pr = wr[4];
    double ss = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) * rcp_nr(rl * (sl - ul) - rr * (sr - ur));
    const bool left = ss >= 0.0;
    const double* w = left ? wl : wr;
    const double* q = left ? ql : qr;
    const double irho = left ? irl : irr;
    double s = left ? sl : sr;
    double fx[5];
    flux_wq(w, q, un, fx);
    double rho = w[0], u = w[un];
    const double smu = s - u;
    double fac = rho * smu * rcp_nr(s - ss);
    double qs[5];
    qs[0] = fac;
    qs[1] = fac * w[1];
    qs[2] = fac * w[2];
    qs[3] = fac * w[3];
    qs[un] = fac * ss;
    qs[4] = fac * (q[4] * irho + (ss - u) * (ss + w[4] * irho * rcp_nr(smu)));
#pragma unroll
    for (int k = 0; k < 5; k++) f[k] = fx[k] + s * (qs[k] - q[k]);
    return ss;
}

// WENO-Z combination (scheme.rs:76-86); eps 1e-40 in f64 (scheme.rs:55), 1e-30 in f32.
template <typename R> struct WenoEps;
template <> struct WenoEps<double> { static constexpr double v = 1e-40; };
template <> struct WenoEps<float> { static constexpr float v = 1e-30f; };

template <typename R> __device__ __forceinline__ R sq(R x) { return x * x; }

// WENO5-Z interpolation of point values to the midpoint x_{2+1/2} (scheme.rs:67-74).
template <typename R> __device__ __forceinline__ R weno5z_interp(R v0, R v1, R v2, R v3, R v4) {
    const R eps = WenoEps<R>::v;
    // x/8 == x*0.125 exactly (power-of-two scaling)
    R q0 = (R(3) * v0 - R(10) * v1 + R(15) * v2) * R(0.125);
    R q1 = (-v1 + R(6) * v2 + R(3) * v3) * R(0.125);
    R q2 = (R(3) * v2 + R(6) * v3 - v4) * R(0.125);
    R b0 = R(13.0 / 12.0) * sq(v0 - R(2) * v1 + v2) + R(0.25) * sq(v0 - R(4) * v1 + R(3) * v2);
    R b1 = R(13.0 / 12.0) * sq(v1 - R(2) * v2 + v3) + R(0.25) * sq(v1 - v3);
    R b2 = R(13.0 / 12.0) * sq(v2 - R(2) * v3 + v4) + R(0.25) * sq(R(3) * v2 - R(4) * v3 + v4);
    R tau = rabs(b0 - b2);
    if constexpr (sizeof(R) == 4) {
        // FP32: the reference weights a_k = d_k (1 + (τ/(β_k+ε))²) overflow when a
        // stencil is flat (β_k = 0: (1e-6/1e-30)² = 1e48 > FLT_MAX) and the
        // interpolant turns NaN. Scale every a_k by (m/t)², m = min_k(β_k+ε),
        // t = max(τ, m): identical weights in exact arithmetic, all terms ≤ 2 d_k.
        const R b0e = b0 + eps, b1e = b1 + eps, b2e = b2 + eps;
        const R m = rmin(b0e, rmin(b1e, b2e));
        const R t = rmax(tau, m);
        const R g = m / t, h = tau / t;
        const R r0 = (m / b0e) * h, r1 = (m / b1e) * h, r2 = (m / b2e) * h;
        const R g2 = g * g;
        const R a0 = R(1.0 / 16.0) * (g2 + r0 * r0);
        const R a1 = R(10.0 / 16.0) * (g2 + r1 * r1);
        const R a2 = R(5.0 / 16.0) * (g2 + r2 * r2);
        return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
    } else {
        R a0 = R(1.0 / 16.0) * (R(1) + sq(tau / (b0 + eps)));
        R a1 = R(10.0 / 16.0) * (R(1) + sq(tau / (b1 + eps)));
        R a2 = R(5.0 / 16.0) * (R(1) + sq(tau / (b2 + eps)));
        return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
    }
}

// ------------------------------------------------------------------ fast FP64 form
// Reciprocal and square roots to about one ulp without the correctly rounded
// division: the PTX estimate (good to about 2^-20) refined by one step of the
// series 1/(1 − h) = 1 + h + h² + …, which cubes its relative error (Newton's
// method with the quadratic term kept; for 1/y, h = 1 − y·r0 and
// r = r0·(1 + h + h²); for 1/√x, h = 1 − x·r0² and r = r0·(1 + h/2 + 3h²/8),
// the binomial series of (1 − h)^(−1/2)). The estimate's 2^-20 becomes
// 2^-60, below the final rounding, so results are within about one ulp of the
// correctly rounded ones. Zero, infinite and NaN inputs give non-finite
// results, which the admissibility tests treat as they treat infinities;
// subnormal inputs are flushed to zero. The fast FP64 form (EMG_PRECISION_
// F64_FAST) uses these in its sweep, the mixed form in its primitive recovery
// and its limiter's conserved states; the plain FP64 form never does.
__device__ __forceinline__ double rcp_f(double y) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(y));
    const double h = fma(-y, r, 1.0);
    return fma(r, fma(h, h, h), r);
}
__device__ __forceinline__ double rsqrt_f(double x) {
    double r;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
    const double h = fma(-(x * r), r, 1.0);
    return fma(r * h, fma(0.375, h, 0.5), r);
}

// Fast FP64 form of the NASG/Euler maps. Algebraically equal to the
// reference's formulas (eos.rs:37-60, system.rs:196-222), rearranged to
// share one reciprocal of ρ: ρ·(1/ρ − b) = 1 − bρ removes the division of
// ρe, and 1/(1/ρ − b) = ρ/(1 − bρ). `igm1` is 1/(γ − 1).
__device__ __forceinline__ void to_prim_f(const Eos<double>& e, const double* u, double* w) {
    const double rho = u[0];
    const double irho = rcp_f(rho);
    const double vx = u[1] * irho, vy = u[2] * irho, vz = u[3] * irho;
    const double ein = u[4] * irho - 0.5 * (vx * vx + vy * vy + vz * vz);
    const double rv = e.b == 0.0 ? rho : rho * rcp_f(1.0 - e.b * rho);  // 1/(v − b)
    w[0] = rho;
    w[1] = vx;
    w[2] = vy;
    w[3] = vz;
    w[4] = (e.gamma - 1.0) * (ein - e.q) * rv - e.gamma * e.p_inf;
}
__device__ __forceinline__ double rho_e_f(const Eos<double>& e, double igm1, double rho, double p) {
    return (p + e.gamma * e.p_inf) * (1.0 - e.b * rho) * igm1 + rho * e.q;
}
__device__ __forceinline__ void to_cons_f(const Eos<double>& e, double igm1, const double* w, double* u) {
    const double rho = w[0];
    const double ke = 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
    u[0] = rho;
    u[1] = rho * w[1];
    u[2] = rho * w[2];
    u[3] = rho * w[3];
    u[4] = rho_e_f(e, igm1, rho, w[4]) + ke;
}
// c² = γ(p + p∞)·v²/(v − b), v = 1/ρ, as γ(p + p∞)/(ρ(1 − bρ))
__device__ __forceinline__ double sound_speed_sq_f(const Eos<double>& e, double rho, double p) {
    return e.gamma * (p + e.p_inf) * rcp_f(rho * (1.0 - e.b * rho));
}
__device__ __forceinline__ double sqrt_f(double x) {
    // x ≥ 0; zero and +∞ pass through
    return x > 0.0 && x <= 1.79769313486231570e308 ? x * rsqrt_f(x) : x;
}
__device__ __forceinline__ double sound_speed_f(const Eos<double>& e, double rho, double p) {
    return sqrt_f(fmax(sound_speed_sq_f(e, rho, p), 0.0));
}
// system.rs:404-407 with eos.rs:75-79: 1/ρ > b ⟺ bρ < 1 for finite ρ > 0
__device__ __forceinline__ bool admissible_f(const Eos<double>& e, double rho, double p) {
    return isfinite(rho) && isfinite(p) && rho > 0.0 && e.b * rho < 1.0 && p + e.p_inf > 0.0;
}

// HLLC of the fast form (system.rs:260-312): the same wave-speed bounds,
// contact speed and star states with shared reciprocals.
__device__ __forceinline__ double hllc_f(const Eos<double>& e, double igm1, const double* wl, const double* wr, int un,
                                         double* f) {
    const double cl = sound_speed_f(e, wl[0], wl[4]), cr = sound_speed_f(e, wr[0], wr[4]);
    const double ul = wl[un], ur = wr[un];
    const double sl = fmin(ul - cl, ur - cr);
    const double sr = fmax(ul + cl, ur + cr);
    double ql[5], qr[5];
    to_cons_f(e, igm1, wl, ql);
    to_cons_f(e, igm1, wr, qr);
    if (sl >= 0.0) {
        flux_wq(wl, ql, un, f);
        return ul;
    }
    if (sr <= 0.0) {
        flux_wq(wr, qr, un, f);
        return ur;
    }
    const double rl = wl[0], rr = wr[0], pl = wl[4], pr = wr[4];
    const double ss = (pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur)) * rcp_f(rl * (sl - ul) - rr * (sr - ur));
    const bool left = ss >= 0.0;
    const double* w = left ? wl : wr;
    const double* q = left ? ql : qr;
    const double s = left ? sl : sr;
    double fx[5];
    flux_wq(w, q, un, fx);
    const double rho = w[0], u = w[un];
    const double smu = s - u;
    const double fac = rho * smu * rcp_f(s - ss);
    // E/ρ + (S* − u)(S* + p/(ρ(S − u))), with 1/ρ and 1/(S − u) from one reciprocal
    const double ir = rcp_f(rho * smu);
    const double irho = ir * smu;
    double qs[5];
    qs[0] = fac;
    qs[1] = fac * w[1];
    qs[2] = fac * w[2];
    qs[3] = fac * w[3];
    qs[un] = fac * ss;
    qs[4] = fac * (q[4] * irho + (ss - u) * (ss + w[4] * ir));
#pragma unroll
    for (int k = 0; k < 5; k++) f[k] = fx[k] + s * (qs[k] - q[k]);
    return ss;
}

// WENO5-Z interpolation of the fast form (scheme.rs:67-86): the three
// reciprocals 1/(β_k + ε) from one reciprocal of their product (each β_k + ε
// lies in [1e-40, 1e100] for any state whose values stay below 1e50, so the
// product neither under- nor overflows), and the normalisation by one more.
__device__ __forceinline__ double weno5z_interp_f(double v0, double v1, double v2, double v3, double v4) {
    const double eps = 1e-40;
    const double q0 = (3.0 * v0 - 10.0 * v1 + 15.0 * v2) * 0.125;
    const double q1 = (-v1 + 6.0 * v2 + 3.0 * v3) * 0.125;
    const double q2 = (3.0 * v2 + 6.0 * v3 - v4) * 0.125;
    const double b0 = (13.0 / 12.0) * sq(v0 - 2.0 * v1 + v2) + 0.25 * sq(v0 - 4.0 * v1 + 3.0 * v2);
    const double b1 = (13.0 / 12.0) * sq(v1 - 2.0 * v2 + v3) + 0.25 * sq(v1 - v3);
    const double b2 = (13.0 / 12.0) * sq(v2 - 2.0 * v3 + v4) + 0.25 * sq(3.0 * v2 - 4.0 * v3 + v4);
    const double tau = fabs(b0 - b2);
    const double x0 = b0 + eps, x1 = b1 + eps, x2 = b2 + eps;
    const double x01 = x0 * x1;
    const double t = tau * rcp_f(x01 * x2);
    const double r0 = t * (x1 * x2), r1 = t * (x0 * x2), r2 = t * x01;
    const double a0 = (1.0 / 16.0) * (1.0 + r0 * r0);
    const double a1 = (10.0 / 16.0) * (1.0 + r1 * r1);
    const double a2 = (5.0 / 16.0) * (1.0 + r2 * r2);
    return (a0 * q0 + a1 * q1 + a2 * q2) * rcp_f(a0 + a1 + a2);
}

// Coefficients of the 6th-order schemes (scheme.rs:88-92).
__device__ __forceinline__ double s6(int s) {
    return s == 0 ? (75.0 / 64.0 - 25.0 / 384.0 + 3.0 / 640.0) : (s == 1 ? (-25.0 / 384.0 + 3.0 / 640.0) : 3.0 / 640.0);
}

}  // namespace emg
