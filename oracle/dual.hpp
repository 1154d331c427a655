// CPU ORACLE — test infrastructure only (see oracle.hpp).
//
// Forward-mode dual number a + b·ε (ε² = 0) with one tangent, so that the
// templated restatement of the reference solver (oracle.hpp) runs as a CPU
// f64 forward-mode derivative of the reference scheme: every arithmetic
// operation carries the directional derivative along one input direction.
// The value part rounds exactly as the plain f64 instantiation (same
// operations in the same order), so branch decisions (HLLC wave cases,
// admissibility fallbacks, limiter bisection, CFL) are those of the f64 run.
//
// Conventions at the non-smooth points, shared with the device adjoint:
//  |x|      derivative sign(x), +1 at x = 0
//  min/max  the first argument's derivative on ties (a ≤ b for min, a ≥ b for max)
//  the limiter's bisection parameter is built from constants and comparisons
//  only, so its tangent is zero: θ is held fixed, as in the adjoint.
//  WENO-Z smoothness indicators: an undivided difference of a sub-stencil
//  whose magnitude is at the rounding level of its inputs (|A| ≤ 2^-46·Σ|v|)
//  is zero in exact arithmetic, and its tangent is taken as zero. Without this
//  rule the floating-point residue of a flat stencil (e.g. 3x − 4x + x ≠ 0)
//  enters a weight derivative scaled by 1/(β + 1e-40)² and the derivative of a
//  flat stencil comes out O(10) wrong (scheme.rs:55, :76-86). For the same
//  reason the weight derivatives multiply q_k − y formed from differences of
//  the candidate values rather than from the rounded interpolant.
// The reference crate has a second-order dual of its own inside the
// Helmholtz EOS (fluid/crates/compressible/src/helmholtz.rs:5-6); it is not
// on this path and is not reused.
#pragma once
#include <cmath>

namespace oracle {

struct Dual {
    double v = 0.0, d = 0.0;
    Dual() = default;
    Dual(double x) : v(x), d(0.0) {}  // NOLINT: implicit, as T(1.0) etc. in the templates
    Dual(double x, double dx) : v(x), d(dx) {}
};

inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}
inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }

inline Dual sqrt(Dual a) {
    const double s = std::sqrt(a.v);
    return {s, a.d / (2.0 * s)};
}
inline Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
inline Dual log(Dual a) { return {std::log(a.v), a.d / a.v}; }

// Rust f64::max/min semantics on the value (a NaN operand yields the other).
inline Dual fmax_(Dual a, Dual b) {
    if (std::isnan(a.v)) return b;
    if (std::isnan(b.v)) return a;
    return a.v >= b.v ? a : b;
}
inline Dual fmin_(Dual a, Dual b) {
    if (std::isnan(a.v)) return b;
    if (std::isnan(b.v)) return a;
    return a.v <= b.v ? a : b;
}
inline bool finite_(Dual a) { return std::isfinite(a.v); }
inline double value_(Dual a) { return a.v; }

// Undivided difference with the rounding-level rule above; `scale` is the sum
// of the magnitudes of the sub-stencil's three values.
inline Dual weno_diff(Dual a, double scale) {
    if (std::fabs(a.v) <= 0x1p-46 * scale) a.d = 0.0;
    return a;
}

// WENO5-Z interpolation to x_{2+1/2} (scheme.rs:67-86) in dual numbers: the
// value part is the f64 formula in the reference's operation order.
inline Dual weno5z_interp(Dual v0, Dual v1, Dual v2, Dual v3, Dual v4) {
    auto sq = [](Dual x) { return x * x; };
    const double s0 = std::fabs(v0.v) + std::fabs(v1.v) + std::fabs(v2.v);
    const double s1 = std::fabs(v1.v) + std::fabs(v2.v) + std::fabs(v3.v);
    const double s2 = std::fabs(v2.v) + std::fabs(v3.v) + std::fabs(v4.v);
    Dual q0 = (Dual(3.0) * v0 - Dual(10.0) * v1 + Dual(15.0) * v2) / Dual(8.0);
    Dual q1 = (-v1 + Dual(6.0) * v2 + Dual(3.0) * v3) / Dual(8.0);
    Dual q2 = (Dual(3.0) * v2 + Dual(6.0) * v3 - v4) / Dual(8.0);
    Dual b0 = Dual(13.0 / 12.0) * sq(weno_diff(v0 - Dual(2.0) * v1 + v2, s0)) +
              Dual(0.25) * sq(weno_diff(v0 - Dual(4.0) * v1 + Dual(3.0) * v2, s0));
    Dual b1 = Dual(13.0 / 12.0) * sq(weno_diff(v1 - Dual(2.0) * v2 + v3, s1)) + Dual(0.25) * sq(weno_diff(v1 - v3, s1));
    Dual b2 = Dual(13.0 / 12.0) * sq(weno_diff(v2 - Dual(2.0) * v3 + v4, s2)) +
              Dual(0.25) * sq(weno_diff(Dual(3.0) * v2 - Dual(4.0) * v3 + v4, s2));
    Dual tau = fabs(b0 - b2);
    const double eps = 1e-40;  // scheme.rs:55
    Dual a0 = Dual(1.0 / 16.0) * (Dual(1.0) + sq(tau / (b0 + Dual(eps))));
    Dual a1 = Dual(10.0 / 16.0) * (Dual(1.0) + sq(tau / (b1 + Dual(eps))));
    Dual a2 = Dual(5.0 / 16.0) * (Dual(1.0) + sq(tau / (b2 + Dual(eps))));
    // value: the reference formula; tangent: Σ_k a_k' (q_k − y) + a_k q_k', over
    // S, with q_k − y formed as Σ_m a_m (q_k − q_m)/S (no cancellation against
    // the rounded y, whose residue the near-flat weight derivatives amplify)
    const double S = a0.v + a1.v + a2.v;
    const double y = (a0.v * q0.v + a1.v * q1.v + a2.v * q2.v) / S;
    const double d0 = (a1.v * (q0.v - q1.v) + a2.v * (q0.v - q2.v)) / S;
    const double d1 = (a0.v * (q1.v - q0.v) + a2.v * (q1.v - q2.v)) / S;
    const double d2 = (a0.v * (q2.v - q0.v) + a1.v * (q2.v - q1.v)) / S;
    const double dy = (a0.d * d0 + a1.d * d1 + a2.d * d2 + a0.v * q0.d + a1.v * q1.d + a2.v * q2.d) / S;
    return Dual(y, dy);
}

}  // namespace oracle
