// Hand-written reverse mode (vector–Jacobian products) of the FP64 WCNS /
// HLLC / positivity-limited scheme of the compressible Euler step.
//
// Each *_vjp function recomputes the forward quantities it needs with the
// same code and operation order as the forward kernels (physics.cuh,
// sweep.cuh), so branch decisions — HLLC wave case, admissibility fallback to
// first order, Davis min/max — are exactly those of the forward run, and then
// propagates cotangents backwards. Cotangents are accumulated with +=.
//
// Non-smooth points follow one convention, shared with the dual-number CPU
// check: d|x| = sign(x) with +1 at 0; min/max take the first argument's
// derivative on ties; the positivity-limiter blend weight θ is held at its
// forward value (a constant), as is the admissibility fallback flag.
// `gb` accumulates the cotangent of the ratio of specific heats γ.
//
// The forward formulas are those of the reference CPU solver
// (fluid/crates/compressible/src/eos.rs:37-60, system.rs:197-312,
// scheme.rs:67-86 and 286-333 and 395-464); the reference has no adjoint.
#pragma once
#include "physics.cuh"

namespace emg {
namespace adj {

// ---- EOS and conserved/primitive maps ------------------------------------

// w = to_prim(U): given wb, add Ub and gb (system.rs:197-203, eos.rs:37-41).
__device__ __forceinline__ void to_prim_vjp(const Eos<double>& e, const double* U, const double* wb, double* Ub,
                                            double& gb) {
    const double rho = U[0];
    const double vx = U[1] / rho, vy = U[2] / rho, vz = U[3] / rho;
    const double ein = U[4] / rho - 0.5 * (vx * vx + vy * vy + vz * vz);
    const double v = 1.0 / rho;
    const double vmb = v - e.b;
    const double pb = wb[4];
    const double einb = pb * (e.gamma - 1.0) / vmb;
    const double vb = -pb * (e.gamma - 1.0) * (ein - e.q) / (vmb * vmb);
    gb += pb * ((ein - e.q) / vmb - e.p_inf);
    double rhob = wb[0] - vb * v * v;
    Ub[4] += einb / rho;
    rhob -= einb * (U[4] / rho) / rho;
    const double vel[3] = {vx, vy, vz};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const double velb = wb[1 + k] - einb * vel[k];
        Ub[1 + k] += velb / rho;
        rhob -= velb * vel[k] / rho;
    }
    Ub[0] += rhob;
}

// q = to_cons(w): given qb, add wb and gb (system.rs:210-217, eos.rs:44-54).
__device__ __forceinline__ void to_cons_vjp(const Eos<double>& e, const double* w, const double* qb, double* wb,
                                            double& gb) {
    const double rho = w[0], p = w[4];
    const double v = 1.0 / rho, vmb = v - e.b, gm1 = e.gamma - 1.0;
    const double ppi = p + e.gamma * e.p_inf;
    const double en = ppi * vmb / gm1 + e.q;  // specific internal energy
    const double ke2 = w[1] * w[1] + w[2] * w[2] + w[3] * w[3];
    double rhob = qb[0] + qb[4] * (0.5 * ke2);
#pragma unroll
    for (int k = 1; k < 4; k++) {
        rhob += qb[k] * w[k];
        wb[k] += qb[k] * rho + qb[4] * rho * w[k];
    }
    // ρe = ρ·en(ρ, p, γ)
    rhob += qb[4] * (en - ppi * v / gm1);
    wb[4] += qb[4] * rho * vmb / gm1;
    gb += qb[4] * rho * (e.p_inf * vmb / gm1 - ppi * vmb / (gm1 * gm1));
    wb[0] += rhob;
}

// c = sqrt(max(c², 0)), c² = γ(p + p∞)v²/(v − b), v = 1/ρ (system.rs:219-222,
// eos.rs:56-60): given cb, add ρb, pb and gb.
__device__ __forceinline__ void sound_speed_vjp(const Eos<double>& e, double rho, double p, double cb, double& rhob,
                                                double& pb, double& gb) {
    const double c2 = e.sound_speed_sq(rho, p);
    if (!(c2 > 0.0)) return;
    const double c = sqrt(c2);
    const double c2b = cb / (2.0 * c);
    const double v = 1.0 / rho, vmb = v - e.b, pp = p + e.p_inf;
    const double dv = e.gamma * pp * v * (v - 2.0 * e.b) / (vmb * vmb);
    rhob -= c2b * dv * v * v;
    pb += c2b * e.gamma * v * v / vmb;
    gb += c2b * pp * v * v / vmb;
}

// f = flux_wq(w, q) along normal index un (system.rs:268-278): given fb, add
// qb and the (u_n, p) parts of wb.
template <int UN>
__device__ __forceinline__ void flux_wq_vjp(const double* w, const double* q, const double* fb, double* wb,
                                            double* qb) {
    const double u = w[UN], p = w[4];
    double ub = 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        qb[k] += fb[k] * u;
        ub += fb[k] * q[k];
    }
    qb[4] += fb[4] * u;
    ub += fb[4] * (q[4] + p);
    wb[UN] += ub;
    wb[4] += fb[UN] + fb[4] * u;
}

// ---- HLLC with Davis wave-speed bounds (system.rs:260-312) ----------------

template <int UN>
__device__ __forceinline__ void hllc_vjp(const Eos<double>& e, const double* wl, const double* wr, const double* fb,
                                         double* wlb, double* wrb, double& gb) {
    const double cl = sound_speed(e, wl[0], wl[4]), cr = sound_speed(e, wr[0], wr[4]);
    const double ul = wl[UN], ur = wr[UN];
    const double al = ul - cl, ar = ur - cr, bl = ul + cl, br = ur + cr;
    const double sl = rmin(al, ar), sr = rmax(bl, br);
    double ql[5], qr[5];
    to_cons(e, wl, ql);
    to_cons(e, wr, qr);
    // the side whose state enters the flux is copied element-wise (selecting
    // a whole array by pointer would force the arrays into local memory)
    double w[5], q[5], wb[5] = {0, 0, 0, 0, 0};
    if (sl >= 0.0 || sr <= 0.0) {
        // supersonic: f = flux(w, q) of one side; sl, sr only chose the branch
        const bool L = sl >= 0.0;
#pragma unroll
        for (int k = 0; k < 5; k++) {
            w[k] = L ? wl[k] : wr[k];
            q[k] = L ? ql[k] : qr[k];
        }
        double qb[5] = {0, 0, 0, 0, 0};
        flux_wq_vjp<UN>(w, q, fb, wb, qb);
        to_cons_vjp(e, w, qb, wb, gb);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            wlb[k] += L ? wb[k] : 0.0;
            wrb[k] += L ? 0.0 : wb[k];
        }
        return;
    }
    const double rl = wl[0], rr = wr[0], pl = wl[4], pr = wr[4];
    const double num = pr - pl + rl * ul * (sl - ul) - rr * ur * (sr - ur);
    const double den = rl * (sl - ul) - rr * (sr - ur);
    const double ss = num / den;
    const bool L = ss >= 0.0;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        w[k] = L ? wl[k] : wr[k];
        q[k] = L ? ql[k] : qr[k];
    }
    const double s = L ? sl : sr;
    const double rho = w[0], u = w[UN], p = w[4];
    const double sm = s - u;
    const double K = rho * sm;
    const double M = s - ss;
    const double fac = K / M;
    const double H = ss + p / K;
    const double G = q[4] / rho + (ss - u) * H;
    double qs[5];
    qs[0] = fac;
    qs[1] = fac * w[1];
    qs[2] = fac * w[2];
    qs[3] = fac * w[3];
    qs[UN] = fac * ss;
    qs[4] = fac * G;
    // f_k = fx_k + s (qs_k − q_k)
    double sb = 0.0, qb[5], qsb[5];
#pragma unroll
    for (int k = 0; k < 5; k++) {
        sb += fb[k] * (qs[k] - q[k]);
        qsb[k] = s * fb[k];
        qb[k] = -s * fb[k];
    }
    double rhob = 0.0, ub = 0.0, pb = 0.0, ssb = 0.0;
    double facb = qsb[0] + qsb[4] * G;
#pragma unroll
    for (int k = 1; k < 4; k++) {
        if (k == UN) continue;
        facb += qsb[k] * w[k];
        wb[k] += qsb[k] * fac;
    }
    facb += qsb[UN] * ss;
    ssb += qsb[UN] * fac;
    const double Gb = qsb[4] * fac;
    qb[4] += Gb / rho;
    rhob -= Gb * (q[4] / rho) / rho;
    ssb += Gb * H;
    ub -= Gb * H;
    const double Hb = Gb * (ss - u);
    ssb += Hb;
    pb += Hb / K;
    double Kb = -Hb * (p / K) / K;
    // fac = K / M
    Kb += facb / M;
    const double Mb = -facb * fac / M;
    sb += Mb;
    ssb -= Mb;
    // K = ρ (s − u)
    rhob += Kb * sm;
    sb += Kb * rho;
    ub -= Kb * rho;
    // fx = flux(w, q)
    flux_wq_vjp<UN>(w, q, fb, wb, qb);
    wb[0] += rhob;
    wb[UN] += ub;
    wb[4] += pb;
    to_cons_vjp(e, w, qb, wb, gb);
#pragma unroll
    for (int k = 0; k < 5; k++) {
        wlb[k] += L ? wb[k] : 0.0;
        wrb[k] += L ? 0.0 : wb[k];
    }
    // ss = num / den
    const double numb = ssb / den, denb = -ssb * ss / den;
    double rlb = numb * ul * (sl - ul) + denb * (sl - ul);
    double ulb = numb * rl * (sl - ul - ul) - denb * rl;
    double slb = numb * rl * ul + denb * rl;
    double rrb = -numb * ur * (sr - ur) - denb * (sr - ur);
    double urb = -numb * rr * (sr - ur - ur) + denb * rr;
    double srb = -numb * rr * ur - denb * rr;
    double plb = -numb, prb = numb;
    if (L)
        slb += sb;
    else
        srb += sb;
    // Davis bounds: first argument on ties
    double clb = 0.0, crb = 0.0;
    if (al <= ar) {
        ulb += slb;
        clb -= slb;
    } else {
        urb += slb;
        crb -= slb;
    }
    if (bl >= br) {
        ulb += srb;
        clb += srb;
    } else {
        urb += srb;
        crb += srb;
    }
    sound_speed_vjp(e, wl[0], wl[4], clb, rlb, plb, gb);
    sound_speed_vjp(e, wr[0], wr[4], crb, rrb, prb, gb);
    wlb[0] += rlb;
    wlb[UN] += ulb;
    wlb[4] += plb;
    wrb[0] += rrb;
    wrb[UN] += urb;
    wrb[4] += prb;
}

// ---- WENO5-Z interpolation (scheme.rs:67-86) -------------------------------

// Gradient g[0..4] of the interpolant with respect to v0..v4. An undivided
// difference (A_k, B_k of the smoothness indicator β_k) whose magnitude is at
// the rounding level of its three inputs (|A| ≤ 2^-46·Σ|v|) is zero in exact
// arithmetic and contributes no derivative: otherwise the floating-point
// residue of a flat stencil (3x − 4x + x ≠ 0) is amplified by 1/(β + 1e-40)²
// and a flat stencil's gradient comes out O(10) wrong.
__device__ __forceinline__ double weno_dd(double a, double scale) { return fabs(a) <= 0x1p-46 * scale ? 0.0 : a; }

__device__ __forceinline__ void weno5z_grad(double v0, double v1, double v2, double v3, double v4, double* g) {
    const double eps = 1e-40;
    const double q[3] = {(3.0 * v0 - 10.0 * v1 + 15.0 * v2) * 0.125, (-v1 + 6.0 * v2 + 3.0 * v3) * 0.125,
                         (3.0 * v2 + 6.0 * v3 - v4) * 0.125};
    const double A0 = v0 - 2.0 * v1 + v2, B0 = v0 - 4.0 * v1 + 3.0 * v2;
    const double A1 = v1 - 2.0 * v2 + v3, B1 = v1 - v3;
    const double A2 = v2 - 2.0 * v3 + v4, B2 = 3.0 * v2 - 4.0 * v3 + v4;
    const double b[3] = {13.0 / 12.0 * (A0 * A0) + 0.25 * (B0 * B0), 13.0 / 12.0 * (A1 * A1) + 0.25 * (B1 * B1),
                         13.0 / 12.0 * (A2 * A2) + 0.25 * (B2 * B2)};
    const double dw[3] = {1.0 / 16.0, 10.0 / 16.0, 5.0 / 16.0};
    const double tau = fabs(b[0] - b[2]);
    // derivative arithmetic only: reciprocals instead of the reference's
    // divisions (the interpolated value itself comes from weno5z_interp)
    double ib[3], r[3], a[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        ib[k] = 1.0 / (b[k] + eps);
        r[k] = tau * ib[k];
        a[k] = dw[k] * (1.0 + r[k] * r[k]);
    }
    const double iS = 1.0 / (a[0] + a[1] + a[2]);
    // q_k − y = Σ_m a_m (q_k − q_m) / S, formed from differences of the
    // candidate values: subtracting the rounded y would leave a rounding
    // residue that the large weight derivatives of near-flat stencils
    // (∝ 1/(β + 1e-40)) amplify into spurious gradient terms
    const double dq[3] = {(a[1] * (q[0] - q[1]) + a[2] * (q[0] - q[2])) * iS,
                          (a[0] * (q[1] - q[0]) + a[2] * (q[1] - q[2])) * iS,
                          (a[0] * (q[2] - q[0]) + a[1] * (q[2] - q[1])) * iS};
    double qb[3], bb[3], taub = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        qb[k] = a[k] * iS;
        const double rb = (dq[k] * iS) * dw[k] * 2.0 * r[k];
        taub += rb * ib[k];
        bb[k] = -rb * r[k] * ib[k];
    }
    const double sgn = (b[0] - b[2]) < 0.0 ? -1.0 : 1.0;
    bb[0] += sgn * taub;
    bb[2] -= sgn * taub;
    const double s0 = fabs(v0) + fabs(v1) + fabs(v2), s1 = fabs(v1) + fabs(v2) + fabs(v3),
                 s2 = fabs(v2) + fabs(v3) + fabs(v4);
    const double A0b = 13.0 / 6.0 * weno_dd(A0, s0) * bb[0], B0b = 0.5 * weno_dd(B0, s0) * bb[0];
    const double A1b = 13.0 / 6.0 * weno_dd(A1, s1) * bb[1], B1b = 0.5 * weno_dd(B1, s1) * bb[1];
    const double A2b = 13.0 / 6.0 * weno_dd(A2, s2) * bb[2], B2b = 0.5 * weno_dd(B2, s2) * bb[2];
    g[0] = A0b + B0b + 0.375 * qb[0];
    g[1] = -2.0 * A0b - 4.0 * B0b + A1b + B1b - 1.25 * qb[0] - 0.125 * qb[1];
    g[2] = A0b + 3.0 * B0b - 2.0 * A1b + A2b + 3.0 * B2b + 1.875 * qb[0] + 0.75 * qb[1] + 0.375 * qb[2];
    g[3] = A1b - B1b - 2.0 * A2b - 4.0 * B2b + 0.375 * qb[1] + 0.75 * qb[2];
    g[4] = A2b + B2b - 0.125 * qb[2];
}

// ---- characteristic WCNS midpoint flux (scheme.rs:286-333) ---------------

// Stencil accessors: W(s, k) reads primitive k of stencil row s (0..5);
// B.add(s, k, v) accumulates a cotangent. Plain arrays on the host; the
// device kernel reads shared memory and writes a per-thread slot, which keeps
// the 2×30 stencil values out of registers.
struct RowsIn {
    const double (*w)[5];
    __device__ __forceinline__ double operator()(int s, int k) const { return w[s][k]; }
};
struct RowsOut {
    double (*b)[5];
    __device__ __forceinline__ void add(int s, int k, double v) const { b[s][k] += v; }
};

// Midpoint between stencil rows 2 and 3 of the six primitive rows W(s, k);
// given the cotangent fb of its HLLC flux, accumulate the stencil cotangents
// and gb. Sparse form of the dense eigenvector products, as in the forward
// sweep; the characteristic fields are reversed one at a time.
template <int D, class WIn, class WOut>
__device__ __forceinline__ void midpoint_vjp_acc(const Eos<double>& e, const WIn& W, const double* fb, const WOut& B,
                                                 double& gb) {
    constexpr int un = 1 + D;
    constexpr int t1 = 1 + (D + 1) % 3, t2 = 1 + (D + 2) % 3;
    const double avg0 = 0.5 * (W(2, 0) + W(3, 0));
    const double avg4 = 0.5 * (W(2, 4) + W(3, 4));
    const double rho = avg0;
    const double c = sound_speed(e, avg0, avg4);
    const double l4un = rho / (2.0 * c);
    const double l0un = -l4un;
    const double l04 = 1.0 / (2.0 * c * c);
    const double l14 = -1.0 / (c * c);
    const double run4 = c / rho;
    const double run0 = -run4;
    const double r40 = c * c;
    // characteristic values of field a at stencil row s (exact forward order)
    auto chv = [&](int a, int s) -> double {
        switch (a) {
            case 0: return l0un * W(s, un) + l04 * W(s, 4);
            case 1: return W(s, 0) + l14 * W(s, 4);
            case 2: return W(s, t1);
            case 3: return W(s, t2);
            default: return l4un * W(s, un) + l04 * W(s, 4);
        }
    };
    double cl[5], cr[5];
#pragma unroll
    for (int a = 0; a < 5; a++) {
        const double v0 = chv(a, 0), v1 = chv(a, 1), v2 = chv(a, 2), v3 = chv(a, 3), v4 = chv(a, 4), v5 = chv(a, 5);
        cl[a] = weno5z_interp(v0, v1, v2, v3, v4);
        cr[a] = weno5z_interp(v5, v4, v3, v2, v1);
    }
    double wl[5], wr[5];
    wl[0] = (cl[0] + cl[1]) + cl[4];
    wr[0] = (cr[0] + cr[1]) + cr[4];
    wl[un] = run0 * cl[0] + run4 * cl[4];
    wr[un] = run0 * cr[0] + run4 * cr[4];
    wl[t1] = cl[2];
    wr[t1] = cr[2];
    wl[t2] = cl[3];
    wr[t2] = cr[3];
    wl[4] = r40 * cl[0] + r40 * cl[4];
    wr[4] = r40 * cr[0] + r40 * cr[4];
    double wlb[5] = {0, 0, 0, 0, 0}, wrb[5] = {0, 0, 0, 0, 0};
    if (!admissible(e, wl[0], wl[4]) || !admissible(e, wr[0], wr[4])) {
        // first-order fallback: the flux of the two adjacent cells
        double w2[5], w3[5];
#pragma unroll
        for (int k = 0; k < 5; k++) {
            w2[k] = W(2, k);
            w3[k] = W(3, k);
        }
        hllc_vjp<un>(e, w2, w3, fb, wlb, wrb, gb);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            B.add(2, k, wlb[k]);
            B.add(3, k, wrb[k]);
        }
        return;
    }
    hllc_vjp<un>(e, wl, wr, fb, wlb, wrb, gb);
    // back-projection w = R·c
    double clb[5], crb[5];
    clb[0] = wlb[0] + run0 * wlb[un] + r40 * wlb[4];
    crb[0] = wrb[0] + run0 * wrb[un] + r40 * wrb[4];
    clb[1] = wlb[0];
    crb[1] = wrb[0];
    clb[2] = wlb[t1];
    crb[2] = wrb[t1];
    clb[3] = wlb[t2];
    crb[3] = wrb[t2];
    clb[4] = wlb[0] + run4 * wlb[un] + r40 * wlb[4];
    crb[4] = wrb[0] + run4 * wrb[un] + r40 * wrb[4];
    const double run0b = wlb[un] * cl[0] + wrb[un] * cr[0];
    const double run4b = wlb[un] * cl[4] + wrb[un] * cr[4];
    const double r40b = wlb[4] * (cl[0] + cl[4]) + wrb[4] * (cr[0] + cr[4]);
    // WENO-Z interpolations and the projection c = L·w, one field at a time
    double l0unb = 0.0, l4unb = 0.0, l04b = 0.0, l14b = 0.0;
    // not unrolled: keeps one field's stencil, gradients and cotangents live at a time
#pragma unroll 1
    for (int a = 0; a < 5; a++) {
        if (clb[a] == 0.0 && crb[a] == 0.0) continue;
        double v[6], chb[6], g[5];
#pragma unroll
        for (int s2 = 0; s2 < 6; s2++) v[s2] = chv(a, s2);
        weno5z_grad(v[0], v[1], v[2], v[3], v[4], g);
#pragma unroll
        for (int s2 = 0; s2 < 5; s2++) chb[s2] = clb[a] * g[s2];
        chb[5] = 0.0;
        weno5z_grad(v[5], v[4], v[3], v[2], v[1], g);
#pragma unroll
        for (int s2 = 0; s2 < 5; s2++) chb[5 - s2] += crb[a] * g[s2];
#pragma unroll
        for (int s2 = 0; s2 < 6; s2++) {
            const double cb = chb[s2];
            switch (a) {
                case 0:
                    B.add(s2, un, l0un * cb);
                    B.add(s2, 4, l04 * cb);
                    l0unb += W(s2, un) * cb;
                    l04b += W(s2, 4) * cb;
                    break;
                case 1:
                    B.add(s2, 0, cb);
                    B.add(s2, 4, l14 * cb);
                    l14b += W(s2, 4) * cb;
                    break;
                case 2: B.add(s2, t1, cb); break;
                case 3: B.add(s2, t2, cb); break;
                default:
                    B.add(s2, un, l4un * cb);
                    B.add(s2, 4, l04 * cb);
                    l4unb += W(s2, un) * cb;
                    l04b += W(s2, 4) * cb;
            }
        }
    }
    // eigenvector entries as functions of (ρ, c) at the midpoint average
    const double l4unt = l4unb - l0unb;
    const double run4t = run4b - run0b;
    const double cb = l4unt * (-l4un / c) + l04b * (-2.0 * l04 / c) + l14b * (-2.0 * l14 / c) + run4t / rho +
                      r40b * (2.0 * c);
    double avgb0 = l4unt / (2.0 * c) - run4t * run4 / rho;
    double avgb4 = 0.0;
    sound_speed_vjp(e, avg0, avg4, cb, avgb0, avgb4, gb);
    B.add(2, 0, 0.5 * avgb0);
    B.add(3, 0, 0.5 * avgb0);
    B.add(2, 4, 0.5 * avgb4);
    B.add(3, 4, 0.5 * avgb4);
}

// Array form of midpoint_vjp: w6[s][k] in, wb6[s][k] accumulated.
template <int D>
__device__ __forceinline__ void midpoint_vjp(const Eos<double>& e, const double (*w6)[5], const double* fb,
                                             double (*wb6)[5], double& gb) {
    midpoint_vjp_acc<D>(e, RowsIn{w6}, fb, RowsOut{wb6}, gb);
}

// ---- positivity limiter with the blend weight θ held fixed (scheme.rs:395-464)

// Face between cells with primitives wi, wj whose limited flux is
// θ·F̃ + (1 − θ)·F_LF: given the cotangent Fb of the face flux, add the
// Lax–Friedrichs part's cotangents to wib, wjb and gb (the caller scales the
// high-order part by θ).
template <int D>
__device__ __forceinline__ void lf_vjp(const Eos<double>& e, const double* wi, const double* wj, double theta,
                                       const double* Fb, double* wib, double* wjb, double& gb) {
    constexpr int un = 1 + D;
    double ul[5], ur[5];
    to_cons(e, wi, ul);
    to_cons(e, wj, ur);
    const double ci = sound_speed(e, wi[0], wi[4]), cj = sound_speed(e, wj[0], wj[4]);
    const double ai = fabs(wi[un]) + ci, aj = fabs(wj[un]) + cj;
    const double alpha = rmax(ai, aj);
    double flfb[5], flpb[5], frpb[5], ulb[5], urb[5];
    double alphab = 0.0;
#pragma unroll
    for (int k = 0; k < 5; k++) {
        flfb[k] = (1.0 - theta) * Fb[k];
        flpb[k] = 0.5 * flfb[k];
        frpb[k] = 0.5 * flfb[k];
        alphab -= 0.5 * flfb[k] * (ur[k] - ul[k]);
        urb[k] = -0.5 * alpha * flfb[k];
        ulb[k] = 0.5 * alpha * flfb[k];
    }
    const bool I = ai >= aj;  // Davis-style max: first argument on ties
    const double wun = I ? wi[un] : wj[un], w0 = I ? wi[0] : wj[0], w4 = I ? wi[4] : wj[4];
    double rb = 0.0, pb = 0.0;
    sound_speed_vjp(e, w0, w4, alphab, rb, pb, gb);
    const double unb = (wun < 0.0 ? -1.0 : 1.0) * alphab;
    wib[0] += I ? rb : 0.0;
    wib[un] += I ? unb : 0.0;
    wib[4] += I ? pb : 0.0;
    wjb[0] += I ? 0.0 : rb;
    wjb[un] += I ? 0.0 : unb;
    wjb[4] += I ? 0.0 : pb;
    flux_wq_vjp<un>(wi, ul, flpb, wib, ulb);
    flux_wq_vjp<un>(wj, ur, frpb, wjb, urb);
    to_cons_vjp(e, wi, ulb, wib, gb);
    to_cons_vjp(e, wj, urb, wjb, gb);
}

}  // namespace adj
}  // namespace emg
