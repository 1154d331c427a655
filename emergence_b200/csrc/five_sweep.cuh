// Fused per-axis sweep of the WCNS / HLLC / positivity scheme for the
// five-equation system (uniform grids, FP64). Same streaming design as the
// Euler sweep (sweep.cuh): a CTA of 256 threads owns P adjacent pencils over
// one segment of the sweep axis and streams it in rounds of RM = 256/P rows
// through shared-memory rings:
//
//   A  rows of the 7 conserved fields → primitives (plus ρe for the central
//      flux and the 3 sensor values for the hybrid switch) in the W ring;
//   Θ  (hybrid) the blend weight of each face from the sensors;
//   B  one thread per (midpoint, pencil): characteristic WENO5-Z
//      interpolation of the 7 fields, admissibility fallback, HLLC flux and
//      contact speed (MF ring);
//   C  one thread per (face, pencil): 6th-order WCNS combination of the
//      midpoint fluxes and contact speeds, central KEEP-PE flux and face
//      velocity where θ < 1, positivity limiter (F ring, 7 fluxes + face
//      velocity);
//   D  one thread per (cell, pencil): −(F⁺ − F⁻)/dx and the non-conservative
//      term (α + K)(Ũ⁺ − Ũ⁻)/dx of the α equation into the residual; on the
//      last active axis the SSP-RK3 combination into the next stage state.
//
// Operation order follows the reference CPU solver (scheme.rs:132-464,
// solver.rs:431-442) so that the FP64 results are bit-identical with it.
#pragma once
#include "five_physics.cuh"
#include "sweep.cuh"

namespace emg {

struct FiveSweepParams {
    const double* __restrict__ uin;
    double* rhs;
    const double* base;
    const double* cur;
    double* dest;
    StepCtl* ctl;
    int64_t ncell;
    int64_t sd, sl, so;
    int nd, nl, no;
    int gd, gl, go;
    int d;
    int seg;
    int first, last;
    int stage;
    int rows_contig;
    double dx;
    double ndim;
    int positivity;
    double tol;
    FiveSysD sys;
    // ---- batched block-AMR leaves (the AMR instantiation)
    const int* leaf_slot;   // pool slot of launch leaf x / ngroups
    const int* leaf_level;  // level of each pool slot
    int64_t bcell;          // cells per pool block (ghost-extended)
    int ngroups;            // CTAs per leaf along the other axis
    int lw;                 // lanes of one block row (≤ P)
    double dx_level[16];    // cell size along d per level
    double* face;           // block-face flux record for refluxing
    int64_t nface;          // its length (doubles)
    int npen;               // pencils per block face (padded)
    int pen_lane_major;     // pencil index = lane*no + other (lane axis is the lower of the two others)
    // optional chains of same-level leaves along d, as in SweepParams (null:
    // one leaf per launch chain)
    const int* chain_off;
    const int* chain_slot;
};

template <int P, int MODE> struct FiveSmem {
    static constexpr int RM = SWEEP_THREADS / P;
    static constexpr int RS = RingSize<RM, MODE>::value;  // W (and TH) ring rows
    // flux rings of exactly what one round keeps alive, as in the Euler sweep:
    // midpoints [RM r − 4, RM r + RM), faces [RM r − 5, RM r + RM − 4)
    static constexpr int RSM = RM + 4;
    static constexpr int RSF = RM + 1;
    // per cell: 7 primitives, + ρe (central flux), + 3 sensor values (hybrid)
    static constexpr int NW = MODE == MODE_WENO ? NF : (MODE == MODE_CENTRAL ? NF + 1 : NF + 4);
    static constexpr int STRW = NW * P + 1;
    static constexpr int STR = (NF + 1) * P + 1;  // 7 fluxes + velocity
    static constexpr bool MID = MODE != MODE_CENTRAL;
    static constexpr size_t bytes() {
        return (size_t)RS * STRW * sizeof(double) + (MID ? (size_t)RSM * STR * sizeof(double) : 0) +
               (size_t)RSF * STR * sizeof(double) + (MODE == MODE_HYBRID ? (size_t)RS * P * sizeof(double) : 0);
    }
};

// FAST: the fast FP64 form (built with FMA contraction, WENO5-Z weights from
// the one-ulp reciprocals of physics.cuh's fast section)
template <int P, int D, int MODE, bool AMR = false, bool FAST = false> struct FiveSweep {
    using SM = FiveSmem<P, MODE>;
    static constexpr int T = SWEEP_THREADS;
    static constexpr int RM = SM::RM;
    static constexpr int RS = SM::RS;
    static constexpr int STRW = SM::STRW;
    static constexpr int STR = SM::STR;
    static constexpr bool MID = SM::MID;
    static constexpr int AHEAD = MODE == MODE_HYBRID ? 7 : 5;
    static constexpr int UN = F_IU + D;
    static constexpr int T1 = F_IU + (D + 1) % 3, T2 = F_IU + (D + 2) % 3;

    __device__ static __forceinline__ int slot(int x) { return x & (RS - 1); }
    template <int S> __device__ static __forceinline__ int at(int x, int k, int l) { return slot(x) * S + k * P + l; }
    // midpoint and face flux rings (x ≥ 0)
    __device__ static __forceinline__ int atM(int x, int k, int l) {
        return (int)((unsigned)x % (unsigned)SM::RSM) * STR + k * P + l;
    }
    __device__ static __forceinline__ int atF(int x, int k, int l) {
        return (int)((unsigned)x % (unsigned)SM::RSF) * STR + k * P + l;
    }

    // scheme.rs:286-333 with the five-equation eigenvectors (multiphase.rs:202-236)
    __device__ static __forceinline__ double midpoint(const Five& s, const double* __restrict__ W, int m, int l,
                                                      double* f, bool& fb) {
        const int j = m + 2;
        double avg[NF];
#pragma unroll
        for (int k = 0; k < NF; k++) avg[k] = 0.5 * (W[at<STRW>(j, k, l)] + W[at<STRW>(j + 1, k, l)]);
        const double rh = Five::rho(avg);
        const double kk = s.kapila_k<FAST>(avg);
        double c;
        {
            double d, b;
            s.db<FAST>(avg, d, b);
            c = Five::sound_speed_rc2<FAST>(avg, s.rho_c2_db<FAST>(avg, d, b, kk));
        }
        const double c2 = c * c;
        double l0p, l1p, l2u, l2p, l5u, l5p, l6p;  // rows of L (multiphase.rs:202-220)
        double r0, r1, ru2, ru5, r6;               // columns of R (multiphase.rs:222-236)
        if constexpr (FAST) {
            const double irh = rcp_f(rh), ic = rcp_f(c), ic2 = ic * ic;
            l0p = -avg[0] * irh * ic2;
            l1p = -avg[1] * irh * ic2;
            l2u = -0.5 * rh * ic;
            l2p = 0.5 * ic2;
            l5u = 0.5 * rh * ic;
            l5p = 0.5 * ic2;
            l6p = kk * irh * ic2;
            r0 = avg[0] * irh;
            r1 = avg[1] * irh;
            ru2 = -c * irh;
            ru5 = c * irh;
            r6 = -kk * irh;
        } else {
            l0p = -avg[0] / rh / c2;
            l1p = -avg[1] / rh / c2;
            l2u = -rh / (2.0 * c);
            l2p = 1.0 / (2.0 * c2);
            l5u = rh / (2.0 * c);
            l5p = 1.0 / (2.0 * c2);
            l6p = kk / rh / c2;
            r0 = avg[0] / rh;
            r1 = avg[1] / rh;
            ru2 = -1.0 * c / rh;
            ru5 = 1.0 * c / rh;
            r6 = -kk / rh;
        }
        double cl[NF], cr[NF];
#pragma unroll
        for (int a = 0; a < NF; a++) {
            double ch[6];
#pragma unroll
            for (int s6 = 0; s6 < 6; s6++) {
                const int row = m + s6;
                switch (a) {
                    case 0: ch[s6] = W[at<STRW>(row, 0, l)] + l0p * W[at<STRW>(row, F_IP, l)]; break;
                    case 1: ch[s6] = W[at<STRW>(row, 1, l)] + l1p * W[at<STRW>(row, F_IP, l)]; break;
                    case 2: ch[s6] = l2u * W[at<STRW>(row, UN, l)] + l2p * W[at<STRW>(row, F_IP, l)]; break;
                    case 3: ch[s6] = W[at<STRW>(row, T1, l)]; break;
                    case 4: ch[s6] = W[at<STRW>(row, T2, l)]; break;
                    case 5: ch[s6] = l5u * W[at<STRW>(row, UN, l)] + l5p * W[at<STRW>(row, F_IP, l)]; break;
                    default: ch[s6] = l6p * W[at<STRW>(row, F_IP, l)] + W[at<STRW>(row, F_IA, l)];
                }
            }
            if constexpr (FAST) {
                cl[a] = weno5z_interp_f(ch[0], ch[1], ch[2], ch[3], ch[4]);
                cr[a] = weno5z_interp_f(ch[5], ch[4], ch[3], ch[2], ch[1]);
            } else {
                cl[a] = weno5z_interp(ch[0], ch[1], ch[2], ch[3], ch[4]);
                cr[a] = weno5z_interp(ch[5], ch[4], ch[3], ch[2], ch[1]);
            }
        }
        // back-projection (columns of R in the reference's order)
        double wl[NF], wr[NF];
        wl[0] = (cl[0] + r0 * cl[2]) + r0 * cl[5];
        wr[0] = (cr[0] + r0 * cr[2]) + r0 * cr[5];
        wl[1] = (cl[1] + r1 * cl[2]) + r1 * cl[5];
        wr[1] = (cr[1] + r1 * cr[2]) + r1 * cr[5];
        wl[UN] = ru2 * cl[2] + ru5 * cl[5];
        wr[UN] = ru2 * cr[2] + ru5 * cr[5];
        wl[T1] = cl[3];
        wr[T1] = cr[3];
        wl[T2] = cl[4];
        wr[T2] = cr[4];
        wl[F_IP] = c2 * cl[2] + c2 * cl[5];
        wr[F_IP] = c2 * cr[2] + c2 * cr[5];
        wl[F_IA] = (r6 * cl[2] + r6 * cl[5]) + cl[6];
        wr[F_IA] = (r6 * cr[2] + r6 * cr[5]) + cr[6];
        fb = false;
        Five::St stl = s.state<FAST>(wl), str_ = s.state<FAST>(wr);
        if (!Five::admissible_rc2(wl, stl.rc2) || !Five::admissible_rc2(wr, str_.rc2)) {
            fb = true;
#pragma unroll
            for (int k = 0; k < NF; k++) {
                wl[k] = W[at<STRW>(j, k, l)];
                wr[k] = W[at<STRW>(j + 1, k, l)];
            }
            stl = s.state<FAST>(wl);
            str_ = s.state<FAST>(wr);
        }
        return s.riemann_st<FAST>(wl, wr, stl, str_, UN, f);
    }

    // KEEP-PE two-point flux with cached ρe (multiphase.rs:291-309)
    __device__ static __forceinline__ void split_flux(const double* __restrict__ W, int ra, int rb, int l, double* f) {
        double a[NF + 1], b[NF + 1];
#pragma unroll
        for (int k = 0; k <= NF; k++) {
            a[k] = W[at<STRW>(ra, k, l)];
            b[k] = W[at<STRW>(rb, k, l)];
        }
        const double u = 0.5 * (a[UN] + b[UN]);
        const double rh = 0.5 * (Five::rho(a) + Five::rho(b));
        const double c = rh * u;
        f[0] = 0.5 * (a[0] + b[0]) * u;
        f[1] = 0.5 * (a[1] + b[1]) * u;
        f[2] = c * 0.5 * (a[2] + b[2]);
        f[3] = c * 0.5 * (a[3] + b[3]);
        f[4] = c * 0.5 * (a[4] + b[4]);
        f[UN] = f[UN] + 0.5 * (a[F_IP] + b[F_IP]);
        const double kin = c * 0.5 * (a[2] * b[2] + a[3] * b[3] + a[4] * b[4]);
        const double rhoe = 0.5 * (a[NF] + b[NF]);
        const double pw = 0.5 * (a[UN] * b[F_IP] + b[UN] * a[F_IP]);
        f[5] = kin + u * rhoe + pw;
        f[6] = 0.5 * (a[F_IA] + b[F_IA]) * u;
    }

    // one-sided admissibility of the limiter (scheme.rs:408-416)
    __device__ static __forceinline__ bool lim_ok(const Five& s, const double* fx, const double* ul, const double* fl,
                                                  const double* ur, const double* fr, double lam2) {
        double a[NF], w[NF], d, b;
#pragma unroll
        for (int k = 0; k < NF; k++) a[k] = ul[k] - lam2 * (fx[k] - fl[k]);
        s.to_prim_db<FAST>(a, w, d, b);
        if (!Five::admissible_rc2(w, s.rho_c2_db<FAST>(w, d, b, s.kapila_k<FAST>(w)))) return false;
#pragma unroll
        for (int k = 0; k < NF; k++) a[k] = ur[k] + lam2 * (fx[k] - fr[k]);
        s.to_prim_db<FAST>(a, w, d, b);
        return Five::admissible_rc2(w, s.rho_c2_db<FAST>(w, d, b, s.kapila_k<FAST>(w)));
    }

    __device__ static __forceinline__ double d4(double q0, double q1, double q2, double q3, double q4) {
        return fabs(q0 - 4.0 * q1 + 6.0 * q2 - 4.0 * q3 + q4);
    }

    __device__ static void run(const FiveSweepParams& p) {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        unsigned char* sp = smem_raw;
        double* W = reinterpret_cast<double*>(sp);
        sp += (size_t)RS * STRW * sizeof(double);
        double* MF = nullptr;
        if constexpr (MID) {
            MF = reinterpret_cast<double*>(sp);
            sp += (size_t)SM::RSM * STR * sizeof(double);
        }
        double* F = reinterpret_cast<double*>(sp);
        sp += (size_t)SM::RSF * STR * sizeof(double);
        double* TH = reinterpret_cast<double*>(sp);

        __shared__ unsigned int s_fallback, s_limited, s_weno;
        __shared__ int64_t s_loff[P];
        __shared__ int s_lok[P];
        if (p.ctl->done) return;
        const double dt = p.ctl->dt;
        const int tid = threadIdx.x;
        if (tid == 0) {
            s_fallback = 0;
            s_limited = 0;
            s_weno = 0;
        }
        // uniform grids: x = lane tile, y = segment, z = other-axis row;
        // AMR batches: x = (leaf, group of other-axis rows), one segment
        const int lane0 = AMR ? 0 : blockIdx.x * P;
        const int s0 = blockIdx.y * p.seg;
        int Ls = min(p.seg, p.nd - s0);
        int ob = blockIdx.z;
        int64_t blk = 0;
        int slot_id = 0;
        double dx = p.dx;
        __shared__ int s_pen[P];
        // AMR: the blocks of this CTA's chain (pool slots and offsets)
        constexpr int CHN = AMR ? AMR_CHAIN_MAX : 1;
        __shared__ int64_t s_cblk[CHN];
        __shared__ int s_cslot[CHN];
        int nch = 1;
        if constexpr (AMR) {
            const int z = blockIdx.x / p.ngroups;
            int c0 = z;
            const int* slots = p.leaf_slot;
            if (p.chain_off) {
                c0 = p.chain_off[z];
                nch = p.chain_off[z + 1] - c0;
                slots = p.chain_slot;
                if (nch > CHN || nch < 1) {
                    if (BOUNDS_CHECK && tid == 0) atomicCAS(&p.ctl->status, 0, STATUS_BOUNDS);
                    nch = max(1, min(nch, CHN));
                }
            }
            slot_id = slots[c0];
            if (tid < nch) {
                s_cslot[tid] = slots[c0 + tid];
                s_cblk[tid] = (int64_t)slots[c0 + tid] * p.bcell;
            }
            blk = (int64_t)slot_id * p.bcell;
            dx = p.dx_level[p.leaf_level[slot_id]];
            Ls = nch * p.nd;
            if (tid < P) {
                const int la = tid % p.lw, ob1 = (blockIdx.x % p.ngroups) * (P / p.lw) + tid / p.lw;
                s_lok[tid] = la < p.nl && ob1 < p.no;
                s_loff[tid] = (int64_t)(p.gl + la) * p.sl + (int64_t)(p.go + ob1) * p.so;
                s_pen[tid] = p.pen_lane_major ? la * p.no + ob1 : ob1 * p.nl + la;
            }
        } else if (tid < P) {
            const int la = lane0 + tid;
            s_lok[tid] = la < p.nl && ob < p.no;
            s_loff[tid] = (int64_t)(p.gl + la) * p.sl + (int64_t)(p.go + ob) * p.so;
        }
        const int64_t base0 = blk + (int64_t)(p.gd + s0 - 5) * p.sd;
        // padded offset of row r without the lane offset (AMR chains: row r
        // lies in block min((r − 5)/nd, nch − 1), as in the Euler sweep)
        auto rowg = [&](int r) -> int64_t {
            if constexpr (AMR) {
                const int j = r < 5 ? 0 : min((r - 5) / p.nd, nch - 1);
                return s_cblk[j] + (int64_t)(p.gd - 5 + r - p.nd * j) * p.sd;
            } else {
                return base0 + (int64_t)r * p.sd;
            }
        };
        // statistics of an AMR chain: each midpoint (ext 5) or face (ext 1)
        // once per block whose own sweep computes it
        auto chain_mult = [&](int x, int ext) -> unsigned {
            if constexpr (!AMR) {
                return 1u;
            } else {
                const int jhi = min(x / p.nd, nch - 1);
                const int jlo = x < p.nd + ext ? 0 : (x - p.nd - ext) / p.nd + 1;
                return (unsigned)(jhi - jlo + 1);
            }
        };
        const bool tail = AMR || s0 + Ls == p.nd;
        const Five sys = Five::from(p.sys);
        const double lam = (p.ndim * dt) / dx;  // λ = ndim·dt/dx (C/solver.rs:393, C/amr.rs:1245)
        const double lam2 = 2.0 * lam;
        const bool lim_on = p.positivity && lam > 0.0;
        const double inv = 1.0 / dx;
        __syncthreads();
        const int nrounds = (Ls + 5 + RM - 1) / RM;
        const int nrows = Ls + 10;

        for (int r = 0; r < nrounds; r++) {
            // ---- A: rows [lo, hi) → primitives (ρe, sensors)
            {
                const int lo = r == 0 ? 0 : RM * r + AHEAD;
                const int hi = min(RM * r + RM + AHEAD, nrows);
                const int cnt = (hi - lo) * P;
                for (int idx = tid; idx < cnt; idx += T) {
                    int rr, l;
                    if (p.rows_contig) {
                        rr = idx % (hi - lo);
                        l = idx / (hi - lo);
                    } else {
                        rr = idx / P;
                        l = idx % P;
                    }
                    const int row = lo + rr;
                    const int64_t g = rowg(row) + s_loff[l];
                    if (s_lok[l] && in_bounds(p.ctl, g, p.ncell)) {
                        double u[NF], w[NF], d, b;
#pragma unroll
                        for (int k = 0; k < NF; k++) u[k] = __ldg(p.uin + k * p.ncell + g);
                        sys.to_prim_db<FAST>(u, w, d, b);
#pragma unroll
                        for (int k = 0; k < NF; k++) W[at<STRW>(row, k, l)] = w[k];
                        if constexpr (MODE != MODE_WENO) W[at<STRW>(row, NF, l)] = w[F_IP] * d + b;  // ρe (multiphase.rs:71-75)
                        if constexpr (MODE == MODE_HYBRID) {
                            // sensor values (multiphase.rs:379-384)
                            W[at<STRW>(row, NF + 1, l)] = log(fmax(Five::rho(w), 1e-300));
                            W[at<STRW>(row, NF + 2, l)] = log(fmax(w[F_IP] + sys.p_inf_mix(w), 1e-300));
                            W[at<STRW>(row, NF + 3, l)] = w[F_IA];
                        }
                    }
                }
            }
            __syncthreads();
            if constexpr (MODE == MODE_HYBRID) {
                // ---- Θ: faces [RM r, RM r + RM) (scheme.rs:171-182)
                const int f = RM * r + tid / P;
                const int l = tid % P;
                if (s_lok[l] && f <= Ls) {
                    const int i = f + 4;
                    double rr = 0.0;
#pragma unroll
                    for (int k = NF + 1; k < NF + 4; k++) {
                        const double q0 = W[at<STRW>(i - 2, k, l)], q1 = W[at<STRW>(i - 1, k, l)],
                                     q2 = W[at<STRW>(i, k, l)], q3 = W[at<STRW>(i + 1, k, l)],
                                     q4 = W[at<STRW>(i + 2, k, l)], q5 = W[at<STRW>(i + 3, k, l)];
                        rr = fmax(fmax(rr, d4(q0, q1, q2, q3, q4)), d4(q1, q2, q3, q4, q5));
                    }
                    double x = (rr / p.tol - 0.5) / 0.5;
                    if (x < 0.0) x = 0.0;
                    if (x > 1.0) x = 1.0;
                    TH[slot(f) * P + l] = isfinite(rr) ? x * x * (3.0 - 2.0 * x) : 1.0;
                }
                __syncthreads();
            }
            if constexpr (MID) {
                // ---- B: midpoints [RM r, RM r + RM)
                const int m = RM * r + tid / P;
                const int l = tid % P;
                if (s_lok[l] && m < Ls + 5) {
                    bool need = true;
                    if constexpr (MODE == MODE_HYBRID) {
                        need = false;
                        for (int ff = max(m - 4, 0); ff <= min(m, Ls); ff++) need = need || TH[slot(ff) * P + l] > 0.0;
                    }
                    if (need) {
                        double f[NF];
                        bool fb;
                        const double us = midpoint(sys, W, m, l, f, fb);
#pragma unroll
                        for (int k = 0; k < NF; k++) MF[atM(m, k, l)] = f[k];
                        MF[atM(m, NF, l)] = us;
                        if (fb && (m < Ls || tail)) atomicAdd(&s_fallback, chain_mult(m, 5));
                    }
                }
                __syncthreads();
            }
            // ---- C: faces [RM r − 4, RM r + RM − 4)
            {
                const int fidx = RM * r - 4 + tid / P;
                const int l = tid % P;
                if (s_lok[l] && fidx >= 0 && fidx <= Ls) {
                    const int i = fidx + 4;
                    double theta = MODE == MODE_WENO ? 1.0 : 0.0;
                    if constexpr (MODE == MODE_HYBRID) theta = TH[slot(fidx) * P + l];
                    double fh[NF], cen[NF], uf = 0.0, ufc = 0.0;
                    if constexpr (MODE != MODE_WENO) {
                        if (theta < 1.0) {
                            // scheme.rs:188-222 (lags 1..3, pairs in order)
                            constexpr double A6[3] = {0.75, -0.15, 1.0 / 60.0};
#pragma unroll
                            for (int k = 0; k < NF; k++) cen[k] = 0.0;
#pragma unroll
                            for (int li = 0; li < 3; li++) {
                                const int lag = li + 1;
#pragma unroll
                                for (int mm = 0; mm < lag; mm++) {
                                    double ft[NF];
                                    split_flux(W, i - mm, i - mm + lag, l, ft);
#pragma unroll
                                    for (int k = 0; k < NF; k++) cen[k] = cen[k] + 2.0 * A6[li] * ft[k];
                                    ufc = ufc + A6[li] * (W[at<STRW>(i - mm, UN, l)] + W[at<STRW>(i - mm + lag, UN, l)]);
                                }
                            }
                        }
                    }
                    if (theta == 0.0) {
#pragma unroll
                        for (int k = 0; k < NF; k++) fh[k] = cen[k];
                        uf = ufc;
                    } else {
                        if constexpr (MID) {
                            if constexpr (MODE == MODE_HYBRID) {
                                if (fidx < Ls || tail) atomicAdd(&s_weno, chain_mult(fidx, 1));
                            }
                            // F̃ = Σ_s S6[s] (F̂_{+s} + F̂_{−s}) and the same for Ũ (scheme.rs:226-250)
#pragma unroll
                            for (int k = 0; k <= NF; k++) {
                                double acc = 0.0;
                                acc = acc + s6(0) * MF[atM(fidx + 2, k, l)];
                                acc = acc + s6(1) * MF[atM(fidx + 3, k, l)];
                                acc = acc + s6(1) * MF[atM(fidx + 1, k, l)];
                                acc = acc + s6(2) * MF[atM(fidx + 4, k, l)];
                                acc = acc + s6(2) * MF[atM(fidx, k, l)];
                                if (k < NF)
                                    fh[k] = acc;
                                else
                                    uf = acc;
                            }
                            if (theta < 1.0) {  // scheme.rs:270-276
#pragma unroll
                                for (int k = 0; k < NF; k++) fh[k] = theta * fh[k] + (1.0 - theta) * cen[k];
                                uf = theta * uf + (1.0 - theta) * ufc;
                            }
                        }
                    }
                    if (lim_on) {
                        // Hu–Adams–Shu limiter (scheme.rs:395-464) between rows i and i+1
                        double wi[NF], wj[NF], ul[NF], ur[NF], flp[NF], frp[NF];
#pragma unroll
                        for (int k = 0; k < NF; k++) {
                            wi[k] = W[at<STRW>(i, k, l)];
                            wj[k] = W[at<STRW>(i + 1, k, l)];
                        }
                        sys.to_cons<FAST>(wi, ul);
                        sys.to_cons<FAST>(wj, ur);
                        Five::flux_wq(wi, ul, UN, flp);
                        Five::flux_wq(wj, ur, UN, frp);
                        bool finite = true;
#pragma unroll
                        for (int k = 0; k < NF; k++) finite = finite && isfinite(fh[k]);
                        if (!(finite && lim_ok(sys, fh, ul, flp, ur, frp, lam2))) {
                            const double alpha = fmax(fabs(wi[UN]) + sys.sound_speed(wi), fabs(wj[UN]) + sys.sound_speed(wj));
                            double flf[NF], bl[NF];
#pragma unroll
                            for (int k = 0; k < NF; k++) flf[k] = 0.5 * (flp[k] + frp[k]) - 0.5 * alpha * (ur[k] - ul[k]);
                            double lo = 0.0, hi = 1.0;
                            for (int it = 0; it < 30; it++) {
                                const double mid = 0.5 * (lo + hi);
#pragma unroll
                                for (int k = 0; k < NF; k++) bl[k] = isfinite(fh[k]) ? mid * fh[k] + (1.0 - mid) * flf[k] : flf[k];
                                if (lim_ok(sys, bl, ul, flp, ur, frp, lam2))
                                    lo = mid;
                                else
                                    hi = mid;
                            }
#pragma unroll
                            for (int k = 0; k < NF; k++) fh[k] = isfinite(fh[k]) ? lo * fh[k] + (1.0 - lo) * flf[k] : flf[k];
                            const double um = 0.5 * (wi[UN] + wj[UN]);
                            uf = isfinite(uf) ? lo * uf + (1.0 - lo) * um : um;
                            if (fidx < Ls || tail) atomicAdd(&s_limited, chain_mult(fidx, 1));
                        }
                    }
#pragma unroll
                    for (int k = 0; k < NF; k++) F[atF(fidx, k, l)] = fh[k];
                    F[atF(fidx, NF, l)] = uf;
                    if (AMR && fidx % p.nd == 0) {
                        // block boundary faces for refluxing (C/amr.rs:1291-1295): the low
                        // face of block j and the high face of block j − 1 of the chain
                        const int jb = fidx / p.nd;
#pragma unroll
                        for (int side = 0; side < 2; side++) {
                            const int j = jb - side;
                            if (j < 0 || j >= nch) continue;
                            const int64_t f0 = ((((int64_t)s_cslot[j] * 3 + D) * 2 + side) * NF) * p.npen + s_pen[l];
                            if (!in_bounds(p.ctl, f0 + (int64_t)(NF - 1) * p.npen, p.nface)) continue;
                            double* fo = p.face + f0;
#pragma unroll
                            for (int k = 0; k < NF; k++) fo[(int64_t)k * p.npen] = fh[k];
                        }
                    }
                }
            }
            __syncthreads();
            // ---- D: cells [RM r − 5, RM r + RM − 5)
            {
                int c, l;
                if (p.rows_contig) {
                    c = RM * r - 5 + tid % RM;
                    l = tid / RM;
                } else {
                    c = RM * r - 5 + tid / P;
                    l = tid % P;
                }
                const int64_t g = rowg(c + 5) + s_loff[l];
                if (s_lok[l] && c >= 0 && c < Ls && in_bounds(p.ctl, g, p.ncell)) {
                    double res[NF];
#pragma unroll
                    for (int k = 0; k < NF; k++) {
                        // the block solver divides by dx (C/amr.rs:1273), the uniform one multiplies by 1/dx
                        const double df = F[atF(c + 1, k, l)] - F[atF(c, k, l)];
                        const double x = AMR ? df / dx : df * inv;
                        const double prev = p.first ? 0.0 : p.rhs[k * p.ncell + g];
                        res[k] = prev - x;
                    }
                    {
                        // (α + K)(Ũ⁺ − Ũ⁻)/dx of the α equation (solver.rs:440-442)
                        double wc[NF];
#pragma unroll
                        for (int k = 0; k < NF; k++) wc[k] = W[at<STRW>(c + 5, k, l)];
                        const double du = F[atF(c + 1, NF, l)] - F[atF(c, NF, l)];
                        res[F_IA] = res[F_IA] + (AMR ? sys.nc_coef<FAST>(wc) * du / dx : sys.nc_coef<FAST>(wc) * du * inv);
                    }
                    if (!p.last) {
#pragma unroll
                        for (int k = 0; k < NF; k++) p.rhs[k * p.ncell + g] = res[k];
                    } else {
#pragma unroll
                        for (int k = 0; k < NF; k++) {
                            const double o = p.base[k * p.ncell + g];
                            double v;
                            if (p.stage == 1)
                                v = o + dt * res[k];
                            else if (p.stage == 2)
                                v = 0.75 * o + 0.25 * (p.cur[k * p.ncell + g] + dt * res[k]);
                            else
                                v = p.cur[k * p.ncell + g] / 3.0 + (2.0 / 3.0) * (o + dt * res[k]);
                            p.dest[k * p.ncell + g] = v;
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            if (s_weno) atomicAdd(&p.ctl->counters[1], (unsigned long long)s_weno);
            if (s_fallback) atomicAdd(&p.ctl->counters[2], (unsigned long long)s_fallback);
            if (s_limited) atomicAdd(&p.ctl->counters[3], (unsigned long long)s_limited);
        }
    }
};

}  // namespace emg
