// Fused per-axis sweep of the WCNS / HLLC / positivity scheme on sm_100a.
//
// One CTA owns P adjacent pencils (along the "lane" axis) over one segment
// of L interior cells along the sweep axis d. It streams the segment in
// rounds of RM = 256/P rows through shared-memory rings:
//
//   A  load RM new cell rows of the conserved state (SoA f64, coalesced),
//      recover primitives in f64, keep them in the W ring;
//   B  one thread per (midpoint, pencil): characteristic WENO5-Z
//      interpolation to the midpoint and the HLLC flux (MF ring);
//   C  one thread per (face, pencil): 6th-order WCNS combination of five
//      midpoint fluxes, then the Hu–Adams–Shu positivity limiter (F ring);
//   D  one thread per (cell, pencil): the divergence −(F⁺ − F⁻)/dx added to
//      the stage residual; on the last active axis the SSP-RK3 combination
//      is applied in f64 and written straight to the next stage state, and on
//      the third stage the CFL rate of the new state is reduced as well.
//
// Nothing but the state, the residual and the next state touches HBM: the
// primitive array, the midpoint fluxes and the face fluxes of the reference
// GPU design (G/kernels.cu:364-510, each a round trip through global memory)
// live only in shared memory. Midpoints are computed once per pencil segment
// (the reference CPU memoises them per line, C/scheme.rs:148-154).
//
// Index conventions inside a segment with first interior cell s0 (0-based)
// and Ls cells: local row r is padded cell g + s0 − 5 + r along d (row 5 is
// the first interior cell); midpoint m sits between rows m+2 and m+3 and
// reads rows m..m+5; face f (f = 0..Ls) sits between rows f+4 and f+5 and
// combines midpoints f..f+4; cell c (0..Ls−1) is row c+5 and reads faces c
// and c+1.
#pragma once
#include "physics.cuh"
#include "tma.cuh"
#include <stdint.h>

namespace emg {

constexpr int SWEEP_THREADS = 256;
constexpr int AMR_CHAIN_MAX = 8;  // blocks per chain of an AMR sweep


// Device control block of one solver: the time step of the stage kernels is
// read from here so that whole steps can run without a host round trip.
struct StepCtl {
    double dt;                    // step size of the step in flight
    double t;                     // simulation time
    double t_end;                 // stop time of device-driven stepping (+inf: none)
    unsigned long long rate_bits; // max CFL rate of the latest state, as ordered bits of a non-negative double
    unsigned long long steps;     // steps taken on the device
    int done;                     // 1: no further steps (t_end reached or error)
    int status;                   // EMG_* error code raised on the device (0: ok)
    unsigned long long counters[4]; // faces, shock-path faces, fallbacks, limited faces
};

struct SweepParams {
    const double* __restrict__ uin;  // stage input (ghost-filled along d), SoA with field stride ncell
    double* rhs;                     // stage residual, same indexing as uin
    const double* base;              // RK base state ("old"), last axis only
    const double* cur;               // previous value of the RK destination, last axis stages 2-3
    double* dest;                    // RK destination, last axis only
    StepCtl* ctl;
    int64_t ncell;
    int64_t sd, sl, so;  // strides of the sweep, lane and other axes
    int nd, nl, no;      // interior extents
    int gd, gl, go;      // ghost offsets
    int d;               // sweep axis (momentum index 1+d)
    int seg;             // segment length L
    int first, last;     // first / last active axis of the residual
    int stage;           // SSP-RK3 stage 1..3
    int rows_contig;     // sd == 1: rows contiguous in memory
    int cfl_fuse;        // stage 3 of the last axis: reduce the CFL rate
    double dx;           // cell size along d
    double ndim;         // number of active axes (λ = ndim·dt/dx)
    int positivity;      // limiter on/off
    int cfl_active[3];   // active axes for the fused CFL rate
    double cfl_dx[3];
    double tol;          // hybrid sensor tolerance (C/solver.rs:218)
    EosD eos;
    // lanes: lane l sits at lane-axis index lane0 + l % lw and other-axis
    // index ob0 + l / lw (lw = P unless a CTA spans several rows of the other
    // axis, as for the 16-wide AMR blocks)
    int lw;
    // ---- batched block-AMR leaves (amr != 0)
    int amr;
    const int* leaf_slot;   // pool slot of launch leaf z / ngroups
    const int* leaf_level;  // level of each pool slot
    int64_t bcell;          // cells per pool block (ghost-extended)
    int ngroups;            // CTAs per leaf along the other axis
    double dx_level[16];    // cell size along d per level
    double* face;           // boundary face fluxes [slot][d][side][q][pencil]
    int npen;               // pencils per block face (padded)
    int pen_lane_major;     // pencil index = lane*no + other (lane axis is the lower of the two others)
    // optional chains of same-level leaves along d (launch chain z / ngroups is
    // blocks chain_slot[chain_off[z] .. chain_off[z+1]), each the +d neighbour
    // of the one before, at most AMR_CHAIN_MAX): the CTA streams the chain's
    // rows as one pencil, reading the neighbours' interiors at the joints (the
    // values their ghost copies hold); null: one leaf per launch chain
    const int* chain_off;
    const int* chain_slot;
    // ---- batched independent 1-D lines (batch != 0): every lane is one
    // segment of one instance with its own length, dx and dt
    const struct BatchSeg* segs;
    int nseg;
    const double* inst_dx;
    const double* inst_dt;  // 0: instance finished, its segments are skipped
    // optional (uniform grids and batched lines): the limiter's blend weight θ
    // of every face, stored at the index of the face's left cell (1 where the
    // high-order flux was kept); read back by the discrete adjoint
    double* theta_rec;
    int64_t nface;  // elements of `face` (bounds-check build)
};

// index check of the bounds-check build: true when 0 <= i < n; otherwise the
// control block's status becomes EMG_ERR_BOUNDS (first error kept)
__device__ __forceinline__ bool in_bounds(StepCtl* ctl, int64_t i, int64_t n) {
    if constexpr (!BOUNDS_CHECK) {
        return true;
    } else {
        if (i >= 0 && i < n) return true;
        atomicCAS(&ctl->status, 0, STATUS_BOUNDS);
        return false;
    }
}

// A segment of an instance line: `base` is the flat index of the cell five
// rows before its first cell, `len` its cell count.
struct BatchSeg {
    int64_t base;
    int len;
    int inst;
    int tail;  // the instance's last segment (owns the shared boundary midpoints/faces)
    int pad;
};

// Flux modes (C/scheme.rs:39-47), a compile-time parameter of the sweep.
enum SweepMode { MODE_HYBRID = 0, MODE_WENO = 1, MODE_CENTRAL = 2 };

// Ring tag of the fast FP64 form: FP64 rings and arithmetic, with the
// reciprocals and square roots of physics.cuh's fast section
struct F64Fast {};

template <typename R> struct RingTypes {
    static constexpr bool MIXED = false;
    static constexpr bool FAST = false;
};
template <> struct RingTypes<float> {
    static constexpr bool MIXED = true;
    static constexpr bool FAST = false;
};
template <> struct RingTypes<F64Fast> {
    static constexpr bool MIXED = false;
    static constexpr bool FAST = true;
};

// Ring slots: a power of two holding every row one round touches. WENO:
// RM + 5 rows (midpoint stencils); central: RM + 7 (the split-form stencil
// reaches two rows behind the round's first face); hybrid: RM + 9 (plus the
// sensor stencil two rows ahead of the last midpoint).
template <int RM, int MODE> struct RingSize {
    static constexpr int need = RM + (MODE == MODE_HYBRID ? 9 : (MODE == MODE_CENTRAL ? 7 : 5));
    static constexpr int value = need <= 16 ? 16 : (need <= 32 ? 32 : (need <= 64 ? 64 : 128));
};

template <typename RF, int P, int MODE> struct SweepSmem {
    static constexpr int RM = SWEEP_THREADS / P;
    static constexpr int RS = RingSize<RM, MODE>::value;  // W (and TH) ring rows
    // the flux rings hold exactly what one round keeps alive: phase C of round
    // r reads midpoints [RM r − 4, RM r + RM) and phase D faces [RM r − 5,
    // RM r + RM − 4), so RM + 4 and RM + 1 slots (indexed modulo)
    static constexpr int RSM = RM + 4;
    static constexpr int RSF = RM + 1;
    // values per cell in the primitive ring: w(5), plus ρe for the central
    // flux, plus the two sensor logarithms for the hybrid switch
    static constexpr int NW = MODE == MODE_WENO ? 5 : (MODE == MODE_CENTRAL ? 6 : 8);
    // row strides in elements: conflict-free for runs of consecutive rows
    // (16 rows of one pencil when P <= 16, 8 rows × 2 pencils when P = 32)
    static constexpr int STRW = P == 32 ? NW * P + 2 : NW * P + 1;
    static constexpr int STR = P == 32 ? 5 * P + 2 : 5 * P + 1;
    static constexpr bool MID = MODE != MODE_CENTRAL;
    static constexpr size_t bytes() {
        return (size_t)RS * STRW * sizeof(double)                                    // W (f64 primitives, ρe, sensors)
               + (MID ? (size_t)RSM * STR * sizeof(double) : 0)                        // MF (midpoint fluxes)
               + (size_t)RSF * STR * sizeof(double)                                   // F (face fluxes)
               + (MODE == MODE_HYBRID ? (size_t)RS * P * sizeof(double) : 0);         // TH (blend weights)
    }
};

// KIND_GRID_TMA: a uniform 3-D grid whose phase-A rows arrive by TMA (one
// box of the next round's RM rows × P lanes × 5 fields per round, issued a
// round ahead into a shared-memory staging buffer) instead of per-thread loads.
enum SweepKind { KIND_GRID = 0, KIND_AMR = 1, KIND_BATCH = 2, KIND_GRID_TMA = 3 };

// Staging buffer of KIND_GRID_TMA (bytes, plus 128 for its alignment).
template <int P> constexpr size_t tma_stage_bytes() { return (size_t)5 * P * (SWEEP_THREADS / P) * sizeof(double) + 128; }

template <typename RF, int P, int D, int MODE, int KIND = KIND_GRID>
struct Sweep {
    static constexpr bool AMR = KIND == KIND_AMR;
    static constexpr bool BATCH = KIND == KIND_BATCH;
    static constexpr bool TMA = KIND == KIND_GRID_TMA;
    using SM = SweepSmem<RF, P, MODE>;
    static constexpr int T = SWEEP_THREADS;
    static constexpr int RM = T / P;
    static constexpr int RS = SM::RS;
    static constexpr int STR = SM::STR;
    static constexpr int STRW = SM::STRW;
    static constexpr bool MIXED = RingTypes<RF>::MIXED;
    static constexpr bool FAST = RingTypes<RF>::FAST;
    // the fast forms' FP64 maps (one reciprocal of ρ for the primitive
    // recovery, division-free conserved states): the fast FP64 form and the
    // mixed form, whose error is set by its FP32 interpolation
    static constexpr bool FMAPS = FAST || MIXED;
    static constexpr bool MID = SM::MID;
    static constexpr int AHEAD = MODE == MODE_HYBRID ? 7 : 5;  // rows loaded beyond the round's midpoints

    __device__ static __forceinline__ int slot(int x) { return x & (RS - 1); }
    // element (row x, field k, lane l) of a ring with row stride S
    template <int S> __device__ static __forceinline__ int at(int x, int k, int l) { return slot(x) * S + k * P + l; }
    // midpoint and face flux rings (x ≥ 0)
    __device__ static __forceinline__ int atM(int x, int k, int l) {
        return (int)((unsigned)x % (unsigned)SM::RSM) * STR + k * P + l;
    }
    __device__ static __forceinline__ int atF(int x, int k, int l) {
        return (int)((unsigned)x % (unsigned)SM::RSF) * STR + k * P + l;
    }

    // Characteristic WENO5-Z interpolation to midpoint m and its HLLC flux:
    // sparse form of C/scheme.rs:286-333. The zero entries of the Euler
    // eigenvectors (C/system.rs:232-258) are skipped, which leaves every
    // non-zero sum of the dense products unchanged.
    template <int S>
    __device__ static __forceinline__ void midpoint(const Eos<RF>& e, const RF* __restrict__ Wr, int m, int l, RF* f,
                                                    bool& fb) {
        constexpr int un = 1 + D;
        constexpr int t1 = 1 + (D + 1) % 3, t2 = 1 + (D + 2) % 3;
        const int j = m + 2;
        RF avg[5];
#pragma unroll
        for (int k = 0; k < 5; k++) avg[k] = RF(0.5) * (Wr[at<S>(j, k, l)] + Wr[at<S>(j + 1, k, l)]);
        const RF rho = avg[0];
        const RF c = sound_speed(e, avg[0], avg[4]);
        // (−a)/b == −(a/b) exactly, so the negated entries need no division
        const RF l4un = rho / (RF(2) * c);
        const RF l0un = -l4un;
        const RF l04 = RF(1) / (RF(2) * c * c);
        const RF l14 = -RF(1) / (c * c);
        const RF run4 = c / rho;
        const RF run0 = -run4;
        const RF r40 = c * c;
        // one characteristic field at a time: six live stencil values instead
        // of thirty keep the kernel within 80 registers (3 CTAs per SM)
        RF cl[5], cr[5];
#pragma unroll
        for (int a = 0; a < 5; a++) {
            RF ch[6];
#pragma unroll
            for (int s = 0; s < 6; s++) {
                const int row = m + s;
                switch (a) {
                    case 0: ch[s] = l0un * Wr[at<S>(row, un, l)] + l04 * Wr[at<S>(row, 4, l)]; break;
                    case 1: ch[s] = Wr[at<S>(row, 0, l)] + l14 * Wr[at<S>(row, 4, l)]; break;
                    case 2: ch[s] = Wr[at<S>(row, t1, l)]; break;
                    case 3: ch[s] = Wr[at<S>(row, t2, l)]; break;
                    default: ch[s] = l4un * Wr[at<S>(row, un, l)] + l04 * Wr[at<S>(row, 4, l)];
                }
            }
            cl[a] = weno5z_interp(ch[0], ch[1], ch[2], ch[3], ch[4]);
            cr[a] = weno5z_interp(ch[5], ch[4], ch[3], ch[2], ch[1]);
        }
        RF wl[5], wr[5];
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
        fb = false;
        if (!admissible(e, wl[0], wl[4]) || !admissible(e, wr[0], wr[4])) {
            fb = true;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                wl[k] = Wr[at<S>(j, k, l)];
                wr[k] = Wr[at<S>(j + 1, k, l)];
            }
        }
        hllc(e, wl, wr, un, f);
    }

    // Mixed form of the midpoint flux: the characteristic projection, the
    // back-projection, the admissibility test and the HLLC flux in FP64 (its
    // wave-speed bounds from FP32 sound speeds, hllc_fs), with Newton-refined
    // reciprocals (rcp_nr, rsqrt_nr: ~1e-12 relative) in place of the
    // correctly rounded divisions and square root; the
    // ten WENO-Z interpolations (the bulk of the arithmetic) in FP32 on the
    // deviations of each characteristic stencil from its FP64 value at the
    // cell beside the midpoint. WENO-Z is translation invariant (the candidate
    // weights sum to 1, the smoothness indicators use differences only), so
    // the deviation form is the same interpolant in exact arithmetic, and its
    // FP32 rounding scales with the local variation of the data instead of
    // with the state. FP32 HLLC or FP32 interpolation of the raw values leave
    // ~5e-6 relative error in the residual per step; this form ~5e-8.
    __device__ static __forceinline__ void midpoint_mixed(const Eos<double>& e, const double* __restrict__ Wd, int m,
                                                          int l, double* f, bool& fb) {
        constexpr int un = 1 + D;
        constexpr int t1 = 1 + (D + 1) % 3, t2 = 1 + (D + 2) % 3;
        const int j = m + 2;
        const double rho = 0.5 * (Wd[at<STRW>(j, 0, l)] + Wd[at<STRW>(j + 1, 0, l)]);
        const double p4 = 0.5 * (Wd[at<STRW>(j, 4, l)] + Wd[at<STRW>(j + 1, 4, l)]);
        // c² (eos.rs:56-60), 1/c and 1/ρ from three Newton-refined estimates
        // instead of six correctly rounded divisions and a square root
        const double irho = rcp_nr(rho);
        const double c2 = fmax(e.gamma * (p4 + e.p_inf) * irho * irho * rcp_nr(irho - e.b), 0.0);
        const double ic = rsqrt_nr(c2);
        const double c = c2 * ic;
        const double l4un = 0.5 * rho * ic;
        const double l0un = -l4un;
        const double l04 = 0.5 * (ic * ic);
        const double l14 = -(ic * ic);
        const double run4 = c * irho;
        const double run0 = -run4;
        const double r40 = c2;
        double cl[5], cr[5];
#pragma unroll
        for (int a = 0; a < 5; a++) {
            double ch[6];
#pragma unroll
            for (int s2 = 0; s2 < 6; s2++) {
                const int row = m + s2;
                switch (a) {
                    case 0: ch[s2] = l0un * Wd[at<STRW>(row, un, l)] + l04 * Wd[at<STRW>(row, 4, l)]; break;
                    case 1: ch[s2] = Wd[at<STRW>(row, 0, l)] + l14 * Wd[at<STRW>(row, 4, l)]; break;
                    case 2: ch[s2] = Wd[at<STRW>(row, t1, l)]; break;
                    case 3: ch[s2] = Wd[at<STRW>(row, t2, l)]; break;
                    default: ch[s2] = l4un * Wd[at<STRW>(row, un, l)] + l04 * Wd[at<STRW>(row, 4, l)];
                }
            }
            const double bl = ch[2], br = ch[3];
            cl[a] = bl + (double)weno5z_interp<float>((float)(ch[0] - bl), (float)(ch[1] - bl), 0.0f, (float)(ch[3] - bl),
                                                      (float)(ch[4] - bl));
            cr[a] = br + (double)weno5z_interp<float>((float)(ch[5] - br), (float)(ch[4] - br), 0.0f, (float)(ch[2] - br),
                                                      (float)(ch[1] - br));
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
        fb = false;
        if (!admissible_nr(e, wl[0], wl[4]) || !admissible_nr(e, wr[0], wr[4])) {
            fb = true;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                wl[k] = Wd[at<STRW>(j, k, l)];
                wr[k] = Wd[at<STRW>(j + 1, k, l)];
            }
        }
        hllc_fs(e, wl, wr, un, f);
    }

    // Fast FP64 form of the midpoint flux: the arithmetic of `midpoint` in
    // FP64 with FMA contraction, one reciprocal of ρ and one reciprocal square
    // root of c² for the eigenvector coefficients, and the fast WENO5-Z and
    // HLLC of physics.cuh (about one ulp per reciprocal instead of a
    // correctly rounded division).
    __device__ static __forceinline__ void midpoint_fast(const Eos<double>& e, double igm1,
                                                         const double* __restrict__ Wd, int m, int l, double* f,
                                                         bool& fb) {
        constexpr int un = 1 + D;
        constexpr int t1 = 1 + (D + 1) % 3, t2 = 1 + (D + 2) % 3;
        const int j = m + 2;
        const double rho = 0.5 * (Wd[at<STRW>(j, 0, l)] + Wd[at<STRW>(j + 1, 0, l)]);
        const double p4 = 0.5 * (Wd[at<STRW>(j, 4, l)] + Wd[at<STRW>(j + 1, 4, l)]);
        const double c2 = fmax(sound_speed_sq_f(e, rho, p4), 0.0);
        const double ic = rsqrt_f(c2);
        const double c = c2 * ic;
        const double l4un = 0.5 * rho * ic;
        const double l0un = -l4un;
        const double l04 = 0.5 * (ic * ic);
        const double l14 = -(ic * ic);
        const double run4 = c * rcp_f(rho);
        const double run0 = -run4;
        const double r40 = c2;
        double cl[5], cr[5];
#pragma unroll
        for (int a = 0; a < 5; a++) {
            double ch[6];
#pragma unroll
            for (int s2 = 0; s2 < 6; s2++) {
                const int row = m + s2;
                switch (a) {
                    case 0: ch[s2] = l0un * Wd[at<STRW>(row, un, l)] + l04 * Wd[at<STRW>(row, 4, l)]; break;
                    case 1: ch[s2] = Wd[at<STRW>(row, 0, l)] + l14 * Wd[at<STRW>(row, 4, l)]; break;
                    case 2: ch[s2] = Wd[at<STRW>(row, t1, l)]; break;
                    case 3: ch[s2] = Wd[at<STRW>(row, t2, l)]; break;
                    default: ch[s2] = l4un * Wd[at<STRW>(row, un, l)] + l04 * Wd[at<STRW>(row, 4, l)];
                }
            }
            cl[a] = weno5z_interp_f(ch[0], ch[1], ch[2], ch[3], ch[4]);
            cr[a] = weno5z_interp_f(ch[5], ch[4], ch[3], ch[2], ch[1]);
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
        wl[4] = r40 * (cl[0] + cl[4]);
        wr[4] = r40 * (cr[0] + cr[4]);
        fb = false;
        if (!admissible_f(e, wl[0], wl[4]) || !admissible_f(e, wr[0], wr[4])) {
            fb = true;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                wl[k] = Wd[at<STRW>(j, k, l)];
                wr[k] = Wd[at<STRW>(j + 1, k, l)];
            }
        }
        hllc_f(e, igm1, wl, wr, un, f);
    }

    // KEEP-PE two-point flux with cached ρe (C/system.rs:317-334).
    __device__ static __forceinline__ void split_flux(const double* __restrict__ W, int ra, int rb, int l, double* f) {
        constexpr int un = 1 + D;
        double a[6], b[6];
#pragma unroll
        for (int k = 0; k < 6; k++) {
            a[k] = W[at<STRW>(ra, k, l)];
            b[k] = W[at<STRW>(rb, k, l)];
        }
        const double rho = 0.5 * (a[0] + b[0]);
        const double u = 0.5 * (a[un] + b[un]);
        const double c = rho * u;
        f[0] = c;
        f[1] = c * 0.5 * (a[1] + b[1]);
        f[2] = c * 0.5 * (a[2] + b[2]);
        f[3] = c * 0.5 * (a[3] + b[3]);
        f[un] = f[un] + 0.5 * (a[4] + b[4]);
        const double kin = c * 0.5 * (a[1] * b[1] + a[2] * b[2] + a[3] * b[3]);
        const double rhoe = 0.5 * (a[5] + b[5]);
        const double pw = 0.5 * (a[un] * b[4] + b[un] * a[4]);
        f[4] = kin + u * rhoe + pw;
    }

    // 6th-order split-form central flux of the face between rows i and i+1
    // (C/scheme.rs:188-214): Σ over lags 1..3 and their pairs, in order.
    __device__ static __forceinline__ void central_flux(const double* __restrict__ W, int i, int l, double* cen) {
        constexpr double A6[3] = {0.75, -0.15, 1.0 / 60.0};
#pragma unroll
        for (int k = 0; k < 5; k++) cen[k] = 0.0;
#pragma unroll
        for (int li = 0; li < 3; li++) {
            const int lag = li + 1;
#pragma unroll
            for (int m = 0; m < lag; m++) {
                double ft[5];
                split_flux(W, i - m, i - m + lag, l, ft);
#pragma unroll
                for (int k = 0; k < 5; k++) cen[k] = cen[k] + 2.0 * A6[li] * ft[k];
            }
        }
    }

    // Division-free sufficient condition for the admissibility test of a
    // conserved state a of an ideal gas (b = q = p∞ = 0): ρ > 0 and
    // 2ρE − |ρu|² > 0 with a relative margin of 1e-11, values bounded so that
    // nothing over- or underflows. Whenever it holds, the reference's test
    // (to_prim: ein = E/ρ − ½|u|², p = (γ−1)·ein/(1/ρ); then ρ > 0, p > 0,
    // both finite, 1/ρ > 0) holds as well: the computed ein is within a few
    // ulps of (2ρE − |ρu|²)/(2ρ²), far inside the margin. Where it does not
    // hold, the reference's test runs as is, so the decision is always the
    // reference's.
    __device__ static __forceinline__ bool surely_admissible(const double* a) {
        const double r = a[0], E = a[4];
        if (!(r > 1e-100 && r < 1e100 && E > 1e-100 && E < 1e100 && fabs(a[1]) < 1e100 && fabs(a[2]) < 1e100 &&
              fabs(a[3]) < 1e100))
            return false;
        const double m2 = a[1] * a[1] + a[2] * a[2] + a[3] * a[3];
        const double twore = 2.0 * r * E;
        return twore - m2 > 1e-11 * (twore + m2);
    }

    // one-sided admissibility of the limiter (C/scheme.rs:408-416), in f64;
    // `ideal`: the equation of state is an ideal gas with 1 < γ < 100, which
    // admits the division-free test above
    __device__ static __forceinline__ bool lim_ok(const Eos<double>& e, const double* fx, const double* ul,
                                                  const double* fl, const double* ur, const double* fr, double lam2,
                                                  bool ideal) {
        double a[5], w[5];
#pragma unroll
        for (int k = 0; k < 5; k++) a[k] = ul[k] - lam2 * (fx[k] - fl[k]);
        if (!(ideal && surely_admissible(a))) {
            to_prim(e, a, w);
            if (!admissible(e, w[0], w[4])) return false;
        }
#pragma unroll
        for (int k = 0; k < 5; k++) a[k] = ur[k] + lam2 * (fx[k] - fr[k]);
        if (ideal && surely_admissible(a)) return true;
        to_prim(e, a, w);
        return admissible(e, w[0], w[4]);
    }

    __device__ static __forceinline__ double d4(double q0, double q1, double q2, double q3, double q4) {
        return fabs(q0 - 4.0 * q1 + 6.0 * q2 - 4.0 * q3 + q4);  // C/scheme.rs:97-99
    }

    // tm: the stage input as a 4-D tensor map (dims k, j, i, field; box of
    // RM rows along D × P lanes × 1 × 5 fields), KIND_GRID_TMA only
    __device__ static void run(const SweepParams& p, const CUtensorMap* tm = nullptr) {
        extern __shared__ __align__(16) unsigned char smem_raw[];
        unsigned char* sp = smem_raw;
        double* stg = nullptr;  // TMA staging buffer [field][row][lane] (D = 2: [field][lane][row])
        if constexpr (TMA) {
            const uintptr_t a = reinterpret_cast<uintptr_t>(sp);
            stg = reinterpret_cast<double*>(sp + ((128 - (a & 127)) & 127));
            sp += tma_stage_bytes<P>();
        }
        double* W = reinterpret_cast<double*>(sp);
        sp += (size_t)RS * STRW * sizeof(double);
        double* MF = nullptr;  // midpoint fluxes (FP64 in both forms)
        if constexpr (MID) {
            MF = reinterpret_cast<double*>(sp);
            sp += (size_t)SM::RSM * STR * sizeof(double);
        }
        double* F = reinterpret_cast<double*>(sp);
        sp += (size_t)SM::RSF * STR * sizeof(double);
        double* TH = reinterpret_cast<double*>(sp);

        __shared__ unsigned int s_fallback, s_limited, s_weno;
        __shared__ double s_rate[T / 32];

        const StepCtl* ctl = p.ctl;
        if (ctl->done) return;
        const double dt = ctl->dt;
        const int tid = threadIdx.x;
        if (tid == 0) {
            s_fallback = 0;
            s_limited = 0;
            s_weno = 0;
        }
        __shared__ __align__(8) uint64_t s_bar;
        if constexpr (TMA) {
            if (tid == 0) {
                mbar_init(smem_u32(&s_bar), 1);
                fence_mbar_init();
            }
            // published by the lane-table barrier below
        }

        // uniform grids: x = lane tile, y = segment, z = other-axis row;
        // AMR batches: x = (leaf, group of other-axis rows), lanes cover the block
        const int lane0 = AMR ? 0 : blockIdx.x * P;
        const int s0 = blockIdx.y * p.seg;
        int Ls = min(p.seg, p.nd - s0);
        int64_t blk = 0;   // pool offset of the block (AMR) or 0
        int ob0 = blockIdx.z;
        int slot_id = 0;
        double dx = p.dx;
        // AMR: the blocks of this CTA's chain (pool slots and offsets)
        constexpr int CHN = AMR ? AMR_CHAIN_MAX : 1;
        __shared__ int64_t s_cblk[CHN];
        __shared__ int s_cslot[CHN];
        int nch = 1;
        if constexpr (AMR) {
            const int z = blockIdx.x / p.ngroups;
            ob0 = (blockIdx.x % p.ngroups) * (P / p.lw);
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
        }
        __shared__ int64_t s_loff[P];
        __shared__ int s_lok[P];
        __shared__ int s_pen[P];
        __shared__ int s_len[BATCH ? P : 1], s_tail[BATCH ? P : 1];
        __shared__ double s_dt[BATCH ? P : 1], s_dx[BATCH ? P : 1];
        __shared__ int s_maxlen;
        if constexpr (BATCH) {
            if (tid == 0) s_maxlen = 0;
            __syncthreads();
            if (tid < P) {
                const int si = blockIdx.x * P + tid;
                int len = 0;
                if (si < p.nseg) {
                    const BatchSeg sg = p.segs[si];
                    const double dti = p.inst_dt[sg.inst];
                    s_loff[tid] = sg.base;
                    s_dt[tid] = dti;
                    s_dx[tid] = p.inst_dx[sg.inst];
                    s_tail[tid] = sg.tail;
                    len = dti > 0.0 ? sg.len : 0;
                }
                s_len[tid] = len;
                s_lok[tid] = len > 0;
                atomicMax(&s_maxlen, len);
            }
        } else if (tid < P) {
            const int lw = AMR ? p.lw : P;
            const int la = lane0 + tid % lw, ob = ob0 + tid / lw;
            s_lok[tid] = la < p.nl && ob < p.no;
            s_loff[tid] = (int64_t)(p.gl + la) * p.sl + (int64_t)(p.go + ob) * p.so;
            if constexpr (AMR) s_pen[tid] = p.pen_lane_major ? la * p.no + ob : ob * p.nl + la;
        }
        // padded offset of row 0 (lane offsets are added per lane)
        const int64_t base0 = BATCH ? 0 : blk + (int64_t)(p.gd + s0 - 5) * p.sd;
        // padded offset of row r without the lane offset; in an AMR chain row r
        // lies in block min((r − 5)/nd, nch − 1) (the first block's rows start
        // with its 5 low ghost rows, the last block's end with its 5 high ones)
        auto rowg = [&](int r) -> int64_t {
            if constexpr (AMR) {
                const int j = r < 5 ? 0 : min((r - 5) / p.nd, nch - 1);
                return s_cblk[j] + (int64_t)(p.gd - 5 + r - p.nd * j) * p.sd;
            } else {
                return base0 + (int64_t)r * p.sd;
            }
        };
        // statistics: neighbouring segments recompute the 5 midpoints and 1
        // face they share and only the owner counts them; an AMR chain counts
        // each midpoint (ext 5) or face (ext 1) once per block of the chain
        // whose own sweep computes it, as the block-by-block reference does
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
        const Eos<double> ed = Eos<double>::from(p.eos);
        constexpr int un = 1 + D;
        const double lam = (p.ndim * dt) / dx;  // λ = ndim·dt/dx (C/solver.rs:393, C/amr.rs:1246)
        const double lam2 = 2.0 * lam;
        const bool lim_on = p.positivity && lam > 0.0;  // C/scheme.rs:278
        const double inv = 1.0 / dx;
        const bool ideal_gas = ed.b == 0.0 && ed.q == 0.0 && ed.p_inf == 0.0 && ed.gamma > 1.0 && ed.gamma < 100.0;
        const double igm1 = FMAPS ? 1.0 / (ed.gamma - 1.0) : 0.0;  // fast maps: 1/(γ − 1)
        __syncthreads();  // lane table
        const int Lmax = BATCH ? s_maxlen : Ls;
        const int nrounds = (Lmax + 5 + RM - 1) / RM;
        const int nrows = Lmax + 10;
        // per-lane length (batched lines differ), time step and cell size
        auto lane_len = [&](int l) { return BATCH ? s_len[l] : Ls; };
        auto lane_tail = [&](int l) { return BATCH ? s_tail[l] != 0 : tail; };
        double rate_max = 0.0;
        int bad_state = 0;  // a non-finite or inadmissible new state (fused CFL only)

        // TMA: the box of round rr's rows [RM rr + AHEAD, RM rr + AHEAD + RM)
        // (3-D grids: D = 0 rows along i, lanes along k; D = 1 rows along j,
        // lanes along k; D = 2 rows along k, lanes along j; the host enables
        // this kind only where every start coordinate along k is even)
        auto tma_issue = [&](int rr) {
            if constexpr (TMA) {
                const int row0 = p.gd + s0 - 5 + RM * rr + AHEAD;
                const int lane_c = p.gl + lane0, other_c = p.go + ob0;
                int c0, c1, c2;
                if constexpr (D == 0) {
                    c0 = lane_c;
                    c1 = other_c;
                    c2 = row0;
                } else if constexpr (D == 1) {
                    c0 = lane_c;
                    c1 = row0;
                    c2 = other_c;
                } else {
                    c0 = row0;
                    c1 = lane_c;
                    c2 = other_c;
                }
                const uint32_t bar = smem_u32(&s_bar);
                fence_proxy_async();  // the previous round's reads of the buffer come first
                mbar_arrive_expect_tx(bar, (uint32_t)(5 * RM * P * sizeof(double)));
                tma_load_4d(smem_u32(stg), tm, c0, c1, c2, 0, bar);
            }
        };

        for (int r = 0; r < nrounds; r++) {
            // ---- A: load rows [lo, hi) and recover primitives (and ρe, sensors)
            if (TMA && r > 0) {
                // rows of this round staged by TMA (issued during the previous round)
                const int lo = RM * r + AHEAD;
                const int hi = min(RM * r + RM + AHEAD, nrows);
                const uint32_t bar = smem_u32(&s_bar);
                const bool ok = mbar_wait_bounded(bar, (uint32_t)((r - 1) & 1), TMA_WAIT_LIMIT);
                if (__syncthreads_or(!ok)) {
                    // the copy did not land in time: report it, give the copy in
                    // flight one more bounded wait, and leave
                    if (tid == 0) atomicCAS(&p.ctl->status, 0, STATUS_TIMEOUT);
                    mbar_wait_bounded(bar, (uint32_t)((r - 1) & 1), TMA_WAIT_LIMIT);
                    return;
                }
                const int cnt = (hi - lo) * P;
                for (int idx = tid; idx < cnt; idx += T) {
                    int rr, l;
                    if (D == 2) {
                        rr = idx % (hi - lo);
                        l = idx / (hi - lo);
                    } else {
                        rr = idx / P;
                        l = idx % P;
                    }
                    if (s_lok[l] && lo + rr < lane_len(l) + 10) {
                        const int row = lo + rr;
                        double u[5], w[5];
#pragma unroll
                        for (int k = 0; k < 5; k++) u[k] = D == 2 ? stg[(k * P + l) * RM + rr] : stg[(k * RM + rr) * P + l];
                        if constexpr (FMAPS)
                            to_prim_f(ed, u, w);
                        else
                            to_prim(ed, u, w);
#pragma unroll
                        for (int k = 0; k < 5; k++) W[at<STRW>(row, k, l)] = w[k];
                        if constexpr (MODE != MODE_WENO)
                            W[at<STRW>(row, 5, l)] = FMAPS ? rho_e_f(ed, igm1, w[0], w[4]) : ed.rho_e(w[0], w[4]);
                        if constexpr (MODE == MODE_HYBRID) {
                            W[at<STRW>(row, 6, l)] = log(fmax(w[0], 1e-300));
                            W[at<STRW>(row, 7, l)] = log(fmax(w[4] + ed.p_inf, 1e-300));
                        }
                    }
                }
            } else {
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
                    if (s_lok[l] && lo + rr < lane_len(l) + 10 && in_bounds(p.ctl, rowg(lo + rr) + s_loff[l], p.ncell)) {
                        const int row = lo + rr;
                        const int64_t g = rowg(row) + s_loff[l];
                        double u[5], w[5];
#pragma unroll
                        for (int k = 0; k < 5; k++) u[k] = __ldg(p.uin + k * p.ncell + g);
                        if constexpr (FMAPS)
                            to_prim_f(ed, u, w);
                        else
                            to_prim(ed, u, w);
#pragma unroll
                        for (int k = 0; k < 5; k++) {
                            W[at<STRW>(row, k, l)] = w[k];
                        }
                        if constexpr (MODE != MODE_WENO)
                            W[at<STRW>(row, 5, l)] = FMAPS ? rho_e_f(ed, igm1, w[0], w[4]) : ed.rho_e(w[0], w[4]);
                        if constexpr (MODE == MODE_HYBRID) {
                            // sensor values ln ρ, ln(p + p∞) (C/system.rs:409-413)
                            W[at<STRW>(row, 6, l)] = log(fmax(w[0], 1e-300));
                            W[at<STRW>(row, 7, l)] = log(fmax(w[4] + ed.p_inf, 1e-300));
                        }
                    }
                }
            }
            __syncthreads();
            // every thread is done with the staging buffer: fetch the next round's rows
            if (TMA && tid == 0 && r + 1 < nrounds) tma_issue(r + 1);
            if constexpr (MODE == MODE_HYBRID) {
                // ---- Θ: blend weights of faces [RM r, RM r + RM) (C/scheme.rs:171-182)
                const int f = RM * r + tid / P;
                const int l = tid % P;
                if (s_lok[l] && f <= lane_len(l)) {
                    const int i = f + 4;
                    double rr = 0.0;
#pragma unroll
                    for (int k = 6; k < 8; k++) {
                        const double q0 = W[at<STRW>(i - 2, k, l)], q1 = W[at<STRW>(i - 1, k, l)],
                                     q2 = W[at<STRW>(i, k, l)], q3 = W[at<STRW>(i + 1, k, l)],
                                     q4 = W[at<STRW>(i + 2, k, l)], q5 = W[at<STRW>(i + 3, k, l)];
                        rr = fmax(fmax(rr, d4(q0, q1, q2, q3, q4)), d4(q1, q2, q3, q4, q5));
                    }
                    double x = (rr / p.tol - 0.5) / 0.5;
                    if (x < 0.0) x = 0.0;  // Rust clamp(0, 1): NaN stays NaN
                    if (x > 1.0) x = 1.0;
                    TH[slot(f) * P + l] = isfinite(rr) ? x * x * (3.0 - 2.0 * x) : 1.0;
                }
                __syncthreads();
            }
            if constexpr (MID) {
                // ---- B: midpoints [RM r, RM r + RM)
                const int m = RM * r + tid / P;
                const int l = tid % P;
                if (s_lok[l] && m < lane_len(l) + 5) {
                    bool need = true;
                    if constexpr (MODE == MODE_HYBRID) {
                        // only midpoints of faces on the shock path (computed on demand, C/scheme.rs:233-238)
                        need = false;
                        for (int ff = max(m - 4, 0); ff <= min(m, lane_len(l)); ff++) need = need || TH[slot(ff) * P + l] > 0.0;
                    }
                    if (need) {
                        double f[5];
                        bool fb;
                        if constexpr (MIXED)
                            midpoint_mixed(ed, W, m, l, f, fb);
                        else if constexpr (FAST)
                            midpoint_fast(ed, igm1, W, m, l, f, fb);
                        else
                            midpoint<STRW>(ed, W, m, l, f, fb);
#pragma unroll
                        for (int k = 0; k < 5; k++) MF[atM(m, k, l)] = f[k];
                        if (fb && (m < lane_len(l) || lane_tail(l))) atomicAdd(&s_fallback, chain_mult(m, 5));
                    }
                }
                __syncthreads();
            }
            // ---- C: faces [RM r − 4, RM r + RM − 4)
            {
                const int fidx = RM * r - 4 + tid / P;
                const int l = tid % P;
                if (s_lok[l] && fidx >= 0 && fidx <= lane_len(l)) {
                    const int i = fidx + 4;
                    double theta = MODE == MODE_WENO ? 1.0 : 0.0;
                    if constexpr (MODE == MODE_HYBRID) theta = TH[slot(fidx) * P + l];
                    double fh[5], cen[5];
                    if constexpr (MODE != MODE_WENO) {
                        if (theta < 1.0) central_flux(W, i, l, cen);
                    }
                    if (theta == 0.0) {
#pragma unroll
                        for (int k = 0; k < 5; k++) fh[k] = cen[k];
                    } else {
                        if constexpr (MID) {
                            if constexpr (MODE == MODE_HYBRID) {
                                if (fidx < lane_len(l) || lane_tail(l)) atomicAdd(&s_weno, chain_mult(fidx, 1));
                            }
                            // F̃ = Σ_s S6[s] (F̂_{+s} + F̂_{−s}), order as C/scheme.rs:230-246
#pragma unroll
                            for (int k = 0; k < 5; k++) {
                                double acc = 0.0;
                                acc = acc + s6(0) * double(MF[atM(fidx + 2, k, l)]);
                                acc = acc + s6(1) * double(MF[atM(fidx + 3, k, l)]);
                                acc = acc + s6(1) * double(MF[atM(fidx + 1, k, l)]);
                                acc = acc + s6(2) * double(MF[atM(fidx + 4, k, l)]);
                                acc = acc + s6(2) * double(MF[atM(fidx, k, l)]);
                                fh[k] = acc;
                            }
                            if (theta < 1.0) {  // C/scheme.rs:270-276
#pragma unroll
                                for (int k = 0; k < 5; k++) fh[k] = theta * fh[k] + (1.0 - theta) * cen[k];
                            }
                        }
                    }
                    double lam2_l = lam2;
                    bool lim_l = lim_on;
                    if constexpr (BATCH) {
                        const double lm = (p.ndim * s_dt[l]) / s_dx[l];
                        lam2_l = 2.0 * lm;
                        lim_l = p.positivity && lm > 0.0;
                    }
                    double th_rec = 1.0;  // blend weight kept by the limiter (1: untouched)
                    if (lim_l) {
                        // Hu–Adams–Shu limiter (C/scheme.rs:395-464) between rows i and i+1
                        double wi[5], wj[5], ul[5], ur[5], flp[5], frp[5];
#pragma unroll
                        for (int k = 0; k < 5; k++) {
                            wi[k] = W[at<STRW>(i, k, l)];
                            wj[k] = W[at<STRW>(i + 1, k, l)];
                        }
                        if constexpr (FMAPS) {
                            to_cons_f(ed, igm1, wi, ul);
                            to_cons_f(ed, igm1, wj, ur);
                        } else {
                            to_cons(ed, wi, ul);
                            to_cons(ed, wj, ur);
                        }
                        flux_wq(wi, ul, un, flp);
                        flux_wq(wj, ur, un, frp);
                        bool finite = true;
#pragma unroll
                        for (int k = 0; k < 5; k++) finite = finite && isfinite(fh[k]);
                        if (!(finite && lim_ok(ed, fh, ul, flp, ur, frp, lam2_l, ideal_gas))) {
                            const double alpha = fmax(fabs(wi[un]) + sound_speed(ed, wi[0], wi[4]),
                                                      fabs(wj[un]) + sound_speed(ed, wj[0], wj[4]));
                            double flf[5], bl[5];
#pragma unroll
                            for (int k = 0; k < 5; k++) flf[k] = 0.5 * (flp[k] + frp[k]) - 0.5 * alpha * (ur[k] - ul[k]);
                            double lo = 0.0, hi = 1.0;
                            for (int it = 0; it < 30; it++) {
                                const double mid = 0.5 * (lo + hi);
#pragma unroll
                                for (int k = 0; k < 5; k++)
                                    bl[k] = isfinite(fh[k]) ? mid * fh[k] + (1.0 - mid) * flf[k] : flf[k];
                                if (lim_ok(ed, bl, ul, flp, ur, frp, lam2_l, ideal_gas))
                                    lo = mid;
                                else
                                    hi = mid;
                            }
#pragma unroll
                            for (int k = 0; k < 5; k++) fh[k] = isfinite(fh[k]) ? lo * fh[k] + (1.0 - lo) * flf[k] : flf[k];
                            if (fidx < lane_len(l) || lane_tail(l)) atomicAdd(&s_limited, chain_mult(fidx, 1));
                            th_rec = lo;
                        }
                    }
#pragma unroll
                    for (int k = 0; k < 5; k++) F[atF(fidx, k, l)] = fh[k];
                    if (!AMR && p.theta_rec && in_bounds(p.ctl, base0 + (int64_t)i * p.sd + s_loff[l], p.ncell)) {
                        // recorded for the discrete adjoint, at the face's left cell
                        p.theta_rec[base0 + (int64_t)i * p.sd + s_loff[l]] = th_rec;
                    }
                    if (AMR && fidx % p.nd == 0) {
                        // block boundary faces for refluxing (C/amr.rs:1291-1295): the low
                        // face of block j and the high face of block j − 1 of the chain
                        const int jb = fidx / p.nd;
#pragma unroll
                        for (int side = 0; side < 2; side++) {
                            const int j = jb - side;
                            if (j < 0 || j >= nch) continue;
                            const int64_t f0 = ((((int64_t)s_cslot[j] * 3 + D) * 2 + side) * 5) * p.npen + s_pen[l];
                            if (!in_bounds(p.ctl, f0 + 4 * (int64_t)p.npen, p.nface)) continue;
                            double* fo = p.face + f0;
#pragma unroll
                            for (int k = 0; k < 5; k++) fo[(int64_t)k * p.npen] = fh[k];
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
                if (s_lok[l] && c >= 0 && c < lane_len(l) && in_bounds(p.ctl, rowg(c + 5) + s_loff[l], p.ncell)) {
                    const int64_t g = rowg(c + 5) + s_loff[l];
                    const double inv_l = BATCH ? 1.0 / s_dx[l] : inv;
                    const double dt_l = BATCH ? s_dt[l] : dt;
                    double res[5];
#pragma unroll
                    for (int k = 0; k < 5; k++) {
                        // the block solver divides by dx (C/amr.rs:1263), the uniform one multiplies by 1/dx
                        const double df = F[atF(c + 1, k, l)] - F[atF(c, k, l)];
                        const double x = AMR ? df / dx : df * inv_l;
                        const double prev = p.first ? 0.0 : p.rhs[k * p.ncell + g];
                        res[k] = prev - x;
                    }
                    if (AMR || !p.last) {
#pragma unroll
                        for (int k = 0; k < 5; k++) p.rhs[k * p.ncell + g] = res[k];
                    } else {
                        double un_[5];
#pragma unroll
                        for (int k = 0; k < 5; k++) {
                            const double o = p.base[k * p.ncell + g];
                            double v;
                            if (p.stage == 1) {
                                v = o + dt_l * res[k];
                            } else if (p.stage == 2) {
                                v = 0.75 * o + 0.25 * (p.cur[k * p.ncell + g] + dt_l * res[k]);
                            } else {
                                v = p.cur[k * p.ncell + g] / 3.0 + (2.0 / 3.0) * (o + dt_l * res[k]);
                            }
                            p.dest[k * p.ncell + g] = v;
                            un_[k] = v;
                        }
                        if (!BATCH && p.cfl_fuse) {
                            // CFL rate Σ_d (|u_d| + c)/dx_d of the new state (C/solver.rs:485-497);
                            // the mixed and fast forms with the fast maps and reciprocals
                            double w[5];
                            double acc = -0.0;
                            if constexpr (FMAPS) {
                                to_prim_f(ed, un_, w);
                                if (!admissible_f(ed, w[0], w[4])) bad_state = 1;
                                const double cs = sound_speed_f(ed, w[0], w[4]);
#pragma unroll
                                for (int dd = 0; dd < 3; dd++)
                                    if (p.cfl_active[dd]) acc = acc + (fabs(w[1 + dd]) + cs) * rcp_f(p.cfl_dx[dd]);
                            } else {
                                to_prim(ed, un_, w);
                                if (!admissible(ed, w[0], w[4])) bad_state = 1;
                                const double cs = sound_speed(ed, w[0], w[4]);
#pragma unroll
                                for (int dd = 0; dd < 3; dd++)
                                    if (p.cfl_active[dd]) acc = acc + (fabs(w[1 + dd]) + cs) / p.cfl_dx[dd];
                            }
                            rate_max = fmax(rate_max, acc);
                        }
                    }
                }
            }
            // the next round's loads only touch W slots whose rows C has finished
            // with (barrier above), and its C writes F slots after two more barriers
        }
        if (!AMR && !BATCH && p.cfl_fuse) {
            double v = rate_max;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            if ((tid & 31) == 0) s_rate[tid >> 5] = v;
        }
        const int any_bad = __syncthreads_or(bad_state);
        if (tid == 0) {
            if (s_weno) atomicAdd(&p.ctl->counters[1], (unsigned long long)s_weno);
            if (s_fallback) atomicAdd(&p.ctl->counters[2], (unsigned long long)s_fallback);
            if (s_limited) atomicAdd(&p.ctl->counters[3], (unsigned long long)s_limited);
            if (!AMR && !BATCH && p.cfl_fuse) {
                double v = s_rate[0];
                for (int w = 1; w < T / 32; w++) v = fmax(v, s_rate[w]);
                if (!isnan(v) && v > 0.0) atomicMax(&p.ctl->rate_bits, (unsigned long long)__double_as_longlong(v));
                if (any_bad) atomicCAS(&p.ctl->status, 0, 4 /* EMG_ERR_INADMISSIBLE */);
            }
        }
    }
};

}  // namespace emg
