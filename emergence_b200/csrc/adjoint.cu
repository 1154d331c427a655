// Discrete adjoint of the uniform-grid FP64 step (emg_adjoint_*): reverse
// mode through SSP-RK3, the per-axis WCNS / HLLC / positivity-limited flux
// divergence and the ghost fill, with √N checkpointing of the forward run.
//
// The reference has no adjoint (its compressible crate only runs forward);
// this is new work whose forward half is the FP64 step of uniform.cu, bit-exact
// with the reference CPU solver. The time steps of the forward run are
// recorded and held fixed, as are the positivity limiter's blend weights
// (recorded by the forward sweeps) and the admissibility fallbacks (recomputed
// identically): the gradient is that of the discrete map the forward run
// applied.
//
// Per stage s with input X_s and output Y_s = α_s·Uⁿ + β_s·(X_s + dt·R(X_s)):
//   Ūⁿ += α_s·Ȳ_s,  X̄_s = β_s·Ȳ_s + (∂R/∂X_s)ᵀ(β_s·dt·Ȳ_s),  ghosts folded back.
// (∂R/∂X)ᵀ runs as one adjoint sweep per active axis (adj_sweep_kernel): a
// CTA stages four pencils' primitives for a segment of 59 rows plus a 5-row
// halo in shared memory, forms the face-flux cotangents, the Lax–Friedrichs
// part of limited faces, the midpoint-flux cotangents (S6 transposed) and the
// midpoint vector–Jacobian products (adjoint.cuh), gathers them per cell in a
// fixed order (deterministic, no atomics) and maps them through the
// primitive recovery to the conserved cotangent.
//
// Built with -fmad=false like the forward units, so the recomputed forward
// quantities (fallback tests, HLLC wave cases) equal the forward run's.
#include "uniform_internal.h"
#include "adjoint.cuh"
#include "adjoint_launch.h"

#include <cmath>
#include <cstring>
#include <mutex>

namespace emg {

__global__ void aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, int64_t ncell);
__global__ void soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int64_t ncell);

// Shared-memory layout of the adjoint sweep (dynamic, ≈94 KB): primitives and
// their cotangents of ADJ_ROWS rows, face-flux cotangents of ADJ_FACES faces
// (all [row][field][pencil]), and one 30-value slot per thread for the
// stencil cotangents of its midpoint ([s·5 + k][thread]).
constexpr size_t ADJ_SMEM = (size_t)(2 * ADJ_ROWS * 5 * ADJ_P + ADJ_FACES * 5 * ADJ_P + 30 * ADJ_T) * sizeof(double);

struct SmemRows {
    const double* W;
    int row0, l;
    __device__ __forceinline__ double operator()(int s, int k) const { return W[((row0 + s) * 5 + k) * ADJ_P + l]; }
};
struct SlotAcc {
    double* slot;
    int t;
    __device__ __forceinline__ void add(int s, int k, double v) const { slot[(s * 5 + k) * ADJ_T + t] += v; }
};

// Reverse of one axis' contribution −(F_{i+½} − F_{i−½})/dx to the stage
// residual (the forward sweep of sweep.cuh, FP64, WENO flux mode).
template <int D, int KIND>
__global__ void __launch_bounds__(ADJ_T, ADJ_MINB) adj_sweep_kernel(const AdjSweepParams p) {
    extern __shared__ __align__(16) double adj_smem[];
    double* W = adj_smem;                             // [ADJ_ROWS][5][ADJ_P] primitives
    double* AW = W + ADJ_ROWS * 5 * ADJ_P;            // [ADJ_ROWS][5][ADJ_P] primitive cotangents
    double* AF = AW + ADJ_ROWS * 5 * ADJ_P;           // [ADJ_FACES][5][ADJ_P] cotangents of F̃
    double* SLOT = AF + ADJ_FACES * 5 * ADJ_P;        // [30][ADJ_T] midpoint stencil cotangents
    __shared__ double s_g[ADJ_T / 32];
    // per-pencil line geometry: offset of padded row 0, interior cells, owned
    // rows [c0, cend), 1/dx and the residual coefficient β·dt
    __shared__ int64_t s_base[ADJ_P];
    __shared__ int s_n[ADJ_P], s_c0[ADJ_P], s_cend[ADJ_P], s_ok[ADJ_P];
    __shared__ double s_inv[ADJ_P], s_coef[ADJ_P];
    auto at = [](int x, int k, int l) { return (x * 5 + k) * ADJ_P + l; };
    const Eos<double> e = Eos<double>::from(p.eos);
    const int tid = threadIdx.x;
    const int ng = p.ng;
    if (tid < ADJ_P) {
        const int l = tid;
        if constexpr (KIND == 0) {
            const int la = blockIdx.x * ADJ_P + l;
            s_ok[l] = la < p.nl;
            s_base[l] = (int64_t)(p.gl + la) * p.sl + (int64_t)(p.go + blockIdx.z) * p.so;
            s_n[l] = p.nd;
            s_c0[l] = ng - 5 + (int)blockIdx.y * ADJ_L;
            s_inv[l] = p.inv;
            s_coef[l] = p.coef;
        } else {
            const int z = blockIdx.x * ADJ_P + l;
            int ok = 0;
            if (z < p.nlanes) {
                const AdjLane ln = p.lanes[z];
                const double dt = p.inst_dt[ln.inst];
                ok = dt > 0.0;
                s_base[l] = ln.base;
                s_n[l] = ln.n;
                s_c0[l] = ln.c0;
                s_inv[l] = 1.0 / p.inst_dx[ln.inst];
                s_coef[l] = p.beta * dt;
            } else {
                s_base[l] = 0;
                s_n[l] = 0;
                s_c0[l] = 0;
                s_inv[l] = 0.0;
                s_coef[l] = 0.0;
            }
            s_ok[l] = ok;
        }
        s_cend[l] = min(s_c0[l] + ADJ_L, ng + s_n[l] + 5);  // rows beyond receive nothing
    }
    __syncthreads();
    // faces f = 0..n sit right of rows ng−1 .. ng+n−1
    auto lane_ok = [&](int l) { return s_ok[l] != 0; };
    auto loff = [&](int l) { return s_base[l]; };
    double gacc = 0.0;

    // A: primitives of rows [c0 − 5, c0 + L + 5)
    for (int idx = tid; idx < ADJ_ROWS * ADJ_P; idx += ADJ_T) {
        const int x = idx / ADJ_P, l = idx % ADJ_P;
        const int c = s_c0[l] - 5 + x;
        double w[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (lane_ok(l) && c >= 0 && c < s_n[l] + 2 * ng) {
            const int64_t g = loff(l) + (int64_t)c * p.sd;
            double u[5];
#pragma unroll
            for (int k = 0; k < 5; k++) u[k] = p.u[k * p.ncell + g];
            to_prim(e, u, w);
        }
#pragma unroll
        for (int k = 0; k < 5; k++) {
            W[at(x, k, l)] = w[k];
            AW[at(x, k, l)] = 0.0;
        }
    }
    // B: face-flux cotangents. R_c = −(F_{c,c+1} − F_{c−1,c})·inv on interior
    // cells, so F̄_i = (R̄_{i+1} − R̄_i)·inv with R̄ = coef·Ȳ; F̃̄ = θ·F̄.
    auto face_bar = [&](int i, int l, double* fb) {
        const int64_t g = loff(l) + (int64_t)i * p.sd;
        const bool in_l = i >= ng, in_r = i + 1 <= ng + s_n[l] - 1;
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const double rl = in_l ? s_coef[l] * p.ybar[k * p.ncell + g] : 0.0;
            const double rr = in_r ? s_coef[l] * p.ybar[k * p.ncell + g + p.sd] : 0.0;
            fb[k] = (rr - rl) * s_inv[l];
        }
    };
    for (int idx = tid; idx < ADJ_FACES * ADJ_P; idx += ADJ_T) {
        const int x = idx / ADJ_P, l = idx % ADJ_P;
        const int i = s_c0[l] - 5 + x;
        double fb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (lane_ok(l) && i >= ng - 1 && i <= ng + s_n[l] - 1) {
            face_bar(i, l, fb);
            if (p.theta) {
                const double th = p.theta[loff(l) + (int64_t)i * p.sd];
#pragma unroll
                for (int k = 0; k < 5; k++) fb[k] = th * fb[k];
            }
        }
#pragma unroll
        for (int k = 0; k < 5; k++) AF[at(x, k, l)] = fb[k];
    }
    __syncthreads();
    // B': Lax–Friedrichs part (1 − θ)·F_LF of limited faces touching owned
    // rows, into the primitive cotangents of rows i and i+1; faces of one
    // parity never share a row.
    if (p.theta) {
        for (int par = 0; par < 2; par++) {
            for (int idx = tid; idx < ADJ_FACES * ADJ_P; idx += ADJ_T) {
                const int x = idx / ADJ_P, l = idx % ADJ_P;
                const int i = s_c0[l] - 5 + x;
                if (!lane_ok(l) || i < ng - 1 || i > ng + s_n[l] - 1 || (i & 1) != par || i < s_c0[l] - 1 ||
                    i >= s_cend[l])
                    continue;
                const double th = p.theta[loff(l) + (int64_t)i * p.sd];
                if (!(th < 1.0)) continue;
                double fb[5], wi[5], wj[5], wib[5] = {0, 0, 0, 0, 0}, wjb[5] = {0, 0, 0, 0, 0};
                face_bar(i, l, fb);
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    wi[k] = W[at(x, k, l)];
                    wj[k] = W[at(x + 1, k, l)];
                }
                double glf = 0.0;
                adj::lf_vjp<D>(e, wi, wj, th, fb, wib, wjb, glf);
                if (i >= s_c0[l]) gacc += glf;  // face c0 − 1 belongs to the previous segment
#pragma unroll
                for (int k = 0; k < 5; k++) {
                    AW[at(x, k, l)] += wib[k];
                    AW[at(x + 1, k, l)] += wjb[k];
                }
            }
            __syncthreads();
        }
    }
    // C: one thread per (midpoint, pencil). Midpoint j (between rows j, j+1)
    // feeds faces j−2..j+2 with S6 weights (C/scheme.rs:226-250), so its flux
    // cotangent is the S6-weighted sum of theirs.
    {
        const int l = tid % ADJ_P, mj = tid / ADJ_P;  // mj < L + 5
        const int j = s_c0[l] - 3 + mj;
#pragma unroll
        for (int q = 0; q < 30; q++) SLOT[q * ADJ_T + tid] = 0.0;
        if (lane_ok(l) && j >= ng - 3 && j <= ng + s_n[l] + 1) {
            double fb[5];
            bool any = false;
#pragma unroll
            for (int k = 0; k < 5; k++) {
                fb[k] = s6(0) * AF[at(mj + 2, k, l)] + s6(1) * (AF[at(mj + 1, k, l)] + AF[at(mj + 3, k, l)]) +
                        s6(2) * (AF[at(mj, k, l)] + AF[at(mj + 4, k, l)]);
                any = any || fb[k] != 0.0;
            }
            if (any) {
                double gm = 0.0;
                adj::midpoint_vjp_acc<D>(e, SmemRows{W, mj, l}, fb, SlotAcc{SLOT, tid}, gm);
                // neighbouring segments recompute the halo midpoints; only
                // the segment owning row j counts its γ cotangent
                if (j >= s_c0[l] && j < s_cend[l]) gacc += gm;
            }
        }
    }
    __syncthreads();
    // gather: row x collects from the midpoints mj = x−5..x in a fixed order
    for (int idx = tid; idx < ADJ_ROWS * 5 * ADJ_P; idx += ADJ_T) {
        const int x = idx / (5 * ADJ_P), k = (idx / ADJ_P) % 5, l = idx % ADJ_P;
        double acc = AW[at(x, k, l)];
        for (int mj = max(0, x - 5); mj <= min(x, ADJ_L + 4); mj++)
            acc += SLOT[((x - mj) * 5 + k) * ADJ_T + mj * ADJ_P + l];
        AW[at(x, k, l)] = acc;
    }
    __syncthreads();
    // D: owned rows: primitive cotangent → conserved cotangent
    for (int idx = tid; idx < ADJ_L * ADJ_P; idx += ADJ_T) {
        const int x = idx / ADJ_P, l = idx % ADJ_P;
        const int c = s_c0[l] + x;
        if (!lane_ok(l) || c >= s_cend[l]) continue;
        const int64_t g = loff(l) + (int64_t)c * p.sd;
        double u[5], wb[5], ub[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        bool any = false;
#pragma unroll
        for (int k = 0; k < 5; k++) {
            u[k] = p.u[k * p.ncell + g];
            wb[k] = AW[at(x + 5, k, l)];
            any = any || wb[k] != 0.0;
        }
        if (!any) continue;
        adj::to_prim_vjp(e, u, wb, ub, gacc);
#pragma unroll
        for (int k = 0; k < 5; k++) p.xbar[k * p.ncell + g] += ub[k];
    }
    // γ cotangent: fixed-order CTA sum
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gacc += __shfl_xor_sync(0xffffffffu, gacc, o);
    if ((tid & 31) == 0) s_g[tid >> 5] = gacc;
    __syncthreads();
    if (tid == 0 && p.gpart) {
        double s = 0.0;
        for (int w = 0; w < ADJ_T / 32; w++) s += s_g[w];
        p.gpart[((int64_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = s;
    }
}

// Reverse of the ghost fill along axis d (C/solver.rs:278-348 for the
// periodic, outflow, reflecting and Dirichlet kinds on axes with n ≥ ng):
// each ghost cell's cotangent moves to the interior cell it was copied from
// (with the normal momentum negated for reflecting walls; dropped for a
// Dirichlet state) and the ghost's own cotangent is cleared. One thread per
// (line, field), over the padded extents of the two other axes like the forward fill;
// axes run in reverse order (2, 1, 0).
struct AdjGhostParams {
    double* xbar;
    int64_t ncell;
    int64_t m[3], stride[3];
    int n, ng, d, e0, e1;
    int kind[2];
};

// Source cell of ghost layer gi on one side (-1: Dirichlet, no source).
__device__ __forceinline__ int64_t adj_ghost_src(const AdjGhostParams& p, int side, int gi) {
    const int kind = p.kind[side];
    if (kind == EMG_BC_OUTFLOW) return side == 0 ? p.ng : p.n + p.ng - 1;
    if (kind == EMG_BC_PERIODIC) return side == 0 ? p.n + gi : p.ng + gi;
    if (kind == EMG_BC_REFLECT) return side == 0 ? 2 * p.ng - 1 - gi : p.n + p.ng - 1 - gi;
    return -1;
}

constexpr int ADJ_GHOST_MAX = 8;

__global__ void adj_ghost_kernel(const AdjGhostParams p) {
    // one thread per (line, field). The ghost values of a line are gathered
    // first (independent loads), then each side adds its gathered values into
    // its sources: an outflow side folds its layers (gi ascending) into its one
    // source; periodic and reflecting sources of one side are distinct cells
    // for n >= ng. The two sides go one after the other, as their sources may
    // coincide on a short axis.
    const int64_t lines = p.m[p.e0] * p.m[p.e1];
    const int ng = p.ng;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < lines * 5; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t line = t / 5;
        const int k = (int)(t % 5);
        const int64_t a = line / p.m[p.e1], b = line % p.m[p.e1];
        const int64_t base = a * p.stride[p.e0] + b * p.stride[p.e1];
        const int64_t sd = p.stride[p.d];
        double* x = p.xbar + k * p.ncell + base;
        if (ng > ADJ_GHOST_MAX) {
            for (int gi = 0; gi < ng; gi++)
                for (int side = 0; side < 2; side++) {
                    const int64_t dst = (side == 0 ? gi : p.n + ng + gi) * sd;
                    const int64_t src = adj_ghost_src(p, side, gi);
                    const double v = x[dst];
                    x[dst] = 0.0;
                    if (src >= 0 && v != 0.0) x[src * sd] += (p.kind[side] == EMG_BC_REFLECT && k == 1 + p.d) ? -v : v;
                }
            continue;
        }
        double g[2][ADJ_GHOST_MAX];
#pragma unroll
        for (int gi = 0; gi < ADJ_GHOST_MAX; gi++)
            if (gi < ng) {
                g[0][gi] = x[gi * sd];
                g[1][gi] = x[(p.n + ng + gi) * sd];
            }
#pragma unroll
        for (int gi = 0; gi < ADJ_GHOST_MAX; gi++)
            if (gi < ng) {
                x[gi * sd] = 0.0;
                x[(p.n + ng + gi) * sd] = 0.0;
            }
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const int kind = p.kind[side];
            if (kind == EMG_BC_OUTFLOW) {
                double acc = 0.0;
#pragma unroll
                for (int gi = 0; gi < ADJ_GHOST_MAX; gi++)
                    if (gi < ng) acc += g[side][gi];
                if (acc != 0.0) x[adj_ghost_src(p, side, 0) * sd] += acc;
            } else if (kind == EMG_BC_PERIODIC || kind == EMG_BC_REFLECT) {
                const double sg = (kind == EMG_BC_REFLECT && k == 1 + p.d) ? -1.0 : 1.0;
                double s[ADJ_GHOST_MAX];
#pragma unroll
                for (int gi = 0; gi < ADJ_GHOST_MAX; gi++)
                    if (gi < ng) s[gi] = x[adj_ghost_src(p, side, gi) * sd];
#pragma unroll
                for (int gi = 0; gi < ADJ_GHOST_MAX; gi++)
                    if (gi < ng) x[adj_ghost_src(p, side, gi) * sd] = s[gi] + sg * g[side][gi];
            }
        }
    }
}

// Interior-cell combination of the RK reverse: x̄ = beta·ȳ and, when an is
// set, ān (+)= alpha·ȳ (accumulate != 0) or ān = alpha·ȳ.
__global__ void adj_rk_kernel(const double* __restrict__ ybar, double* xbar, double* an, double alpha, double beta,
                              int accumulate, CellRange cr, int64_t ncell) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < cr.cells; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = cr.index(t);
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const double y = ybar[k * ncell + c];
            if (xbar) xbar[k * ncell + c] = beta * y;
            if (an) an[k * ncell + c] = accumulate ? an[k * ncell + c] + alpha * y : alpha * y;
        }
    }
}

// Box objective on interior cells whose centre lo + (i+½)dx lies in
// [blo, bhi] on every active axis: kind 0 = Σ p·vol, kind 1 = Σ E·vol. Writes
// the cotangent ∂J/∂U (zero outside the box) and per-block partial sums of
// J and of ∂J/∂γ at fixed U.
struct BoxParams {
    int active[3];
    double lo[3], dx[3], blo[3], bhi[3];
    double vol;
    int kind;
};

__global__ void adj_objective_kernel(const double* __restrict__ u, double* abar, CellRange cr, int64_t ncell, BoxParams b,
                                     EosD eosd, double* part) {
    __shared__ double sj[ADJ_T / 32], sg[ADJ_T / 32];
    const Eos<double> e = Eos<double>::from(eosd);
    double jacc = 0.0, gacc = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < cr.cells; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t ijk[3] = {t / (cr.n[1] * cr.n[2]), (t / cr.n[2]) % cr.n[1], t % cr.n[2]};
        bool in = true;
        for (int d = 0; d < 3; d++) {
            if (!b.active[d]) continue;
            const double x = b.lo[d] + ((double)ijk[d] + 0.5) * b.dx[d];
            in = in && x >= b.blo[d] && x <= b.bhi[d];
        }
        const int64_t c = cr.index(t);
        double ub[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (in) {
            double uu[5], w[5];
#pragma unroll
            for (int k = 0; k < 5; k++) uu[k] = u[k * ncell + c];
            if (b.kind == 0) {
                to_prim(e, uu, w);
                jacc += w[4] * b.vol;
                const double wb[5] = {0.0, 0.0, 0.0, 0.0, b.vol};
                adj::to_prim_vjp(e, uu, wb, ub, gacc);
            } else {
                jacc += uu[4] * b.vol;
                ub[4] = b.vol;
            }
        }
#pragma unroll
        for (int k = 0; k < 5; k++) abar[k * ncell + c] = ub[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        jacc += __shfl_xor_sync(0xffffffffu, jacc, o);
        gacc += __shfl_xor_sync(0xffffffffu, gacc, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sj[threadIdx.x >> 5] = jacc;
        sg[threadIdx.x >> 5] = gacc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, g = 0.0;
        for (int w = 0; w < ADJ_T / 32; w++) {
            a += sj[w];
            g += sg[w];
        }
        part[2 * blockIdx.x] = a;
        part[2 * blockIdx.x + 1] = g;
    }
}

// out[q] += Σ_b part[stride·b + q] for q < nq, summed in a fixed order.
__global__ void adj_sum_kernel(const double* __restrict__ part, int nblocks, int stride, int nq, double* out) {
    __shared__ double s[ADJ_T];
    for (int q = 0; q < nq; q++) {
        double a = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) a += part[(int64_t)stride * b + q];
        s[threadIdx.x] = a;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[q] += s[0];
        __syncthreads();
    }
}

// Cotangent of the initial primitive state: w̄ = (∂U/∂w)ᵀ Ū at w = to_prim(U)
// (to_cons, C/system.rs:210-217), interior cells; γ part into per-block sums.
__global__ void adj_initial_prim_kernel(const double* __restrict__ u, const double* __restrict__ abar, double* wbar,
                                        CellRange cr, int64_t ncell, EosD eosd, double* part) {
    __shared__ double sg[ADJ_T / 32];
    const Eos<double> e = Eos<double>::from(eosd);
    double gacc = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < cr.cells; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = cr.index(t);
        double uu[5], w[5], qb[5], wb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int k = 0; k < 5; k++) {
            uu[k] = u[k * ncell + c];
            qb[k] = abar[k * ncell + c];
        }
        to_prim(e, uu, w);
        adj::to_cons_vjp(e, w, qb, wb, gacc);
#pragma unroll
        for (int k = 0; k < 5; k++) wbar[k * ncell + c] = wb[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) gacc += __shfl_xor_sync(0xffffffffu, gacc, o);
    if ((threadIdx.x & 31) == 0) sg[threadIdx.x >> 5] = gacc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double g = 0.0;
        for (int w = 0; w < ADJ_T / 32; w++) g += sg[w];
        part[blockIdx.x] = g;
    }
}

// dt of a recorded step into the control block (the forward sweeps read it there).
__global__ void adj_set_dt(StepCtl* ctl, const double* dt) {
    ctl->dt = *dt;
    ctl->done = 0;
    ctl->rate_bits = 0ull;
}

template <int KIND>
cudaError_t adj_sweep_launch_kind(int d, const AdjSweepParams& p, dim3 grid, cudaStream_t s) {
    static std::mutex mu;
    static bool prepared[64] = {};  // dynamic shared-memory opt-in, once per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (!prepared[dev]) {
        cudaError_t e = cudaFuncSetAttribute(adj_sweep_kernel<0, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)ADJ_SMEM);
        if constexpr (KIND == 0) {
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(adj_sweep_kernel<1, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ADJ_SMEM);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(adj_sweep_kernel<2, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ADJ_SMEM);
        }
        if (e != cudaSuccess) return e;
        prepared[dev] = true;
    }
    if constexpr (KIND == 0) {
        if (d == 0)
            adj_sweep_kernel<0, 0><<<grid, ADJ_T, ADJ_SMEM, s>>>(p);
        else if (d == 1)
            adj_sweep_kernel<1, 0><<<grid, ADJ_T, ADJ_SMEM, s>>>(p);
        else
            adj_sweep_kernel<2, 0><<<grid, ADJ_T, ADJ_SMEM, s>>>(p);
    } else {
        adj_sweep_kernel<0, KIND><<<grid, ADJ_T, ADJ_SMEM, s>>>(p);
    }
    return cudaGetLastError();
}

cudaError_t adj_sweep_launch(int d, const AdjSweepParams& p, dim3 grid, cudaStream_t s) {
    return adj_sweep_launch_kind<0>(d, p, grid, s);
}

cudaError_t adj_sweep_launch_batch(const AdjSweepParams& p, cudaStream_t s) {
    const dim3 grid((unsigned)((p.nlanes + ADJ_P - 1) / ADJ_P), 1, 1);
    return adj_sweep_launch_kind<1>(0, p, grid, s);
}

}  // namespace emg

using namespace emg;

// ------------------------------------------------------------------ host object

struct emg_adjoint {
    emg_uniform* f = nullptr;  // forward solver: state, stage buffers, control block, stream
    double* u0 = nullptr;      // initial state (SoA, padded)
    double* ufin = nullptr;    // final state of the recorded run
    uint64_t nsteps = 0;       // steps of the recorded run
    double t_final = 0.0;      // its end time
    std::vector<double> dts;   // their time steps (host copy)
    double* d_dts = nullptr;
    uint64_t dts_cap = 0;
    uint64_t K = 0;            // checkpoint interval
    std::vector<double*> ckpt; // state before steps 0, K, 2K, ...
    double* seg = nullptr;     // stage inputs and blend weights of up to K steps
    uint64_t seg_cap = 0;
    double *a_next = nullptr, *a_n = nullptr, *a_x = nullptr, *a_y = nullptr;
    double* gpart = nullptr;
    int64_t gcap = 0;
    double* dscal = nullptr;   // [0] γ̄ at fixed U, [1] J, [2] γ̄ of the initial primitive map, [3] spare
    bool have_forward = false, seeded = false;
    double ms[3]{};            // device ms: forward, checkpoint recompute, reverse
    int axes[3]{}, naxes = 0;
};

namespace {

int64_t state_doubles(const emg_adjoint* h) { return 5 * h->f->ncell; }
int64_t step_doubles(const emg_adjoint* h) { return (15 + 3 * (int64_t)h->naxes) * h->f->ncell; }
double* seg_x(emg_adjoint* h, uint64_t s, int stage) { return h->seg + s * step_doubles(h) + (stage - 1) * state_doubles(h); }
double* seg_theta(emg_adjoint* h, uint64_t s, int stage, int ai) {
    return h->seg + s * step_doubles(h) + 15 * h->f->ncell + ((stage - 1) * h->naxes + ai) * h->f->ncell;
}

CellRange interior_range(const emg_uniform* f) {
    CellRange cr{};
    for (int d = 0; d < 3; d++) {
        cr.n[d] = f->mesh.n[d];
        cr.g[d] = f->active[d] ? f->mesh.ng : 0;
        cr.stride[d] = f->stride[d];
    }
    cr.cells = f->cells;
    return cr;
}

int grid_for(int64_t work) {
    int64_t b = (work + ADJ_T - 1) / ADJ_T;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 8));
}

EosD eos_of(const emg_uniform* f) { return EosD{f->eos.gamma, f->eos.p_inf, f->eos.b, f->eos.q}; }

int ensure_gpart(emg_adjoint* h, int64_t n) {
    if (n <= h->gcap) return EMG_OK;
    if (h->gpart) cudaFree(h->gpart);
    h->gpart = nullptr;
    EMG_CUDA(cudaMalloc(&h->gpart, n * sizeof(double)));
    h->gcap = n;
    return EMG_OK;
}

// (∂R/∂X)ᵀ(coef·ȳ) added to x̄ over the active axes, then γ̄ partial sums.
int adj_sweeps(emg_adjoint* h, const double* X, double* const* theta, const double* ybar, double coef, double* xbar) {
    emg_uniform* f = h->f;
    for (int ai = 0; ai < h->naxes; ai++) {
        const int d = h->axes[ai];
        const int l = f->lane_axis[d], o = f->other_axis[d];
        AdjSweepParams p{};
        p.u = X;
        p.theta = theta ? theta[ai] : nullptr;
        p.ybar = ybar;
        p.coef = coef;
        p.xbar = xbar;
        p.ncell = f->ncell;
        p.sd = f->stride[d];
        p.sl = f->stride[l];
        p.so = f->stride[o];
        p.nd = (int)f->mesh.n[d];
        p.nl = (int)f->mesh.n[l];
        p.no = (int)f->mesh.n[o];
        p.gl = f->active[l] ? (int)f->mesh.ng : 0;
        p.go = f->active[o] ? (int)f->mesh.ng : 0;
        p.ng = (int)f->mesh.ng;
        p.inv = 1.0 / f->mesh.dx[d];
        p.eos = eos_of(f);
        const dim3 grid((unsigned)((p.nl + ADJ_P - 1) / ADJ_P), (unsigned)((p.nd + 10 + ADJ_L - 1) / ADJ_L),
                        (unsigned)p.no);
        const int64_t nb = (int64_t)grid.x * grid.y * grid.z;
        int rc = ensure_gpart(h, nb);
        if (rc) return rc;
        p.gpart = h->gpart;
        EMG_CUDA(adj_sweep_launch(d, p, grid, f->stream));
        adj_sum_kernel<<<1, ADJ_T, 0, f->stream>>>(h->gpart, (int)nb, 1, 1, h->dscal);
        EMG_CUDA(cudaGetLastError());
        f->launches += 2;
    }
    return EMG_OK;
}

// Reverse ghost fill of x̄ along the active axes, last axis first.
int adj_ghosts(emg_adjoint* h, double* xbar) {
    emg_uniform* f = h->f;
    for (int ai = h->naxes - 1; ai >= 0; ai--) {
        const int d = h->axes[ai];
        AdjGhostParams p{};
        p.xbar = xbar;
        p.ncell = f->ncell;
        for (int k = 0; k < 3; k++) {
            p.m[k] = f->m[k];
            p.stride[k] = f->stride[k];
        }
        p.n = (int)f->mesh.n[d];
        p.ng = (int)f->mesh.ng;
        p.d = d;
        p.e0 = d == 0 ? 1 : 0;
        p.e1 = d == 2 ? 1 : 2;
        p.kind[0] = f->bc[2 * d].kind;
        p.kind[1] = f->bc[2 * d + 1].kind;
        adj_ghost_kernel<<<grid_for(f->m[p.e0] * f->m[p.e1] * 5), ADJ_T, 0, f->stream>>>(p);
        EMG_CUDA(cudaGetLastError());
        f->launches++;
    }
    return EMG_OK;
}

// One forward step from f->u with the time step at dt_dev, keeping its
// stage inputs and the limiter's blend weights in segment slot s.
int record_step(emg_adjoint* h, const double* dt_dev, uint64_t s) {
    emg_uniform* f = h->f;
    const size_t sb = state_doubles(h) * sizeof(double);
    EMG_CUDA(cudaMemcpyAsync(seg_x(h, s, 1), f->u, sb, cudaMemcpyDeviceToDevice, f->stream));
    for (int st = 1; st <= 3; st++)
        for (int ai = 0; ai < h->naxes; ai++) f->theta_rec[st - 1][h->axes[ai]] = seg_theta(h, s, st, ai);
    adj_set_dt<<<1, 1, 0, f->stream>>>(f->ctl, dt_dev);
    EMG_CUDA(cudaGetLastError());
    int rc = launch_step_body(f);
    for (auto& row : f->theta_rec)
        for (auto& t : row) t = nullptr;
    if (rc) return rc;
    EMG_CUDA(cudaMemcpyAsync(seg_x(h, s, 2), f->sa, sb, cudaMemcpyDeviceToDevice, f->stream));
    EMG_CUDA(cudaMemcpyAsync(seg_x(h, s, 3), f->sb, sb, cudaMemcpyDeviceToDevice, f->stream));
    return EMG_OK;
}

// Reverse of a step of size dt recorded in slot s: a_next = Ūⁿ⁺¹ in, Ūⁿ out (in a_next).
int reverse_step(emg_adjoint* h, double dt, uint64_t s) {
    emg_uniform* f = h->f;
    const size_t sb = state_doubles(h) * sizeof(double);
    const CellRange cr = interior_range(f);
    const int g = grid_for(f->cells);
    double* th[3][3];
    for (int st = 1; st <= 3; st++)
        for (int ai = 0; ai < h->naxes; ai++) th[st - 1][ai] = f->opts.positivity ? seg_theta(h, s, st, ai) : nullptr;
    EMG_CUDA(cudaMemsetAsync(h->a_n, 0, sb, f->stream));
    EMG_CUDA(cudaMemsetAsync(h->a_x, 0, sb, f->stream));
    EMG_CUDA(cudaMemsetAsync(h->a_y, 0, sb, f->stream));
    // stage 3: Uⁿ⁺¹ = Uⁿ/3 + ⅔(U² + dt·R(U²))
    adj_rk_kernel<<<g, ADJ_T, 0, f->stream>>>(h->a_next, h->a_x, h->a_n, 1.0 / 3.0, 2.0 / 3.0, 0, cr, f->ncell);
    EMG_CUDA(cudaGetLastError());
    int rc = adj_sweeps(h, seg_x(h, s, 3), f->opts.positivity ? th[2] : nullptr, h->a_next, (2.0 / 3.0) * dt, h->a_x);
    if (rc) return rc;
    if ((rc = adj_ghosts(h, h->a_x))) return rc;
    // stage 2: U² = ¾Uⁿ + ¼(U¹ + dt·R(U¹))
    adj_rk_kernel<<<g, ADJ_T, 0, f->stream>>>(h->a_x, h->a_y, h->a_n, 0.75, 0.25, 1, cr, f->ncell);
    EMG_CUDA(cudaGetLastError());
    if ((rc = adj_sweeps(h, seg_x(h, s, 2), f->opts.positivity ? th[1] : nullptr, h->a_x, 0.25 * dt, h->a_y))) return rc;
    if ((rc = adj_ghosts(h, h->a_y))) return rc;
    // stage 1: U¹ = Uⁿ + dt·R(Uⁿ)
    adj_rk_kernel<<<g, ADJ_T, 0, f->stream>>>(h->a_y, nullptr, h->a_n, 1.0, 1.0, 1, cr, f->ncell);
    EMG_CUDA(cudaGetLastError());
    if ((rc = launch_ghosts(f, seg_x(h, s, 1)))) return rc;  // the slot holds Uⁿ as stored before its ghost fill
    if ((rc = adj_sweeps(h, seg_x(h, s, 1), f->opts.positivity ? th[0] : nullptr, h->a_y, dt, h->a_n))) return rc;
    if ((rc = adj_ghosts(h, h->a_n))) return rc;
    f->launches += 3;
    std::swap(h->a_next, h->a_n);
    return EMG_OK;
}

int ensure_segment(emg_adjoint* h, uint64_t K) {
    if (K <= h->seg_cap) return EMG_OK;
    if (h->seg) cudaFree(h->seg);
    h->seg = nullptr;
    h->seg_cap = 0;
    EMG_CUDA(cudaMalloc(&h->seg, K * step_doubles(h) * sizeof(double)));
    h->seg_cap = K;
    return EMG_OK;
}

int upload_aos(emg_adjoint* h, const double* aos, size_t len, double* dst) {
    emg_uniform* f = h->f;
    if ((int64_t)len != f->ncell) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    EMG_CUDA(cudaMemcpyAsync(f->staging, aos, len * 5 * sizeof(double), cudaMemcpyHostToDevice, f->stream));
    aos_to_soa<<<grid_for(f->ncell), ADJ_T, 0, f->stream>>>(f->staging, dst, f->ncell);
    EMG_CUDA(cudaGetLastError());
    return EMG_OK;
}

int download_aos(emg_adjoint* h, const double* src, double* aos) {
    emg_uniform* f = h->f;
    soa_to_aos<<<grid_for(f->ncell), ADJ_T, 0, f->stream>>>(src, f->staging, f->ncell);
    EMG_CUDA(cudaGetLastError());
    EMG_CUDA(cudaMemcpyAsync(aos, f->staging, f->ncell * 5 * sizeof(double), cudaMemcpyDeviceToHost, f->stream));
    EMG_CUDA(cudaStreamSynchronize(f->stream));
    return EMG_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

}  // namespace

namespace {

int check_adj(emg_adjoint* h) {
    if (!h || !h->f) return set_error(EMG_ERR_INVALID, "null handle");
    return check_handle(h->f);
}

int forward_impl(emg_adjoint* h, uint64_t nsteps, double t_end, uint64_t every, const double* host_dts) {
    emg_uniform* f = h->f;
    if (nsteps == 0 || nsteps > (1ull << 32)) return set_error(EMG_ERR_INVALID, "nsteps must be in [1, 2^32]");
    const uint64_t K = every ? every : (uint64_t)std::ceil(std::sqrt((double)nsteps));
    if (nsteps > h->dts_cap) {
        if (h->d_dts) cudaFree(h->d_dts);
        h->d_dts = nullptr;
        h->dts_cap = 0;
        EMG_CUDA(cudaMalloc(&h->d_dts, nsteps * sizeof(double)));
        h->dts_cap = nsteps;
    }
    if (host_dts)
        EMG_CUDA(cudaMemcpyAsync(h->d_dts, host_dts, nsteps * sizeof(double), cudaMemcpyHostToDevice, f->stream));
    const uint64_t nck = (nsteps + K - 1) / K;
    while (h->ckpt.size() < nck) {
        double* c = nullptr;
        EMG_CUDA(cudaMalloc(&c, state_doubles(h) * sizeof(double)));
        h->ckpt.push_back(c);
    }
    const size_t sb = state_doubles(h) * sizeof(double);
    EMG_CUDA(cudaMemcpyAsync(f->u, h->u0, sb, cudaMemcpyDeviceToDevice, f->stream));
    int rc = sync_ctl(f);
    if (rc) return rc;
    StepCtl c = *f->ctl_host;
    c.t = 0.0;
    c.steps = 0;
    c.t_end = host_dts ? INFINITY : t_end;
    c.done = 0;
    c.status = 0;
    EMG_CUDA(cudaMemcpyAsync(f->ctl, &c, sizeof(StepCtl), cudaMemcpyHostToDevice, f->stream));
    f->rate_valid = false;
    if (!host_dts && (rc = ensure_rate(f))) return rc;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, f->stream);
    const bool bounded = !host_dts && !std::isinf(t_end);
    for (uint64_t n = 0; n < nsteps; n++) {
        if (n % K == 0)
            EMG_CUDA(cudaMemcpyAsync(h->ckpt[n / K], f->u, sb, cudaMemcpyDeviceToDevice, f->stream));
        if (host_dts)
            adj_set_dt<<<1, 1, 0, f->stream>>>(f->ctl, h->d_dts + n);
        else
            ctl_begin_device<<<1, 1, 0, f->stream>>>(f->ctl, f->opts.cfl);
        EMG_CUDA(cudaGetLastError());
        f->launches++;
        if ((rc = launch_step_body(f))) return rc;
        if (!host_dts)
            EMG_CUDA(cudaMemcpyAsync(h->d_dts + n, &f->ctl->dt, sizeof(double), cudaMemcpyDeviceToDevice, f->stream));
        if (bounded && (n + 1) % 8 == 0) {
            if ((rc = sync_ctl(f))) return rc;
            if (f->ctl_host->done) break;
        }
    }
    cudaEventRecord(b, f->stream);
    if ((rc = sync_ctl(f))) return rc;
    h->ms[0] = elapsed(a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (f->ctl_host->status)
        return set_error(f->ctl_host->status, "time step collapsed: the solution lost admissibility");
    h->nsteps = f->ctl_host->steps;
    h->t_final = f->ctl_host->t;
    h->dts.assign(h->nsteps, 0.0);
    if (h->nsteps)
        EMG_CUDA(cudaMemcpy(h->dts.data(), h->d_dts, h->nsteps * sizeof(double), cudaMemcpyDeviceToHost));
    EMG_CUDA(cudaMemcpyAsync(h->ufin, f->u, sb, cudaMemcpyDeviceToDevice, f->stream));
    EMG_CUDA(cudaStreamSynchronize(f->stream));
    h->K = K;
    h->have_forward = h->nsteps > 0;
    h->seeded = false;
    return EMG_OK;
}

int backward_impl(emg_adjoint* h) {
    emg_uniform* f = h->f;
    const uint64_t K = h->K, N = h->nsteps;
    int rc = ensure_segment(h, K);
    if (rc) return rc;
    const size_t sb = state_doubles(h) * sizeof(double);
    const uint64_t nseg = (N + K - 1) / K;
    std::vector<cudaEvent_t> ev(3 * nseg);
    for (auto& e : ev) cudaEventCreate(&e);
    for (uint64_t sg = nseg; sg-- > 0;) {
        const uint64_t n0 = sg * K, n1 = std::min(n0 + K, N);
        cudaEventRecord(ev[3 * sg], f->stream);
        EMG_CUDA(cudaMemcpyAsync(f->u, h->ckpt[sg], sb, cudaMemcpyDeviceToDevice, f->stream));
        for (uint64_t n = n0; n < n1; n++)
            if ((rc = record_step(h, h->d_dts + n, n - n0))) return rc;
        cudaEventRecord(ev[3 * sg + 1], f->stream);
        for (uint64_t n = n1; n-- > n0;)
            if ((rc = reverse_step(h, h->dts[n], n - n0))) return rc;
        cudaEventRecord(ev[3 * sg + 2], f->stream);
    }
    EMG_CUDA(cudaStreamSynchronize(f->stream));
    h->ms[1] = h->ms[2] = 0.0;
    for (uint64_t sg = 0; sg < nseg; sg++) {
        h->ms[1] += elapsed(ev[3 * sg], ev[3 * sg + 1]);
        h->ms[2] += elapsed(ev[3 * sg + 1], ev[3 * sg + 2]);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return EMG_OK;
}

// Ū⁰ (conserved), W̄⁰ (primitive) and γ̄ [U⁰ fixed, W⁰ fixed] from a_next.
int finish_outputs(emg_adjoint* h, const double* ustate, double* ubar0_aos, double* wbar0_aos, double* gamma_bar) {
    emg_uniform* f = h->f;
    const CellRange cr = interior_range(f);
    const int g = grid_for(f->cells);
    int rc = ensure_gpart(h, g);
    if (rc) return rc;
    EMG_CUDA(cudaMemsetAsync(h->a_x, 0, state_doubles(h) * sizeof(double), f->stream));
    EMG_CUDA(cudaMemsetAsync(h->dscal + 2, 0, sizeof(double), f->stream));
    adj_initial_prim_kernel<<<g, ADJ_T, 0, f->stream>>>(ustate, h->a_next, h->a_x, cr, f->ncell, eos_of(f), h->gpart);
    adj_sum_kernel<<<1, ADJ_T, 0, f->stream>>>(h->gpart, g, 1, 1, h->dscal + 2);
    EMG_CUDA(cudaGetLastError());
    if (ubar0_aos && (rc = download_aos(h, h->a_next, ubar0_aos))) return rc;
    if (wbar0_aos && (rc = download_aos(h, h->a_x, wbar0_aos))) return rc;
    double sc[4];
    EMG_CUDA(cudaMemcpyAsync(sc, h->dscal, sizeof sc, cudaMemcpyDeviceToHost, f->stream));
    EMG_CUDA(cudaStreamSynchronize(f->stream));
    if (gamma_bar) {
        gamma_bar[0] = sc[0];
        gamma_bar[1] = sc[0] + sc[2];
    }
    return EMG_OK;
}

}  // namespace

extern "C" {

int emg_adjoint_create(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                       const double* u_aos, size_t len, emg_adjoint** out) {
    if (!mesh || !eos || !bc || !opts || !u_aos || !out) return set_error(EMG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (opts->precision != EMG_PRECISION_F64) return set_error(EMG_ERR_INVALID, "the adjoint differentiates the FP64 form");
    if (opts->mode != EMG_MODE_WENO) return set_error(EMG_ERR_INVALID, "the adjoint supports the WENO flux mode");
    for (int d = 0; d < 3; d++) {
        if (mesh->n[d] <= 1) continue;
        if (mesh->n[d] < mesh->ng) return set_error(EMG_ERR_INVALID, "the adjoint needs n >= ng on every active axis");
        for (int s = 0; s < 2; s++)
            if (bc[2 * d + s].kind == EMG_BC_CHARACTERISTIC)
                return set_error(EMG_ERR_INVALID, "the adjoint supports periodic, outflow, reflect and Dirichlet boundaries");
    }
    emg_uniform* f = nullptr;
    int rc = emg_uniform_create(mesh, eos, bc, opts, u_aos, len, &f);
    if (rc) return rc;
    emg_adjoint* h = new emg_adjoint();
    h->f = f;
    for (int d = 0; d < 3; d++)
        if (f->active[d]) h->axes[h->naxes++] = d;
    const size_t sb = state_doubles(h) * sizeof(double);
    cudaError_t e = cudaSuccess;
    double** bufs[] = {&h->u0, &h->ufin, &h->a_next, &h->a_n, &h->a_x, &h->a_y};
    for (double** b : bufs)
        if (e == cudaSuccess) e = cudaMalloc(b, sb);
    if (e == cudaSuccess) e = cudaMalloc(&h->dscal, 4 * sizeof(double));
    if (e == cudaSuccess) e = cudaMemsetAsync(h->dscal, 0, 4 * sizeof(double), f->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->u0, f->u, sb, cudaMemcpyDeviceToDevice, f->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(f->stream);
    if (e != cudaSuccess) {
        emg_adjoint_destroy(h);
        return set_error(EMG_ERR_CUDA, std::string("adjoint buffers: ") + cudaGetErrorString(e));
    }
    *out = h;
    return EMG_OK;
}

int emg_adjoint_destroy(emg_adjoint* h) {
    if (!h) return EMG_OK;
    if (h->f) cudaSetDevice(h->f->device);
    double* bufs[] = {h->u0, h->ufin, h->a_next, h->a_n, h->a_x, h->a_y, h->dscal, h->gpart, h->seg, h->d_dts};
    for (double* b : bufs)
        if (b) cudaFree(b);
    for (double* c : h->ckpt) cudaFree(c);
    if (h->f) emg_uniform_destroy(h->f);
    delete h;
    return EMG_OK;
}

int emg_adjoint_set_initial(emg_adjoint* h, const double* u_aos, size_t len) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!u_aos) return set_error(EMG_ERR_INVALID, "null state");
    if ((rc = upload_aos(h, u_aos, len, h->u0))) return rc;
    EMG_CUDA(cudaStreamSynchronize(h->f->stream));
    h->have_forward = h->seeded = false;
    return EMG_OK;
}

int emg_adjoint_forward(emg_adjoint* h, uint64_t nsteps, double t_end, uint64_t checkpoint_every, uint64_t* taken) {
    int rc = check_adj(h);
    if (rc) return rc;
    rc = forward_impl(h, nsteps, t_end, checkpoint_every, nullptr);
    if (taken) *taken = h->nsteps;
    return rc;
}

int emg_adjoint_forward_dts(emg_adjoint* h, const double* dts, uint64_t nsteps, uint64_t checkpoint_every) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!dts) return set_error(EMG_ERR_INVALID, "null time steps");
    for (uint64_t n = 0; n < nsteps; n++)
        if (!(std::isfinite(dts[n]) && dts[n] > 0.0)) return set_error(EMG_ERR_INVALID, "time steps must be finite and > 0");
    return forward_impl(h, nsteps, INFINITY, checkpoint_every, dts);
}

int emg_adjoint_dts(emg_adjoint* h, double* out, size_t cap, uint64_t* nsteps) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (nsteps) *nsteps = h->nsteps;
    if (out) {
        if (cap < h->dts.size()) return set_error(EMG_ERR_INVALID, "buffer too small");
        std::memcpy(out, h->dts.data(), h->dts.size() * sizeof(double));
    }
    return EMG_OK;
}

int emg_adjoint_download(emg_adjoint* h, double* u_aos, size_t len) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!u_aos) return set_error(EMG_ERR_INVALID, "null buffer");
    if ((int64_t)len != h->f->ncell) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    return download_aos(h, h->have_forward ? h->ufin : h->u0, u_aos);
}

int emg_adjoint_objective(emg_adjoint* h, int kind, const double box_lo[3], const double box_hi[3], double* J) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!h->have_forward) return set_error(EMG_ERR_INVALID, "no recorded forward run");
    if (kind != EMG_OBJ_PRESSURE && kind != EMG_OBJ_ENERGY) return set_error(EMG_ERR_INVALID, "unknown objective");
    if (!box_lo || !box_hi) return set_error(EMG_ERR_INVALID, "null box");
    emg_uniform* f = h->f;
    BoxParams b{};
    b.vol = 1.0;
    for (int d = 0; d < 3; d++) {
        b.active[d] = f->active[d];
        b.lo[d] = f->mesh.lo[d];
        b.dx[d] = f->mesh.dx[d];
        b.blo[d] = box_lo[d];
        b.bhi[d] = box_hi[d];
        if (f->active[d]) b.vol = b.vol * f->mesh.dx[d];
    }
    b.kind = kind;
    const int g = grid_for(f->cells);
    if ((rc = ensure_gpart(h, 2 * (int64_t)g))) return rc;
    EMG_CUDA(cudaMemsetAsync(h->a_next, 0, state_doubles(h) * sizeof(double), f->stream));
    EMG_CUDA(cudaMemsetAsync(h->dscal, 0, 4 * sizeof(double), f->stream));
    adj_objective_kernel<<<g, ADJ_T, 0, f->stream>>>(h->ufin, h->a_next, interior_range(f), f->ncell, b, eos_of(f),
                                                     h->gpart);
    // dscal[1] += Σ J partials, dscal[0] += Σ γ partials: sum into [1] and [0] via a two-entry scratch
    adj_sum_kernel<<<1, ADJ_T, 0, f->stream>>>(h->gpart, g, 2, 2, h->dscal + 2);
    EMG_CUDA(cudaGetLastError());
    double sc[4];
    EMG_CUDA(cudaMemcpyAsync(sc, h->dscal, sizeof sc, cudaMemcpyDeviceToHost, f->stream));
    EMG_CUDA(cudaStreamSynchronize(f->stream));
    // γ̄ accumulator starts at ∂J/∂γ (fixed U); dscal[2..3] were scratch
    const double init[4] = {sc[3], sc[2], 0.0, 0.0};
    EMG_CUDA(cudaMemcpyAsync(h->dscal, init, sizeof init, cudaMemcpyHostToDevice, f->stream));
    EMG_CUDA(cudaStreamSynchronize(f->stream));
    if (J) *J = sc[2];
    h->seeded = true;
    return EMG_OK;
}

int emg_adjoint_seed(emg_adjoint* h, const double* ubar_aos, size_t len) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!h->have_forward) return set_error(EMG_ERR_INVALID, "no recorded forward run");
    if (!ubar_aos) return set_error(EMG_ERR_INVALID, "null cotangent");
    if ((rc = upload_aos(h, ubar_aos, len, h->a_next))) return rc;
    EMG_CUDA(cudaMemsetAsync(h->dscal, 0, 4 * sizeof(double), h->f->stream));
    EMG_CUDA(cudaStreamSynchronize(h->f->stream));
    h->seeded = true;
    return EMG_OK;
}

int emg_adjoint_backward(emg_adjoint* h, double* ubar0_aos, double* wbar0_aos, double gamma_bar[2]) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!h->have_forward) return set_error(EMG_ERR_INVALID, "no recorded forward run");
    if (!h->seeded) return set_error(EMG_ERR_INVALID, "no cotangent seeded (emg_adjoint_objective or emg_adjoint_seed)");
    if ((rc = backward_impl(h))) return rc;
    h->seeded = false;
    return finish_outputs(h, h->u0, ubar0_aos, wbar0_aos, gamma_bar);
}

int emg_adjoint_step_vjp(emg_adjoint* h, const double* u_aos, size_t len, double dt, const double* ubar_next_aos,
                         double* ubar_aos, double* gamma_bar) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!u_aos || !ubar_next_aos || !ubar_aos) return set_error(EMG_ERR_INVALID, "null argument");
    if (!(std::isfinite(dt) && dt > 0.0)) return set_error(EMG_ERR_INVALID, "dt must be finite and > 0");
    emg_uniform* f = h->f;
    if ((rc = ensure_segment(h, 1))) return rc;
    if ((rc = upload_aos(h, u_aos, len, f->u))) return rc;
    EMG_CUDA(cudaMemcpyAsync(h->dscal + 3, &dt, sizeof(double), cudaMemcpyHostToDevice, f->stream));
    if ((rc = record_step(h, h->dscal + 3, 0))) return rc;
    if ((rc = upload_aos(h, ubar_next_aos, len, h->a_next))) return rc;
    EMG_CUDA(cudaMemsetAsync(h->dscal, 0, sizeof(double), f->stream));
    if ((rc = reverse_step(h, dt, 0))) return rc;
    if ((rc = download_aos(h, h->a_next, ubar_aos))) return rc;
    double g = 0.0;
    EMG_CUDA(cudaMemcpy(&g, h->dscal, sizeof(double), cudaMemcpyDeviceToHost));
    if (gamma_bar) *gamma_bar = g;
    h->seeded = false;
    return EMG_OK;
}

int emg_adjoint_times(emg_adjoint* h, double ms[3]) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!ms) return set_error(EMG_ERR_INVALID, "null buffer");
    for (int k = 0; k < 3; k++) ms[k] = h->ms[k];
    return EMG_OK;
}

int emg_adjoint_stream(emg_adjoint* h, void** stream) {
    int rc = check_adj(h);
    if (rc) return rc;
    if (!stream) return set_error(EMG_ERR_INVALID, "null pointer");
    *stream = (void*)h->f->stream;
    return EMG_OK;
}

}  // extern "C"
