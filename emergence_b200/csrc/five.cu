// Two-phase five-equation solver on uniform grids: host object, ghost and
// CFL kernels and the C ABI of include/emergence_b200.h (emg_five_*).
//
// Replaces compressible-cuda's GpuSolver for GpuSystem::FiveEq (fluid/crates/
// compressible-cuda/src/lib.rs:155-477 with the `five` kernels of
// kernels.cu:116-256), and follows the reference CPU solver's Solver<7,
// FiveEq> step (fluid/crates/compressible/src/solver.rs:351-523,659-738) for
// parity. Per RK stage: one ghost launch per active axis and one fused sweep
// per active axis (five_sweep.cuh), the RK combination fused into the last
// one; the CFL step (acoustic rate and the dilatation limit of the α term)
// by one reduction kernel.
//
// Built with -fmad=false.
#include "../../include/emergence_b200.h"
#include "five_launch.h"
#include "uniform_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace emg;

namespace emg {
int kernel_grid(int64_t work, int threads);
}

namespace {

struct FiveGhostParams {
    double* u;
    StepCtl* ctl;
    int64_t ncell;
    int64_t m[3];
    int64_t stride[3];
    int64_t n, ng;
    int d, e0, e1;
    int kind[2];
    double state[2][NF];
    FiveSysD sys;
};

// Ghost layers along d for every (a, b) of the other padded axes
// (solver.rs:278-348, boundary.rs:34-96); reflecting axes have n >= ng.
__global__ void five_ghost_kernel(const FiveGhostParams p) {
    if (p.ctl->done) return;
    const Five s = Five::from(p.sys);
    const int64_t total = p.m[p.e0] * p.m[p.e1] * p.ng;
    const int64_t n = p.n, ng = p.ng;
    const int mom = F_IU + p.d;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t gi = t % ng;
        const int64_t pq = t / ng;
        const int64_t b = pq % p.m[p.e1];
        const int64_t a = pq / p.m[p.e1];
        const int64_t off = a * p.stride[p.e0] + b * p.stride[p.e1];
        const int64_t sd = p.stride[p.d];
        auto at = [&](int64_t c) { return off + c * sd; };
        auto load = [&](int64_t c, double* v) {
            if (!in_bounds(p.ctl, at(c), p.ncell)) {
                for (int k = 0; k < NF; k++) v[k] = 0.0;
                return;
            }
            for (int k = 0; k < NF; k++) v[k] = p.u[k * p.ncell + at(c)];
        };
        int64_t lo_s, hi_s;  // periodic sources (solver.rs:62-70)
        if (n >= ng) {
            lo_s = n + gi;
            hi_s = ng + gi;
        } else {
            lo_s = ng + (gi + n - ng % n) % n;
            hi_s = ng + gi % n;
        }
        double v[NF];
        for (int side = 0; side < 2; side++) {
            const int kind = p.kind[side];
            if (kind == EMG_BC_PERIODIC) {
                load(side == 0 ? lo_s : hi_s, v);
            } else if (kind == EMG_BC_OUTFLOW) {
                load(side == 0 ? ng : n + ng - 1, v);
            } else if (kind == EMG_BC_DIRICHLET) {
                for (int k = 0; k < NF; k++) v[k] = p.state[side][k];
            } else if (kind == EMG_BC_CHARACTERISTIC) {
                double ub[NF], ub1[NF];
                load(side == 0 ? ng : n + ng - 1, ub);
                load(side == 0 ? ng + 1 : n + ng - 2, ub1);
                CharStencil7D ch;
                ch.init(s, ub, ub1, p.state[side], p.d, side);
                ch.conserved(s, side == 0 ? (double)(ng - gi) : (double)(gi + 1), v);
            } else {
                load(side == 0 ? 2 * ng - 1 - gi : n + ng - 1 - gi, v);
                v[mom] = -v[mom];
            }
            const int64_t dst = side == 0 ? at(gi) : at(n + ng + gi);
            if (in_bounds(p.ctl, dst, p.ncell))
                for (int k = 0; k < NF; k++) p.u[k * p.ncell + dst] = v[k];
        }
    }
}

struct FiveCflParams {
    const double* u;
    StepCtl* ctl;
    int64_t ncell;
    int64_t n[3], g[3], stride[3];
    int act[3];
    double dx[3];
    int kind[3][2];
    double state[3][2][NF];
    FiveSysD sys;
    unsigned long long* source_bits;
};

// CFL rate Σ_d (|u_d| + c)/dx_d and dilatation rate of every interior cell
// (solver.rs:478-523; neighbour states as solver.rs:565-640)
__global__ void five_cfl_kernel(const FiveCflParams p) {
    const Five s = Five::from(p.sys);
    const int64_t cells = p.n[0] * p.n[1] * p.n[2];
    double rate = 0.0, source = 0.0;
    int bad = 0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < cells; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c[3] = {t / (p.n[1] * p.n[2]) + p.g[0], (t / p.n[2]) % p.n[1] + p.g[1], t % p.n[2] + p.g[2]};
        const int64_t q = c[0] * p.stride[0] + c[1] * p.stride[1] + c[2] * p.stride[2];
        double uc[NF], w[NF], d0, b0;
        for (int k = 0; k < NF; k++) uc[k] = p.u[k * p.ncell + q];
        s.to_prim_db(uc, w, d0, b0);
        const double rc2 = s.rho_c2_db(w, d0, b0, s.kapila_k(w));  // once for the sound speed and the dilatation
        // a failed state: a non-finite value or a non-positive density (the
        // model's full admissibility, with its α range and ρc² > 0, is only
        // what the limiter keeps the one-sided updates in: the reference
        // steps on through interior states slightly outside it)
        for (int k = 0; k < NF; k++)
            if (!isfinite(w[k])) bad = 1;
        if (!(Five::rho(w) > 0.0)) bad = 1;
        const double cs = Five::sound_speed_rc2(w, rc2);
        double acc = -0.0;
        for (int d = 0; d < 3; d++)
            if (p.act[d]) acc = acc + (fabs(w[F_IU + d]) + cs) / p.dx[d];
        rate = fmax(rate, acc);
        double divu = 0.0;
        for (int d = 0; d < 3; d++) {
            if (!p.act[d]) continue;
            double vv[2];
            for (int hi = 0; hi < 2; hi++) {
                const bool boundary = hi ? c[d] == p.g[d] + p.n[d] - 1 : c[d] == p.g[d];
                double nb[NF];
                if (!boundary) {
                    const int64_t qn = q + (hi ? p.stride[d] : -p.stride[d]);
                    for (int k = 0; k < NF; k++) nb[k] = p.u[k * p.ncell + qn];
                } else {
                    const int kind = p.kind[d][hi];
                    if (kind == EMG_BC_PERIODIC) {
                        const int64_t qn = q + (hi ? -(p.n[d] - 1) : (p.n[d] - 1)) * p.stride[d];
                        for (int k = 0; k < NF; k++) nb[k] = p.u[k * p.ncell + qn];
                    } else if (kind == EMG_BC_OUTFLOW) {
                        for (int k = 0; k < NF; k++) nb[k] = uc[k];
                    } else if (kind == EMG_BC_DIRICHLET) {
                        for (int k = 0; k < NF; k++) nb[k] = p.state[d][hi][k];
                    } else if (kind == EMG_BC_REFLECT) {
                        for (int k = 0; k < NF; k++) nb[k] = uc[k];
                        nb[F_IU + d] = nb[F_IU + d] * -1.0;
                    } else {
                        const int64_t qi = q + (hi ? -p.stride[d] : p.stride[d]);
                        double u1[NF];
                        for (int k = 0; k < NF; k++) u1[k] = p.u[k * p.ncell + qi];
                        CharStencil7D ch;
                        ch.init(s, uc, u1, p.state[d][hi], d, hi);
                        ch.conserved(s, 1.0, nb);
                    }
                }
                vv[hi] = Five::velocity_conserved(nb, d);
            }
            divu = divu + fabs(vv[1] - vv[0]) / (2.0 * p.dx[d]);
        }
        source = fmax(source, s.dilatation_rate_rc2(w, divu, rc2));
    }
    for (int o = 16; o > 0; o >>= 1) {
        rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, o));
        source = fmax(source, __shfl_xor_sync(0xffffffffu, source, o));
    }
    __shared__ double sr[32], ss[32];
    if ((threadIdx.x & 31) == 0) {
        sr[threadIdx.x >> 5] = rate;
        ss[threadIdx.x >> 5] = source;
    }
    const int any_bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        double v = sr[0], w2 = ss[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            v = fmax(v, sr[k]);
            w2 = fmax(w2, ss[k]);
        }
        if (!isnan(v) && v > 0.0) atomicMax(&p.ctl->rate_bits, (unsigned long long)__double_as_longlong(v));
        if (!isnan(w2) && w2 > 0.0) atomicMax(p.source_bits, (unsigned long long)__double_as_longlong(w2));
        if (any_bad) atomicCAS(&p.ctl->status, 0, (int)EMG_ERR_INADMISSIBLE);
    }
}

__global__ void five_aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, int64_t ncell) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < NF; k++) soa[k * ncell + c] = aos[NF * c + k];
}
__global__ void five_soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int64_t ncell) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x)
        for (int k = 0; k < NF; k++) aos[NF * c + k] = soa[k * ncell + c];
}

__global__ void five_ctl_begin(StepCtl* ctl, double dt, unsigned long long* source_bits) {
    ctl->dt = dt;
    ctl->done = 0;
    ctl->status = 0;
    ctl->rate_bits = 0ull;
    *source_bits = 0ull;
}

// Σ u·vol over interior cells (solver.rs:784-794), deterministic: per-block
// partials, then one thread per field adds them in order
__global__ void five_totals_partial(const double* __restrict__ u, int64_t ncell, CellRange cr, double vol, double* partial) {
    double s[NF];
    for (int k = 0; k < NF; k++) s[k] = 0.0;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < cr.cells; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = cr.index(t);
        for (int k = 0; k < NF; k++) s[k] = s[k] + u[k * ncell + c] * vol;
    }
    __shared__ double sh[NF][256];
    for (int k = 0; k < NF; k++) sh[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h)
            for (int k = 0; k < NF; k++) sh[k][threadIdx.x] = sh[k][threadIdx.x] + sh[k][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < NF; k++) partial[k * gridDim.x + blockIdx.x] = sh[k][0];
}
__global__ void five_totals_final(const double* partial, int nb, double* out) {
    if (threadIdx.x < NF) {
        double s = 0.0;
        for (int b = 0; b < nb; b++) s = s + partial[threadIdx.x * nb + b];
        out[threadIdx.x] = s;
    }
}

template <int P, int D, int MODE>
__global__ void __launch_bounds__(SWEEP_THREADS, 2) five_sweep_kernel(const FiveSweepParams p) {
    FiveSweep<P, D, MODE>::run(p);
}

template <int P, int MODE> cudaError_t five_launch_d(const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    const size_t b = FiveSmem<P, MODE>::bytes();
    if (p.d == 0)
        five_sweep_kernel<P, 0, MODE><<<grid, SWEEP_THREADS, b, s>>>(p);
    else if (p.d == 1)
        five_sweep_kernel<P, 1, MODE><<<grid, SWEEP_THREADS, b, s>>>(p);
    else
        five_sweep_kernel<P, 2, MODE><<<grid, SWEEP_THREADS, b, s>>>(p);
    return cudaGetLastError();
}
template <int MODE> cudaError_t five_launch_p(int P, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    switch (P) {
        case 8: return five_launch_d<8, MODE>(p, grid, s);
        case 16: return five_launch_d<16, MODE>(p, grid, s);
        case 32: return five_launch_d<32, MODE>(p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}
cudaError_t five_launch(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    switch (mode) {
        case MODE_WENO: return five_launch_p<MODE_WENO>(P, p, grid, s);
        case MODE_HYBRID: return five_launch_p<MODE_HYBRID>(P, p, grid, s);
        case MODE_CENTRAL: return five_launch_p<MODE_CENTRAL>(P, p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}
template <int P, int MODE> cudaError_t five_attr_d() {
    const int b = (int)FiveSmem<P, MODE>::bytes();
    cudaError_t e = cudaFuncSetAttribute(five_sweep_kernel<P, 0, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(five_sweep_kernel<P, 1, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(five_sweep_kernel<P, 2, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    return e;
}
// batched block-AMR leaves: one CTA per (leaf, group of block rows), P = 16 or 32
template <int P, int D, int MODE>
__global__ void __launch_bounds__(SWEEP_THREADS, 2) five_sweep_amr_kernel(const FiveSweepParams p) {
    FiveSweep<P, D, MODE, true>::run(p);
}
template <int P, int MODE> cudaError_t five_launch_amr_d(const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    const size_t b = FiveSmem<P, MODE>::bytes();
    if (p.d == 0)
        five_sweep_amr_kernel<P, 0, MODE><<<grid, SWEEP_THREADS, b, s>>>(p);
    else if (p.d == 1)
        five_sweep_amr_kernel<P, 1, MODE><<<grid, SWEEP_THREADS, b, s>>>(p);
    else
        five_sweep_amr_kernel<P, 2, MODE><<<grid, SWEEP_THREADS, b, s>>>(p);
    return cudaGetLastError();
}
template <int MODE> cudaError_t five_launch_amr_p(int P, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    switch (P) {
        case 16: return five_launch_amr_d<16, MODE>(p, grid, s);
        case 32: return five_launch_amr_d<32, MODE>(p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}
cudaError_t five_launch_amr(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    switch (mode) {
        case MODE_WENO: return five_launch_amr_p<MODE_WENO>(P, p, grid, s);
        case MODE_HYBRID: return five_launch_amr_p<MODE_HYBRID>(P, p, grid, s);
        case MODE_CENTRAL: return five_launch_amr_p<MODE_CENTRAL>(P, p, grid, s);
        default: return cudaErrorInvalidValue;
    }
}
template <int P, int MODE> cudaError_t five_attr_amr_d() {
    const int b = (int)FiveSmem<P, MODE>::bytes();
    cudaError_t e = cudaFuncSetAttribute(five_sweep_amr_kernel<P, 0, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(five_sweep_amr_kernel<P, 1, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(five_sweep_amr_kernel<P, 2, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    return e;
}
template <int MODE> cudaError_t five_attr_p() {
    cudaError_t e = five_attr_d<8, MODE>();
    if (e == cudaSuccess) e = five_attr_d<16, MODE>();
    if (e == cudaSuccess) e = five_attr_d<32, MODE>();
    if (e == cudaSuccess) e = five_attr_amr_d<16, MODE>();
    if (e == cudaSuccess) e = five_attr_amr_d<32, MODE>();
    return e;
}
// the sweeps' shared-memory opt-in, once per device
cudaError_t five_prepare_device() {
    static std::mutex mu;
    static bool done[64] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
    e = five_attr_p<MODE_WENO>();
    if (e == cudaSuccess) e = five_attr_p<MODE_HYBRID>();
    if (e == cudaSuccess) e = five_attr_p<MODE_CENTRAL>();
    if (e == cudaSuccess) e = five_sweep_prepare_fast();
    if (e == cudaSuccess && dev >= 0 && dev < 64) done[dev] = true;
    return e;
}

}  // namespace

namespace emg {
cudaError_t five_sweep_launch_amr(int P, int mode, const FiveSweepParams& p, dim3 grid, cudaStream_t s) {
    return five_launch_amr(P, mode, p, grid, s);
}
cudaError_t five_sweep_prepare_device() { return five_prepare_device(); }
}  // namespace emg

struct emg_five {
    int device = 0;
    cudaStream_t stream = nullptr;
    emg_mesh mesh{};
    FiveSysD sys{};
    emg_bc7 bc[6]{};
    emg_opts opts{};
    int64_t m[3]{}, stride[3]{}, ncell = 0, cells = 0;
    int active[3]{};
    int ndim = 0;
    double *u = nullptr, *sa = nullptr, *sb = nullptr, *rhs = nullptr, *staging = nullptr, *partial = nullptr;
    StepCtl* ctl = nullptr;
    StepCtl* ctl_host = nullptr;
    unsigned long long* source_bits = nullptr;
    int sweepP[3]{}, sweepSeg[3]{};
    dim3 sweepGrid[3];
    int lane_axis[3]{}, other_axis[3]{};
    double t = 0.0;
    uint64_t faces = 0, weno_faces = 0, launches = 0;
    bool rate_valid = false;
    double rate = 0.0, source = 0.0;

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        for (double* b : {u, sa, sb, rhs, staging, partial}) cudaFree(b);
        cudaFree(ctl);
        cudaFree(source_bits);
        if (ctl_host) cudaFreeHost(ctl_host);
        if (stream) cudaStreamDestroy(stream);
        u = sa = sb = rhs = staging = partial = nullptr;
        ctl = nullptr;
        source_bits = nullptr;
        ctl_host = nullptr;
        stream = nullptr;
    }

    // launch shape per axis: P pencils per CTA along the lane axis, segments
    // shortened (halving) until the grid covers the SMs once
    void plan() {
        int dev = 0, sms = 148;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            sms = 148;
        }
        for (int d = 0; d < 3; d++) {
            if (!active[d]) continue;
            int o[2], no = 0;
            for (int e = 0; e < 3; e++)
                if (e != d) o[no++] = e;
            int lane = o[1], other = o[0];
            if (!active[o[1]] && active[o[0]]) {
                lane = o[0];
                other = o[1];
            }
            lane_axis[d] = lane;
            other_axis[d] = other;
            const int64_t nd = mesh.n[d], nl = mesh.n[lane], nother = mesh.n[other];
            int P = opts.mode == EMG_MODE_HYBRID ? 16 : 32;
            if (nl <= 8)
                P = 8;
            else if (nl <= 16)
                P = 16;
            const int64_t tiles = (nl + P - 1) / P;
            int64_t seg = nd;
            while (seg > 32 && tiles * ((nd + seg - 1) / seg) * nother < sms) seg = (seg + 1) / 2;
            sweepP[d] = P;
            sweepSeg[d] = (int)seg;
            sweepGrid[d] = dim3((unsigned)tiles, (unsigned)((nd + seg - 1) / seg), (unsigned)nother);
        }
    }

    int ghosts(double* arr) {
        for (int d = 0; d < 3; d++) {
            if (!active[d]) continue;
            FiveGhostParams p{};
            p.u = arr;
            p.ctl = ctl;
            p.ncell = ncell;
            for (int k = 0; k < 3; k++) {
                p.m[k] = m[k];
                p.stride[k] = stride[k];
            }
            p.n = mesh.n[d];
            p.ng = mesh.ng;
            p.d = d;
            p.e0 = d == 0 ? 1 : 0;
            p.e1 = d == 2 ? 1 : 2;
            for (int s = 0; s < 2; s++) {
                p.kind[s] = bc[2 * d + s].kind;
                for (int k = 0; k < NF; k++) p.state[s][k] = bc[2 * d + s].state[k];
            }
            p.sys = sys;
            const int64_t work = m[p.e0] * m[p.e1] * p.ng;
            five_ghost_kernel<<<kernel_grid(work, 256), 256, 0, stream>>>(p);
            launches++;
            EMG_CUDA(cudaGetLastError());
        }
        return EMG_OK;
    }

    int stage(int s) {
        double* in = s == 1 ? u : (s == 2 ? sa : sb);
        int rc = ghosts(in);
        if (rc) return rc;
        int first_axis = -1, last_axis = -1;
        for (int d = 0; d < 3; d++)
            if (active[d]) {
                if (first_axis < 0) first_axis = d;
                last_axis = d;
            }
        for (int d = 0; d < 3; d++) {
            if (!active[d]) continue;
            FiveSweepParams p{};
            p.uin = in;
            p.rhs = rhs;
            p.ctl = ctl;
            p.ncell = ncell;
            const int l = lane_axis[d], o = other_axis[d];
            p.sd = stride[d];
            p.sl = stride[l];
            p.so = stride[o];
            p.nd = (int)mesh.n[d];
            p.nl = (int)mesh.n[l];
            p.no = (int)mesh.n[o];
            p.gd = active[d] ? (int)mesh.ng : 0;
            p.gl = active[l] ? (int)mesh.ng : 0;
            p.go = active[o] ? (int)mesh.ng : 0;
            p.d = d;
            p.seg = sweepSeg[d];
            p.first = d == first_axis;
            p.last = d == last_axis;
            p.stage = s;
            p.rows_contig = p.sd == 1;
            p.dx = mesh.dx[d];
            p.ndim = (double)ndim;
            p.positivity = opts.positivity ? 1 : 0;
            p.tol = opts.tol;
            p.sys = sys;
            if (p.last) {
                if (s == 1) {
                    p.base = u;
                    p.dest = sa;
                } else if (s == 2) {
                    p.base = u;
                    p.cur = sa;
                    p.dest = sb;
                } else {
                    p.base = sb;
                    p.cur = u;
                    p.dest = u;
                }
            }
            cudaError_t e = opts.precision == EMG_PRECISION_F64_FAST
                                ? five_sweep_launch_fast(sweepP[d], opts.mode, p, sweepGrid[d], stream)
                                : five_launch(sweepP[d], opts.mode, p, sweepGrid[d], stream);
            launches++;
            if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("five-equation sweep: ") + cudaGetErrorString(e));
        }
        return EMG_OK;
    }

    int sync() {
        EMG_CUDA(cudaMemcpyAsync(ctl_host, ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, stream));
        EMG_CUDA(cudaStreamSynchronize(stream));
        return EMG_OK;
    }

    int status() const {
        const int st = ctl_host->status;
        if (st == EMG_ERR_INADMISSIBLE)
            return set_error(st, "non-finite state or non-positive density in an interior cell");
        if (st == EMG_ERR_BOUNDS) return set_error(st, "device index out of range (bounds-check build)");
        if (st) return set_error(st, "device error");
        return EMG_OK;
    }

    int step(double dt) {
        five_ctl_begin<<<1, 1, 0, stream>>>(ctl, dt, source_bits);
        launches++;
        EMG_CUDA(cudaGetLastError());
        for (int s = 1; s <= 3; s++) {
            int rc = stage(s);
            if (rc) return rc;
        }
        uint64_t f = 0;
        for (int d = 0; d < 3; d++)
            if (active[d]) f += (uint64_t)(cells / mesh.n[d]) * (uint64_t)(mesh.n[d] + 1);
        faces += 3 * f;
        if (opts.mode == EMG_MODE_WENO) weno_faces += 3 * f;
        t += dt;
        rate_valid = false;
        int rc = sync();
        return rc ? rc : status();
    }

    int dt_cfl(double* dt) {
        if (!rate_valid) {
            five_ctl_begin<<<1, 1, 0, stream>>>(ctl, 0.0, source_bits);
            FiveCflParams p{};
            p.u = u;
            p.ctl = ctl;
            p.ncell = ncell;
            for (int d = 0; d < 3; d++) {
                p.n[d] = mesh.n[d];
                p.g[d] = active[d] ? mesh.ng : 0;
                p.stride[d] = stride[d];
                p.act[d] = active[d];
                p.dx[d] = mesh.dx[d];
                for (int s = 0; s < 2; s++) {
                    p.kind[d][s] = bc[2 * d + s].kind;
                    for (int k = 0; k < NF; k++) p.state[d][s][k] = bc[2 * d + s].state[k];
                }
            }
            p.sys = sys;
            p.source_bits = source_bits;
            five_cfl_kernel<<<kernel_grid(cells, 256), 256, 0, stream>>>(p);
            launches += 2;
            EMG_CUDA(cudaGetLastError());
            unsigned long long sb_host = 0;
            EMG_CUDA(cudaMemcpyAsync(&sb_host, source_bits, sizeof sb_host, cudaMemcpyDeviceToHost, stream));
            int rc = sync();
            if (rc) return rc;
            if ((rc = status())) return rc;
            std::memcpy(&rate, &ctl_host->rate_bits, sizeof rate);
            std::memcpy(&source, &sb_host, sizeof source);
            rate_valid = true;
        }
        double d = opts.cfl / rate;
        if (source > 0.0) d = std::fmin(d, 0.5 / source);
        *dt = d;
        return EMG_OK;
    }
};

extern "C" {

int emg_five_create(const emg_mesh* mesh, const emg_five_system* sys, const emg_bc7 bc[6], const emg_opts* opts,
                    const double* u_aos, size_t len, emg_five** out) {
    if (!mesh || !sys || !bc || !opts || !u_aos || !out) return set_error(EMG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (mesh->ng < 5) return set_error(EMG_ERR_INVALID, "the WCNS stencil needs ng >= 5 ghost layers");
    int ndim = 0;
    size_t padded = 1;
    for (int d = 0; d < 3; d++) {
        if (mesh->n[d] < 1) return set_error(EMG_ERR_INVALID, "mesh extents must be >= 1");
        if (mesh->n[d] > 1) {
            ndim++;
            if (!(mesh->dx[d] > 0.0)) return set_error(EMG_ERR_INVALID, "dx must be > 0 on active axes");
            if (mesh->n[d] > (1 << 30)) return set_error(EMG_ERR_INVALID, "axis too long");
            padded *= (size_t)(mesh->n[d] + 2 * mesh->ng);
        }
    }
    if (ndim == 0) return set_error(EMG_ERR_INVALID, "mesh has no active axis");
    if (padded != len) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    if (opts->mode != EMG_MODE_WENO && opts->mode != EMG_MODE_HYBRID && opts->mode != EMG_MODE_CENTRAL)
        return set_error(EMG_ERR_INVALID, "unknown flux mode");
    if (opts->mode == EMG_MODE_HYBRID && !(opts->tol > 0.0)) return set_error(EMG_ERR_INVALID, "hybrid mode needs tol > 0");
    if (opts->precision != EMG_PRECISION_F64 && opts->precision != EMG_PRECISION_F64_FAST)
        return set_error(EMG_ERR_INVALID, "the five-equation system runs in the plain or fast FP64 form");
    for (int k = 0; k < 2; k++)
        if (!(sys->eos[k].gamma > 1.0)) return set_error(EMG_ERR_INVALID, "each phase needs gamma > 1");
    for (int d = 0; d < 3; d++) {
        for (int s = 0; s < 2; s++)
            if (bc[2 * d + s].kind < 0 || bc[2 * d + s].kind > 4) return set_error(EMG_ERR_INVALID, "unknown boundary condition");
        if (mesh->n[d] > 1) {
            const bool p0 = bc[2 * d].kind == EMG_BC_PERIODIC, p1 = bc[2 * d + 1].kind == EMG_BC_PERIODIC;
            if (p0 != p1) return set_error(EMG_ERR_INVALID, "periodic boundaries must be paired");
            if (mesh->n[d] < mesh->ng && (bc[2 * d].kind == EMG_BC_REFLECT || bc[2 * d + 1].kind == EMG_BC_REFLECT))
                return set_error(EMG_ERR_INVALID, "reflecting axes of the five-equation path need n >= ng cells");
        }
    }
    int dev = 0;
    {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            return set_error(EMG_ERR_NO_DEVICE, "no CUDA device visible");
        }
        EMG_CUDA(cudaGetDevice(&dev));
        cudaDeviceProp pr;
        EMG_CUDA(cudaGetDeviceProperties(&pr, dev));
        if (pr.major != 10) return set_error(EMG_ERR_NO_DEVICE, "device is not sm_100 (B200)");
    }
    emg_five* h = new emg_five();
    h->device = dev;
    h->mesh = *mesh;
    for (int k = 0; k < 2; k++) h->sys.e[k] = EosD{sys->eos[k].gamma, sys->eos[k].p_inf, sys->eos[k].b, sys->eos[k].q};
    h->sys.kapila = sys->kapila ? 1 : 0;
    for (int i = 0; i < 6; i++) h->bc[i] = bc[i];
    h->opts = *opts;
    h->ndim = ndim;
    for (int d = 0; d < 3; d++) {
        h->active[d] = mesh->n[d] > 1;
        h->m[d] = h->active[d] ? mesh->n[d] + 2 * mesh->ng : 1;
    }
    h->stride[2] = 1;
    h->stride[1] = h->m[2];
    h->stride[0] = h->m[1] * h->m[2];
    h->ncell = h->m[0] * h->m[1] * h->m[2];
    h->cells = mesh->n[0] * mesh->n[1] * mesh->n[2];
    auto bail = [&](int rc) {
        h->release();
        delete h;
        return rc;
    };
    {
        cudaError_t e = five_prepare_device();
        if (e != cudaSuccess) return bail(set_error(EMG_ERR_CUDA, std::string("sweep setup: ") + cudaGetErrorString(e)));
    }
    const size_t bytes = (size_t)h->ncell * NF * sizeof(double);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess || cudaMalloc(&h->u, bytes) != cudaSuccess ||
        cudaMalloc(&h->sa, bytes) != cudaSuccess || cudaMalloc(&h->sb, bytes) != cudaSuccess ||
        cudaMalloc(&h->rhs, bytes) != cudaSuccess || cudaMalloc(&h->staging, bytes) != cudaSuccess ||
        cudaMalloc(&h->partial, NF * 4096 * sizeof(double) + NF * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->ctl, sizeof(StepCtl)) != cudaSuccess ||
        cudaMalloc(&h->source_bits, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMallocHost(&h->ctl_host, sizeof(StepCtl)) != cudaSuccess) {
        cudaGetLastError();
        return bail(set_error(EMG_ERR_CUDA, "device allocation failed"));
    }
    cudaMemsetAsync(h->sa, 0, bytes, h->stream);
    cudaMemsetAsync(h->sb, 0, bytes, h->stream);
    cudaMemsetAsync(h->rhs, 0, bytes, h->stream);
    std::memset(h->ctl_host, 0, sizeof(StepCtl));
    h->ctl_host->t_end = INFINITY;
    if (cudaMemcpyAsync(h->ctl, h->ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(h->staging, u_aos, bytes, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return bail(set_error(EMG_ERR_CUDA, "upload failed"));
    five_aos_to_soa<<<kernel_grid(h->ncell, 256), 256, 0, h->stream>>>(h->staging, h->u, h->ncell);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess)
        return bail(set_error(EMG_ERR_CUDA, "upload failed"));
    h->plan();
    for (int d = 0; d < 3; d++)
        if (h->active[d] && (h->sweepGrid[d].y > 65535u || h->sweepGrid[d].z > 65535u))
            return bail(set_error(EMG_ERR_INVALID, "mesh too large for the sweep grid"));
    *out = h;
    return EMG_OK;
}

int emg_five_destroy(emg_five* h) {
    if (!h) return EMG_OK;
    cudaSetDevice(h->device);
    h->release();
    delete h;
    return EMG_OK;
}

static int five_check(emg_five* h) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    if (cudaSetDevice(h->device) != cudaSuccess) return set_error(EMG_ERR_CUDA, "cudaSetDevice failed");
    return EMG_OK;
}

int emg_five_step(emg_five* h, double dt) {
    int rc = five_check(h);
    if (rc) return rc;
    if (!(std::isfinite(dt) && dt > 0.0)) return set_error(EMG_ERR_INVALID, "dt must be finite and > 0");
    return h->step(dt);
}

int emg_five_dt_cfl(emg_five* h, double* dt) {
    int rc = five_check(h);
    if (rc) return rc;
    if (!dt) return set_error(EMG_ERR_INVALID, "null dt");
    return h->dt_cfl(dt);
}

int emg_five_run_to(emg_five* h, double t_end, uint64_t* steps) {
    int rc = five_check(h);
    if (rc) return rc;
    if (!std::isfinite(t_end)) return set_error(EMG_ERR_INVALID, "t_end must be finite");
    uint64_t n = 0;
    while (h->t < t_end - 1e-10 * std::fabs(t_end)) {
        double dt = 0.0;
        if ((rc = h->dt_cfl(&dt))) return rc;
        dt = std::fmin(dt, t_end - h->t);
        if (!(std::isfinite(dt) && dt > 1e-12 * std::fmax(std::fabs(t_end), 1e-300)))
            return set_error(EMG_ERR_DT_COLLAPSED, "time step collapsed");
        if ((rc = h->step(dt))) return rc;
        n++;
    }
    if (steps) *steps = n;
    return EMG_OK;
}

int emg_five_download(emg_five* h, double* u_aos, size_t len) {
    int rc = five_check(h);
    if (rc) return rc;
    if (!u_aos || len != (size_t)h->ncell) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    five_soa_to_aos<<<kernel_grid(h->ncell, 256), 256, 0, h->stream>>>(h->u, h->staging, h->ncell);
    EMG_CUDA(cudaGetLastError());
    EMG_CUDA(cudaMemcpyAsync(u_aos, h->staging, (size_t)h->ncell * NF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_five_counters(emg_five* h, uint64_t out[4]) {
    int rc = five_check(h);
    if (rc) return rc;
    if (!out) return set_error(EMG_ERR_INVALID, "null out");
    if ((rc = h->sync())) return rc;
    out[0] = h->faces;
    out[1] = h->opts.mode == EMG_MODE_WENO ? h->weno_faces : h->ctl_host->counters[1];
    out[2] = h->ctl_host->counters[2];
    out[3] = h->ctl_host->counters[3];
    return EMG_OK;
}

int emg_five_totals(emg_five* h, double out[7]) {
    int rc = five_check(h);
    if (rc) return rc;
    if (!out) return set_error(EMG_ERR_INVALID, "null out");
    CellRange cr{};
    double vol = 1.0;
    for (int d = 0; d < 3; d++) {
        cr.n[d] = h->mesh.n[d];
        cr.g[d] = h->active[d] ? h->mesh.ng : 0;
        cr.stride[d] = h->stride[d];
        if (h->active[d]) vol = vol * h->mesh.dx[d];
    }
    cr.cells = h->cells;
    const int nb = (int)std::min<int64_t>(4096, std::max<int64_t>(1, (h->cells + 255) / 256));
    five_totals_partial<<<nb, 256, 0, h->stream>>>(h->u, h->ncell, cr, vol, h->partial);
    five_totals_final<<<1, 32, 0, h->stream>>>(h->partial, nb, h->partial + NF * 4096);
    EMG_CUDA(cudaGetLastError());
    EMG_CUDA(cudaMemcpyAsync(out, h->partial + NF * 4096, NF * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_five_get_time(emg_five* h, double* t) {
    if (!h || !t) return set_error(EMG_ERR_INVALID, "null argument");
    *t = h->t;
    return EMG_OK;
}

int emg_five_stream(emg_five* h, void** stream) {
    if (!h || !stream) return set_error(EMG_ERR_INVALID, "null argument");
    *stream = (void*)h->stream;
    return EMG_OK;
}

int emg_five_launch_count(emg_five* h, uint64_t* launches) {
    if (!h || !launches) return set_error(EMG_ERR_INVALID, "null argument");
    *launches = h->launches;
    return EMG_OK;
}

}  // extern "C"
