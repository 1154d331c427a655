// Uniform-grid solver: host object, auxiliary kernels and the C ABI of
// include/emergence_b200.h (emg_uniform_*).
//
// Replaces compressible-cuda's GpuSolver (fluid/crates/compressible-cuda/src/
// lib.rs:155-477) for the Euler system. Per RK stage the device runs one
// ghost-fill launch per active axis and one fused sweep per active axis
// (sweep.cuh); the reference runs ghost + prim + 4 launches per axis + rk
// (G/lib.rs:332-400). The CFL rate of each new state is reduced inside the
// last sweep of stage 3 and dt is formed on the device, so steps chain
// without host round trips (the reference copies the rates to the host every
// step, G/lib.rs:430).
//
// Built with -fmad=false: the ghost, CFL and control arithmetic must round as
// the reference CPU solver does.
#include "uniform_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <mutex>
#include <string>
#include <vector>

namespace emg {

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

// ------------------------------------------------------------------ auxiliary kernels

// AoS [cell][5] → SoA [5][cell]
__global__ void aos_to_soa(const double* __restrict__ aos, double* __restrict__ soa, int64_t ncell) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 5; k++) soa[k * ncell + c] = aos[5 * c + k];
    }
}
__global__ void soa_to_aos(const double* __restrict__ soa, double* __restrict__ aos, int64_t ncell) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 5; k++) aos[5 * c + k] = soa[k * ncell + c];
    }
}

struct GhostParams {
    double* u;
    StepCtl* ctl;
    int64_t ncell;
    int64_t m[3];
    int64_t stride[3];
    int64_t n, ng;
    int d, e0, e1;
    int deep;  // a short reflecting axis exists (C/solver.rs:261-262)
    int kind[2];
    double state[2][5];
    EosD eos;
};

// Characteristic ghost stencil (C/boundary.rs:48-96), dense as the reference.
struct CharStencilD {
    double wi[5], wf[5], w1[5];
    double l[5][5], r[5][5];
    bool outgoing[5];
    __device__ void init(const Eos<double>& e, const double* ub, const double* ub1, const double* uf, int d, int side) {
        to_prim(e, ub, wi);
        to_prim(e, uf, wf);
        to_prim(e, ub1, w1);
        const double rho = wi[0], c = sound_speed(e, wi[0], wi[4]);
        const int un = 1 + d, t1 = 1 + (d + 1) % 3, t2 = 1 + (d + 2) % 3;
        for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) l[i][j] = r[i][j] = 0.0;
        l[0][un] = -rho / (2.0 * c);
        l[0][4] = 1.0 / (2.0 * c * c);
        l[1][0] = 1.0;
        l[1][4] = -1.0 / (c * c);
        l[2][t1] = 1.0;
        l[3][t2] = 1.0;
        l[4][un] = rho / (2.0 * c);
        l[4][4] = 1.0 / (2.0 * c * c);
        r[0][0] = 1.0;
        r[un][0] = -c / rho;
        r[4][0] = c * c;
        r[0][1] = 1.0;
        r[t1][2] = 1.0;
        r[t2][3] = 1.0;
        r[0][4] = 1.0;
        r[un][4] = c / rho;
        r[4][4] = c * c;
        const double u = wi[un];
        const double lam[5] = {u - c, u, u, u, u + c};
        const double outward = side == 1 ? 1.0 : -1.0;
        for (int k = 0; k < 5; k++) outgoing[k] = lam[k] * outward > 0.0;
    }
    __device__ void conserved(const Eos<double>& e, double m, double* out) const {
        double dw[5], wg[5];
        for (int k = 0; k < 5; k++) dw[k] = wi[k] - wf[k] + m * (wi[k] - w1[k]);
        for (int k = 0; k < 5; k++) wg[k] = wf[k];
        for (int kf = 0; kf < 5; kf++) {
            if (outgoing[kf]) {
                double amp = -0.0;
                for (int q = 0; q < 5; q++) amp = amp + l[kf][q] * dw[q];
                for (int q = 0; q < 5; q++) wg[q] = wg[q] + r[q][kf] * amp;
            }
        }
        to_cons(e, wg, out);
    }
};

// Ghost layers along axis d for every (a, b) of the two other padded axes
// (C/solver.rs:278-348; G/kernels.cu:567-614). Only interior cells along d
// are read, so threads are independent.
__global__ void ghost_kernel(const GhostParams p) {
    if (p.ctl->done) return;
    const Eos<double> e = Eos<double>::from(p.eos);
    const int64_t total = p.m[p.e0] * p.m[p.e1] * p.ng;
    const int64_t n = p.n, ng = p.ng;
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
                for (int k = 0; k < 5; k++) v[k] = 0.0;
                return;
            }
            for (int k = 0; k < 5; k++) v[k] = p.u[k * p.ncell + at(c)];
        };
        CharStencilD ch[2];
        if (p.kind[0] == EMG_BC_CHARACTERISTIC) {
            double ub[5], ub1[5];
            load(ng, ub);
            load(ng + 1, ub1);
            ch[0].init(e, ub, ub1, p.state[0], p.d, 0);
        }
        if (p.kind[1] == EMG_BC_CHARACTERISTIC) {
            double ub[5], ub1[5];
            load(n + ng - 1, ub);
            load(n + ng - 2, ub1);
            ch[1].init(e, ub, ub1, p.state[1], p.d, 1);
        }
        // deep reflected image on a short axis (C/boundary.rs:98-145)
        auto reflected = [&](int64_t x, double* v) {
            bool flip = false;
            for (int k = 0; k < 5; k++) v[k] = __longlong_as_double(0x7ff8000000000000ll);
            for (int it = 0; it < 4096; it++) {
                if (x >= 0 && x < n) {
                    load(ng + x, v);
                    break;
                }
                const int side = x >= n ? 1 : 0;
                const int kind = p.kind[side];
                if (kind == EMG_BC_REFLECT) {
                    x = side == 0 ? -1 - x : 2 * n - 1 - x;
                    flip = !flip;
                } else if (kind == EMG_BC_PERIODIC) {
                    int64_t r = x % n;
                    if (r < 0) r += n;
                    load(ng + r, v);
                    break;
                } else if (kind == EMG_BC_OUTFLOW) {
                    load(ng + (side == 0 ? 0 : n - 1), v);
                    break;
                } else if (kind == EMG_BC_DIRICHLET) {
                    for (int k = 0; k < 5; k++) v[k] = p.state[side][k];
                    break;
                } else {
                    const int64_t layer = side == 0 ? -x : x - n + 1;
                    ch[side].conserved(e, (double)layer, v);
                    break;
                }
            }
            if (flip) v[1 + p.d] = -v[1 + p.d];
        };
        // periodic sources (C/solver.rs:62-70)
        int64_t lo_s, hi_s;
        if (n >= ng) {
            lo_s = n + gi;
            hi_s = ng + gi;
        } else {
            lo_s = ng + (gi + n - ng % n) % n;
            hi_s = ng + gi % n;
        }
        double v[5];
        switch (p.kind[0]) {
            case EMG_BC_PERIODIC: load(lo_s, v); break;
            case EMG_BC_OUTFLOW: load(ng, v); break;
            case EMG_BC_DIRICHLET:
                for (int k = 0; k < 5; k++) v[k] = p.state[0][k];
                break;
            case EMG_BC_CHARACTERISTIC: ch[0].conserved(e, (double)(ng - gi), v); break;
            default:
                if (p.deep && n < ng) {
                    reflected(gi - ng, v);
                } else {
                    load(2 * ng - 1 - gi, v);
                    v[1 + p.d] = -v[1 + p.d];
                }
        }
        if (in_bounds(p.ctl, at(gi), p.ncell))
            for (int k = 0; k < 5; k++) p.u[k * p.ncell + at(gi)] = v[k];
        switch (p.kind[1]) {
            case EMG_BC_PERIODIC: load(hi_s, v); break;
            case EMG_BC_OUTFLOW: load(n + ng - 1, v); break;
            case EMG_BC_DIRICHLET:
                for (int k = 0; k < 5; k++) v[k] = p.state[1][k];
                break;
            case EMG_BC_CHARACTERISTIC: ch[1].conserved(e, (double)(gi + 1), v); break;
            default:
                if (p.deep && n < ng) {
                    reflected(n + gi, v);
                } else {
                    load(n + ng - 1 - gi, v);
                    v[1 + p.d] = -v[1 + p.d];
                }
        }
        if (in_bounds(p.ctl, at(n + ng + gi), p.ncell))
            for (int k = 0; k < 5; k++) p.u[k * p.ncell + at(n + ng + gi)] = v[k];
    }
}


// CFL rate max over interior cells of Σ_d (|u_d| + c)/dx_d (C/solver.rs:478-516).
__global__ void cfl_kernel(const double* __restrict__ u, int64_t ncell, CellRange cr, int a0, int a1, int a2, double dx0,
                           double dx1, double dx2, EosD eosd, StepCtl* ctl) {
    const Eos<double> e = Eos<double>::from(eosd);
    const int act[3] = {a0, a1, a2};
    const double dx[3] = {dx0, dx1, dx2};
    double rate = 0.0;
    int bad = 0;  // a non-finite or inadmissible interior cell
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < cr.cells; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = cr.index(t);
        double q[5], w[5];
        for (int k = 0; k < 5; k++) q[k] = u[k * ncell + c];
        to_prim(e, q, w);
        if (!admissible(e, w[0], w[4])) bad = 1;
        const double cs = sound_speed(e, w[0], w[4]);
        double acc = -0.0;
        for (int d = 0; d < 3; d++)
            if (act[d]) acc = acc + (fabs(w[1 + d]) + cs) / dx[d];
        rate = fmax(rate, acc);
    }
    for (int o = 16; o > 0; o >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, o));
    __shared__ double s[32];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = rate;
    const int any_bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        double v = s[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = fmax(v, s[w]);
        if (!isnan(v) && v > 0.0) atomicMax(&ctl->rate_bits, (unsigned long long)__double_as_longlong(v));
        if (any_bad) atomicCAS(&ctl->status, 0, (int)EMG_ERR_INADMISSIBLE);
    }
}

// the rate (and the status it may raise) is recomputed from the current state
__global__ void ctl_reset_rate(StepCtl* ctl) {
    ctl->rate_bits = 0ull;
    ctl->status = 0;
}

// Host-given dt (Solver::step / GpuSolver::step).
__global__ void ctl_begin_host(StepCtl* ctl, double dt) {
    ctl->dt = dt;
    ctl->done = 0;
    ctl->status = 0;
    ctl->rate_bits = 0ull;
}

// Device dt = min(cfl / rate, t_end − t) with the stopping rule and collapse
// check of Solver::run_to (C/solver.rs:758-768).
__global__ void ctl_begin_device(StepCtl* ctl, double cfl) {
    if (ctl->done) return;
    if (ctl->status) {  // the previous step left an inadmissible state
        ctl->done = 1;
        return;
    }
    const double rate = __longlong_as_double((long long)ctl->rate_bits);
    const double t = ctl->t, t_end = ctl->t_end;
    double dt = cfl / rate;
    if (isinf(t_end)) {
        if (!(isfinite(dt) && dt > 0.0)) {
            ctl->status = EMG_ERR_DT_COLLAPSED;
            ctl->done = 1;
            return;
        }
    } else {
        if (!(t < t_end - 1e-10 * fabs(t_end))) {
            ctl->done = 1;
            return;
        }
        dt = fmin(dt, t_end - t);
        if (!(isfinite(dt) && dt > 1e-12 * fmax(fabs(t_end), 1e-300))) {
            ctl->status = EMG_ERR_DT_COLLAPSED;
            ctl->done = 1;
            return;
        }
    }
    ctl->dt = dt;
    ctl->rate_bits = 0ull;
}

// Fixed scratch of the allocation-free step: a 256-byte control block, then
// the two stage buffers and the residual for grids up to
// EMG_NOALLOC_MAX_CELLS padded cells.
constexpr size_t NOALLOC_CTL_DOUBLES = 32;
static_assert(sizeof(StepCtl) <= NOALLOC_CTL_DOUBLES * sizeof(double), "control block does not fit");
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_CTL_DOUBLES + 3 * 5 * (size_t)EMG_NOALLOC_MAX_CELLS];

// zero the whole control block (status, counters, flags) and set dt
__global__ void ctl_reset_all(StepCtl* ctl, double dt) {
    unsigned char* b = reinterpret_cast<unsigned char*>(ctl);
    for (int i = threadIdx.x; i < (int)sizeof(StepCtl); i += blockDim.x) b[i] = 0;
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->dt = dt;
        ctl->t_end = INFINITY;
    }
}

__global__ void ctl_end(StepCtl* ctl) {
    if (ctl->done) return;
    ctl->t = ctl->t + ctl->dt;
    ctl->steps += 1;
}

// Σ u·vol over interior cells: per-block partial sums, then one block adds
// the partials in a fixed order (deterministic).
__global__ void totals_partial(const double* __restrict__ u, int64_t ncell, CellRange cr, double vol, double* partial) {
    double s[5] = {0, 0, 0, 0, 0};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < cr.cells; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = cr.index(t);
        for (int k = 0; k < 5; k++) s[k] = s[k] + u[k * ncell + c] * vol;
    }
    __shared__ double sh[5][256];
    for (int k = 0; k < 5; k++) sh[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h)
            for (int k = 0; k < 5; k++) sh[k][threadIdx.x] = sh[k][threadIdx.x] + sh[k][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 5; k++) partial[5 * blockIdx.x + k] = sh[k][0];
}
__global__ void totals_final(const double* partial, int nblocks, double* out) {
    if (threadIdx.x < 5) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s = s + partial[5 * b + threadIdx.x];
        out[threadIdx.x] = s;
    }
}

}  // namespace emg

using namespace emg;

// ------------------------------------------------------------------ solver object (uniform_internal.h)

namespace emg {

cudaError_t sweep_prepare_device() {
    static std::mutex mu;
    static bool prepared[64] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && prepared[dev]) return cudaSuccess;
    e = sweep_prepare_f64();
    if (e == cudaSuccess) e = sweep_prepare_mixed();
    if (e == cudaSuccess) e = sweep_prepare_fast();
    if (e == cudaSuccess && dev >= 0 && dev < 64) prepared[dev] = true;
    return e;
}

int kernel_grid(int64_t work, int threads) {
    int64_t b = (work + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 16) b = 148 * 16;
    return (int)b;
}

cudaEvent_t take_event(emg_uniform* h) {
    if (!h->pool.empty()) {
        cudaEvent_t e = h->pool.back();
        h->pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

struct ProfScope {
    emg_uniform* h;
    int kind;
    cudaEvent_t a = nullptr;
    ProfScope(emg_uniform* hh, int k) : h(hh), kind(k) {
        h->launches++;
        if (h->profiling) {
            a = take_event(h);
            cudaEventRecord(a, h->stream);
        }
    }
    ~ProfScope() {
        if (h->profiling) {
            cudaEvent_t b = take_event(h);
            cudaEventRecord(b, h->stream);
            h->recs.push_back({kind, a, b});
        }
    }
};

// launch grid of the sweep along d for P pencils per CTA and segments of seg cells
dim3 sweep_grid(const emg_uniform* h, int d, int P, int64_t seg) {
    const int64_t nd = h->mesh.n[d], nl = h->mesh.n[h->lane_axis[d]], nother = h->mesh.n[h->other_axis[d]];
    return dim3((unsigned)((nl + P - 1) / P), (unsigned)((nd + seg - 1) / seg), (unsigned)nother);
}

// Segment length of the sweep along d: the fewest (waves of CTAs) × (rows a
// CTA streams, seg + 6 with the halo) over the slots of resident CTAs of the
// whole GPU; a shorter segment only when it is 5 % cheaper. Short segments
// fill the SMs on small grids, and a wave count just above a whole number is
// avoided.
int64_t plan_seg(const emg_uniform* h, int d, int P) {
    const int64_t nd = h->mesh.n[d], nl = h->mesh.n[h->lane_axis[d]], nother = h->mesh.n[h->other_axis[d]];
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    // at most 3 resident CTAs per SM count as slots: a fourth shares the SM's
    // FP64 pipe instead of adding throughput, so cutting pencils into shorter
    // segments to fill it only adds halo rows (the 2-D 512² step measured
    // 20 % slower planned for 4)
    const int per_sm = std::min(3, h->opts.precision == EMG_PRECISION_MIXED      ? sweep_ctas_per_sm_mixed(P, h->opts.mode)
                                   : h->opts.precision == EMG_PRECISION_F64_FAST ? sweep_ctas_per_sm_fast(P, h->opts.mode)
                                                                                 : sweep_ctas_per_sm_f64(P, h->opts.mode));
    const int64_t slots = (int64_t)sms * per_sm;
    const int64_t lane_tiles = (nl + P - 1) / P;
    int64_t best = nd;
    double best_cost = 1e300;
    for (int64_t k = 1; k <= nd; k++) {
        const int64_t seg = (nd + k - 1) / k;
        if (k > 1 && seg < 16) break;
        if ((nd + seg - 1) / seg != k) continue;  // same seg as a smaller k
        const int64_t ctas = lane_tiles * k * nother;
        if (k > 65535) break;
        const double cost = (double)((ctas + slots - 1) / slots) * (double)(seg + 6);
        if (cost < best_cost * 0.95) {  // shorter segments only for a clear gain
            best_cost = cost;
            best = seg;
        }
    }
    return best;
}

void plan_sweeps(emg_uniform* h) {
    for (int d = 0; d < 3; d++) {
        if (!h->active[d]) continue;
        // lane axis: the active other axis with the smallest stride
        int o[2], no = 0;
        for (int e = 0; e < 3; e++)
            if (e != d) o[no++] = e;
        int lane = o[1], other = o[0];  // o[1] has the smaller stride
        if (!h->active[o[1]] && h->active[o[0]]) {
            lane = o[0];
            other = o[1];
        }
        h->lane_axis[d] = lane;
        h->other_axis[d] = other;
        const int64_t nd = h->mesh.n[d], nl = h->mesh.n[lane], nother = h->mesh.n[other];
        // hybrid rings hold RM + 9 rows: P = 16 keeps them at 2 CTAs per SM
        int P = h->opts.mode == EMG_MODE_HYBRID ? 16 : 32;
        if (nl <= 8)
            P = 8;
        else if (nl <= 16)
            P = 16;
        const int64_t lane_tiles = (nl + P - 1) / P;
        const int64_t seg = plan_seg(h, d, P);
        h->sweepP[d] = P;
        h->sweepSeg[d] = (int)seg;
        h->sweepGrid[d] = dim3((unsigned)lane_tiles, (unsigned)((nd + seg - 1) / seg), (unsigned)nother);
    }
}

int launch_ghosts(emg_uniform* h, double* arr) {
    for (int d = 0; d < 3; d++) {
        if (!h->active[d]) continue;
        GhostParams p{};
        p.u = arr;
        p.ctl = h->ctl;
        p.ncell = h->ncell;
        for (int k = 0; k < 3; k++) {
            p.m[k] = h->m[k];
            p.stride[k] = h->stride[k];
        }
        p.n = h->mesh.n[d];
        p.ng = h->mesh.ng;
        p.d = d;
        p.e0 = d == 0 ? 1 : 0;
        p.e1 = d == 2 ? 1 : 2;
        p.deep = h->deep ? 1 : 0;
        for (int s = 0; s < 2; s++) {
            p.kind[s] = h->bc[2 * d + s].kind;
            for (int k = 0; k < 5; k++) p.state[s][k] = h->bc[2 * d + s].state[k];
        }
        p.eos = EosD{h->eos.gamma, h->eos.p_inf, h->eos.b, h->eos.q};
        const int64_t work = h->m[p.e0] * h->m[p.e1] * p.ng;
        ProfScope ps(h, EMG_K_GHOST);
        ghost_kernel<<<kernel_grid(work, 256), 256, 0, h->stream>>>(p);
        EMG_CUDA(cudaGetLastError());
    }
    return EMG_OK;
}

int launch_axis(emg_uniform* h, int stage, int d, double* in, bool first, bool last);

// TMA staging of the sweeps' row loads. Qualifying grids: 3-D, WENO mode,
// ng even and n2 even (so that the k coordinate of every box starts on a
// 16-byte boundary and every stride of the 4-D map (k, j, i, field) is a
// multiple of 16 bytes), and a TMA kernel that keeps the plain kernel's
// resident CTAs per SM. Each map covers one whole stage buffer of this GPU;
// its box is one round of the sweep along d: RM = 8 rows × 32 lanes × 1 ×
// 5 fields. Off unless EMG_TMA=1 is set in the environment: on the B200 the
// staged sweeps measured no faster than the per-thread loads (256³: axis 2
// 10.91 ms per step either way, axes 0-1 and the mixed form 1-2 % slower,
// the 10 KB staging buffer taking shared memory from the L1 that holds the
// sweep's register spills).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        cudaGetLastError();
    });
    return fn;
}

// TMA row staging is an explicit opt-in (EMG_TMA=1): it is used wherever its
// alignment conditions hold, although its staging tile leaves room for fewer
// resident CTAs per SM (3) than the plain-load sweeps (4)
void setup_tma(emg_uniform* h) {
    h->tma = 0;
    const char* on = std::getenv("EMG_TMA");
    if (!on || on[0] != '1') return;
    if (h->ndim != 3 || h->opts.mode != EMG_MODE_WENO || h->mesh.ng % 2 != 0 || h->m[2] % 2 != 0) return;
    if (h->opts.precision == EMG_PRECISION_F64_FAST) return;  // plain loads only
    const bool mixed = h->opts.precision == EMG_PRECISION_MIXED;
    const int staged = mixed ? sweep_tma_ctas_per_sm_mixed() : sweep_tma_ctas_per_sm_f64();
    if (staged < 1) return;
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) return;
    const cuuint64_t dims[4] = {(cuuint64_t)h->m[2], (cuuint64_t)h->m[1], (cuuint64_t)h->m[0], 5};
    const cuuint64_t strides[3] = {(cuuint64_t)h->m[2] * 8, (cuuint64_t)(h->m[1] * h->m[2]) * 8, (cuuint64_t)h->ncell * 8};
    const cuuint32_t ones[4] = {1, 1, 1, 1};
    const int RM = SWEEP_THREADS / 32;
    double* bufs[3] = {h->u, h->sa, h->sb};
    for (int b = 0; b < 3; b++)
        for (int d = 0; d < 3; d++) {
            // box per sweep axis (dims k, j, i, field): rows along d, 32 lanes along the lane axis
            cuuint32_t box[4];
            if (d == 0) {
                box[0] = 32; box[1] = 1; box[2] = RM;
            } else if (d == 1) {
                box[0] = 32; box[1] = RM; box[2] = 1;
            } else {
                box[0] = RM; box[1] = 32; box[2] = 1;
            }
            box[3] = 5;
            CUresult r = enc(&h->tmap[b][d], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, bufs[b], dims, strides, box, ones,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return;
        }
    h->tma = 1;
}

int launch_stage(emg_uniform* h, int stage) {
    double* in = stage == 1 ? h->u : (stage == 2 ? h->sa : h->sb);
    int rc = launch_ghosts(h, in);
    if (rc) return rc;
    int first_axis = -1, last_axis = -1;
    for (int d = 0; d < 3; d++)
        if (h->active[d]) {
            if (first_axis < 0) first_axis = d;
            last_axis = d;
        }
    for (int d = 0; d < 3; d++) {
        if (!h->active[d]) continue;
        if ((rc = launch_axis(h, stage, d, in, d == first_axis, d == last_axis))) return rc;
    }
    return EMG_OK;
}

// one fused sweep of stage `stage` along d with the planned launch shape
int launch_axis(emg_uniform* h, int stage, int d, double* in, bool first, bool last) {
    {
        SweepParams p{};
        p.uin = in;
        p.rhs = h->rhs;
        p.ctl = h->ctl;
        p.ncell = h->ncell;
        const int l = h->lane_axis[d], o = h->other_axis[d];
        p.sd = h->stride[d];
        p.sl = h->stride[l];
        p.so = h->stride[o];
        p.nd = (int)h->mesh.n[d];
        p.nl = (int)h->mesh.n[l];
        p.no = (int)h->mesh.n[o];
        p.gd = h->active[d] ? (int)h->mesh.ng : 0;
        p.gl = h->active[l] ? (int)h->mesh.ng : 0;
        p.go = h->active[o] ? (int)h->mesh.ng : 0;
        p.d = d;
        p.seg = h->sweepSeg[d];
        p.lw = h->sweepP[d];
        p.first = first;
        p.last = last;
        p.stage = stage;
        p.rows_contig = p.sd == 1;
        p.dx = h->mesh.dx[d];
        p.ndim = (double)h->ndim;
        p.positivity = h->opts.positivity ? 1 : 0;
        p.eos = EosD{h->eos.gamma, h->eos.p_inf, h->eos.b, h->eos.q};
        if (p.last) {
            if (stage == 1) {
                p.base = h->u;
                p.cur = nullptr;
                p.dest = h->sa;
            } else if (stage == 2) {
                p.base = h->u;
                p.cur = h->sa;
                p.dest = h->sb;
            } else {
                p.base = h->sb;
                p.cur = h->u;
                p.dest = h->u;
                p.cfl_fuse = 1;
                for (int k = 0; k < 3; k++) {
                    p.cfl_active[k] = h->active[k];
                    p.cfl_dx[k] = h->mesh.dx[k];
                }
            }
        }
        ProfScope ps(h, EMG_K_AXIS_0 + d);
        p.tol = h->opts.tol;
        p.theta_rec = h->theta_rec[stage - 1][d];
        // TMA staging: 32 pencils per CTA, the stage input one of the three
        // mapped buffers, and along k (d = 2) an even first row in every segment
        int buf = -1;
        if (h->tma && h->sweepP[d] == 32 && (d != 2 || h->sweepSeg[d] % 2 == 0 || h->sweepGrid[d].y == 1))
            buf = in == h->u ? 0 : (in == h->sa ? 1 : (in == h->sb ? 2 : -1));
        cudaError_t e;
        if (buf >= 0)
            e = h->opts.precision == EMG_PRECISION_MIXED
                    ? sweep_launch_tma_mixed(p, h->tmap[buf][d], h->sweepGrid[d], h->stream)
                    : sweep_launch_tma_f64(p, h->tmap[buf][d], h->sweepGrid[d], h->stream);
        else if (h->opts.precision == EMG_PRECISION_MIXED)
            e = sweep_launch_mixed(h->sweepP[d], h->opts.mode, p, h->sweepGrid[d], h->stream);
        else if (h->opts.precision == EMG_PRECISION_F64_FAST)
            e = sweep_launch_fast(h->sweepP[d], h->opts.mode, p, h->sweepGrid[d], h->stream);
        else
            e = sweep_launch_f64(h->sweepP[d], h->opts.mode, p, h->sweepGrid[d], h->stream);
        if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("sweep launch: ") + cudaGetErrorString(e));
    }
    return EMG_OK;
}

// Project-written autotuner of the sweep launch shape: per active axis, every
// candidate (pencils per CTA P ∈ {8, 16, 32}, segment length nd, nd/2, nd/4)
// sweeps the current state once untimed and three times timed (residual only:
// no RK epilogue), and the fastest is kept. A sweep's results do not depend on
// its launch shape (each cell's arithmetic is the same), so tuning changes
// speed only. Shapes are cached per (mesh extents, flux mode, precision).
struct TuneKey {
    int64_t n[3];
    int mode, precision;
    bool operator<(const TuneKey& o) const {
        for (int d = 0; d < 3; d++)
            if (n[d] != o.n[d]) return n[d] < o.n[d];
        return mode != o.mode ? mode < o.mode : precision < o.precision;
    }
};
struct TuneVal {
    int P[3];
    int seg[3];
};

int autotune_sweeps(emg_uniform* h) {
    static std::mutex mu;
    static std::map<TuneKey, TuneVal> cache;
    TuneKey key{{h->mesh.n[0], h->mesh.n[1], h->mesh.n[2]}, h->opts.mode, h->opts.precision};
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            for (int d = 0; d < 3; d++)
                if (h->active[d]) {
                    h->sweepP[d] = it->second.P[d];
                    h->sweepSeg[d] = it->second.seg[d];
                    h->sweepGrid[d] = sweep_grid(h, d, h->sweepP[d], h->sweepSeg[d]);
                }
            return EMG_OK;
        }
    }
    int rc = launch_ghosts(h, h->u);
    if (rc) return rc;
    ctl_begin_host<<<1, 1, 0, h->stream>>>(h->ctl, 1e-12);
    EMG_CUDA(cudaGetLastError());
    cudaEvent_t a, b;
    EMG_CUDA(cudaEventCreate(&a));
    EMG_CUDA(cudaEventCreate(&b));
    TuneVal best{};
    for (int d = 0; d < 3; d++) {
        if (!h->active[d]) continue;
        const int64_t nd = h->mesh.n[d], nl = h->mesh.n[h->lane_axis[d]];
        float best_ms = 1e30f;
        best.P[d] = h->sweepP[d];
        best.seg[d] = h->sweepSeg[d];
        for (int P : {8, 16, 32}) {
            if (P > 8 && nl <= P / 2) continue;                         // lanes mostly idle
            if (P == 32 && h->opts.mode == EMG_MODE_HYBRID) continue;  // hybrid rings: one CTA per SM at P = 32
            const int64_t planned = plan_seg(h, d, P);
            std::set<int64_t> segs = {nd, (nd + 1) / 2, (nd + 3) / 4, planned, std::min(nd, 2 * planned), (planned + 1) / 2};
            for (int64_t seg : segs) {
                if (seg < 16 && seg != nd) continue;
                const dim3 g = sweep_grid(h, d, P, seg);
                if (g.y > 65535u || g.z > 65535u) continue;
                h->sweepP[d] = P;
                h->sweepSeg[d] = (int)seg;
                h->sweepGrid[d] = g;
                if ((rc = launch_axis(h, 1, d, h->u, true, false))) return rc;
                cudaEventRecord(a, h->stream);
                for (int r = 0; r < 3; r++)
                    if ((rc = launch_axis(h, 1, d, h->u, true, false))) return rc;
                cudaEventRecord(b, h->stream);
                EMG_CUDA(cudaEventSynchronize(b));
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, a, b);
                if (ms < best_ms) {
                    best_ms = ms;
                    best.P[d] = P;
                    best.seg[d] = (int)seg;
                }
            }
        }
        h->sweepP[d] = best.P[d];
        h->sweepSeg[d] = best.seg[d];
        h->sweepGrid[d] = sweep_grid(h, d, best.P[d], best.seg[d]);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    // the timing sweeps touched the residual and the counters: reset the control block
    std::memset(h->ctl_host, 0, sizeof(StepCtl));
    h->ctl_host->t_end = INFINITY;
    EMG_CUDA(cudaMemcpyAsync(h->ctl, h->ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    h->launches = 0;
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = best;
    return EMG_OK;
}

int launch_step_body(emg_uniform* h) {
    for (int s = 1; s <= 3; s++) {
        int rc = launch_stage(h, s);
        if (rc) return rc;
    }
    {
        ProfScope ps(h, EMG_K_CFL);
        ctl_end<<<1, 1, 0, h->stream>>>(h->ctl);
        EMG_CUDA(cudaGetLastError());
    }
    // host-side face statistics (every face of every pencil, each stage)
    uint64_t f = 0;
    for (int d = 0; d < 3; d++)
        if (h->active[d]) f += (uint64_t)(h->cells / h->mesh.n[d]) * (uint64_t)(h->mesh.n[d] + 1);
    h->faces += 3 * f;
    if (h->opts.mode == EMG_MODE_WENO) h->weno_faces += 3 * f;
    return EMG_OK;
}

int ensure_rate(emg_uniform* h) {
    if (h->rate_valid) return EMG_OK;
    ctl_reset_rate<<<1, 1, 0, h->stream>>>(h->ctl);
    EMG_CUDA(cudaGetLastError());
    CellRange cr{};
    for (int d = 0; d < 3; d++) {
        cr.n[d] = h->mesh.n[d];
        cr.g[d] = h->active[d] ? h->mesh.ng : 0;
        cr.stride[d] = h->stride[d];
    }
    cr.cells = h->cells;
    {
        ProfScope ps(h, EMG_K_CFL);
        cfl_kernel<<<kernel_grid(h->cells, 256), 256, 0, h->stream>>>(
            h->u, h->ncell, cr, h->active[0], h->active[1], h->active[2], h->mesh.dx[0], h->mesh.dx[1], h->mesh.dx[2],
            EosD{h->eos.gamma, h->eos.p_inf, h->eos.b, h->eos.q}, h->ctl);
        EMG_CUDA(cudaGetLastError());
    }
    h->rate_valid = true;
    return EMG_OK;
}

int sync_ctl(emg_uniform* h) {
    EMG_CUDA(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    h->t_host = h->ctl_host->t;
    return EMG_OK;
}

double bits_to_double(unsigned long long b) {
    double v;
    std::memcpy(&v, &b, sizeof v);
    return v;
}

// the status the device raised, as read by the last sync_ctl
int check_status(emg_uniform* h) {
    const int st = h->ctl_host->status;
    if (st == EMG_ERR_DT_COLLAPSED) return set_error(st, "time step collapsed: the solution lost admissibility");
    if (st == EMG_ERR_INADMISSIBLE)
        return set_error(st, "non-finite or inadmissible state (density, pressure or specific volume) in an interior cell");
    if (st == EMG_ERR_BOUNDS) return set_error(st, "device index out of range (bounds-check build)");
    if (st) return set_error(st, "device error");
    return EMG_OK;
}

int check_handle(emg_uniform* h) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return EMG_OK;
}

}  // namespace emg

extern "C" {

const char* emg_last_error(void) { return g_last_error.c_str(); }

const char* emg_version(void) { return "0.1.0"; }

int emg_device_count(int* count) {
    if (!count) return set_error(EMG_ERR_INVALID, "null count");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        *count = 0;
        cudaGetLastError();
        return EMG_OK;
    }
    int c = 0;
    for (int i = 0; i < n; i++) {
        cudaDeviceProp pr;
        if (cudaGetDeviceProperties(&pr, i) == cudaSuccess && pr.major == 10) c++;
    }
    *count = c;
    return EMG_OK;
}

int emg_state_hash(const emg_mesh* mesh, const double* u_aos, size_t len, uint64_t* out) {
    if (!mesh || !u_aos || !out) return set_error(EMG_ERR_INVALID, "null argument");
    int64_t m[3], g[3];
    size_t padded = 1;
    for (int d = 0; d < 3; d++) {
        if (mesh->n[d] < 1 || mesh->ng < 0) return set_error(EMG_ERR_INVALID, "mesh extents must be >= 1");
        g[d] = mesh->n[d] > 1 ? mesh->ng : 0;
        m[d] = mesh->n[d] + 2 * g[d];
        padded *= (size_t)m[d];
    }
    if (padded != len) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    uint64_t h = 0xcbf29ce484222325ull;
    for (int64_t i = 0; i < mesh->n[0]; i++)
        for (int64_t j = 0; j < mesh->n[1]; j++)
            for (int64_t k = 0; k < mesh->n[2]; k++) {
                const double* v = u_aos + 5 * (((i + g[0]) * m[1] + (j + g[1])) * m[2] + (k + g[2]));
                for (int q = 0; q < 5; q++) {
                    uint64_t bits;
                    std::memcpy(&bits, v + q, sizeof bits);
                    h = (h ^ bits) * 0x100000001b3ull;
                }
            }
    *out = h;
    return EMG_OK;
}

// Argument checks shared by emg_uniform_create and emg_uniform_step_noalloc,
// made before any device work. *ndim receives the number of active axes and
// *padded the padded cell count m0·m1·m2.
static int check_uniform_args(const emg_mesh* mesh, const emg_bc bc[6], const emg_opts* opts, int* ndim, size_t* padded) {
    if (mesh->ng < 5) return set_error(EMG_ERR_INVALID, "the WCNS stencil needs ng >= 5 ghost layers");
    int nd = 0;
    size_t cells = 1;
    for (int d = 0; d < 3; d++) {
        if (mesh->n[d] < 1) return set_error(EMG_ERR_INVALID, "mesh extents must be >= 1");
        if (mesh->n[d] > 1) {
            nd++;
            if (!(mesh->dx[d] > 0.0)) return set_error(EMG_ERR_INVALID, "dx must be > 0 on active axes");
            if (mesh->n[d] > (1 << 30)) return set_error(EMG_ERR_INVALID, "axis too long");
            cells *= (size_t)(mesh->n[d] + 2 * mesh->ng);
        }
    }
    if (nd == 0) return set_error(EMG_ERR_INVALID, "mesh has no active axis");
    if (opts->mode != EMG_MODE_WENO && opts->mode != EMG_MODE_HYBRID && opts->mode != EMG_MODE_CENTRAL)
        return set_error(EMG_ERR_INVALID, "unknown flux mode");
    if (opts->mode == EMG_MODE_HYBRID && !(opts->tol > 0.0))
        return set_error(EMG_ERR_INVALID, "hybrid mode needs tol > 0");
    if (opts->precision != EMG_PRECISION_F64 && opts->precision != EMG_PRECISION_MIXED &&
        opts->precision != EMG_PRECISION_F64_FAST)
        return set_error(EMG_ERR_INVALID, "unknown precision");
    for (int i = 0; i < 6; i++)
        if (bc[i].kind < 0 || bc[i].kind > 4) return set_error(EMG_ERR_INVALID, "unknown boundary condition");
    for (int d = 0; d < 3; d++) {
        const bool per0 = bc[2 * d].kind == EMG_BC_PERIODIC, per1 = bc[2 * d + 1].kind == EMG_BC_PERIODIC;
        if (mesh->n[d] > 1 && per0 != per1) return set_error(EMG_ERR_INVALID, "periodic boundaries must be paired");
    }
    *ndim = nd;
    *padded = cells;
    return EMG_OK;
}

}  // extern "C"

namespace {
// The large state buffers of uniform-grid solvers come from a library-owned
// stream-ordered memory pool per device that keeps up to 32 GB of freed
// memory: cudaMalloc of a 256^3 state (4 GB over five buffers) costs 5-60 ms,
// and a solver created after another one was destroyed reuses its memory.
// emg_release_memory returns the kept memory to the device.
std::mutex pool_mu;
cudaMemPool_t pools[64] = {};
cudaMemPool_t state_pool(int dev) {
    if (dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(pool_mu);
    if (!pools[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        uint64_t keep = 32ull << 30;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[dev] = p;
    }
    return pools[dev];
}
}  // namespace

extern "C" {

int emg_release_memory(void) {
    std::lock_guard<std::mutex> lk(pool_mu);
    for (auto& p : pools)
        if (p && cudaMemPoolTrimTo(p, 0) != cudaSuccess) {
            cudaGetLastError();
            return set_error(EMG_ERR_CUDA, "memory pool trim failed");
        }
    return EMG_OK;
}

int emg_uniform_create(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                       const double* u_aos, size_t len, emg_uniform** out) {
    if (!mesh || !eos || !bc || !opts || !u_aos || !out) return set_error(EMG_ERR_INVALID, "null argument");
    *out = nullptr;
    // arguments first, so that a bad call is reported as such on any host
    int ndim = 0;
    size_t padded = 0;
    if (int rc = check_uniform_args(mesh, bc, opts, &ndim, &padded)) return rc;
    if (padded != len) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
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
    emg_uniform* h = new emg_uniform();
    h->device = dev;
    h->mesh = *mesh;
    h->eos = *eos;
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
    for (int d = 0; d < 3; d++)
        if (h->active[d] && mesh->n[d] < mesh->ng &&
            (bc[2 * d].kind == EMG_BC_REFLECT || bc[2 * d + 1].kind == EMG_BC_REFLECT))
            h->deep = true;
    if ((size_t)h->ncell != len) {
        delete h;
        return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    }
    auto bail = [&](int rc) {
        emg_uniform_destroy(h);
        return rc;
    };
    {
        cudaError_t e = sweep_prepare_device();
        if (e != cudaSuccess) return bail(set_error(EMG_ERR_CUDA, std::string("sweep setup: ") + cudaGetErrorString(e)));
    }
    cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(set_error(EMG_ERR_CUDA, "cudaStreamCreate failed"));
    const size_t bytes = (size_t)h->ncell * 5 * sizeof(double);
    cudaMemPool_t pool = state_pool(h->device);
    if (!pool) return bail(set_error(EMG_ERR_CUDA, "device memory pool unavailable"));
    if (cudaMallocFromPoolAsync((void**)&h->u, bytes, pool, h->stream) != cudaSuccess ||
        cudaMallocFromPoolAsync((void**)&h->sa, bytes, pool, h->stream) != cudaSuccess ||
        cudaMallocFromPoolAsync((void**)&h->sb, bytes, pool, h->stream) != cudaSuccess ||
        cudaMallocFromPoolAsync((void**)&h->rhs, bytes, pool, h->stream) != cudaSuccess ||
        cudaMallocFromPoolAsync((void**)&h->staging, bytes, pool, h->stream) != cudaSuccess ||
        cudaMalloc(&h->partial, 5 * 4096 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->ctl, sizeof(StepCtl)) != cudaSuccess ||
        cudaMallocHost(&h->ctl_host, sizeof(StepCtl)) != cudaSuccess) {
        cudaGetLastError();
        return bail(set_error(EMG_ERR_CUDA, "device allocation failed"));
    }
    // ghosts of the stage buffers are always rewritten before they are read; zero them once anyway
    cudaMemsetAsync(h->sa, 0, bytes, h->stream);
    cudaMemsetAsync(h->sb, 0, bytes, h->stream);
    cudaMemsetAsync(h->rhs, 0, bytes, h->stream);
    std::memset(h->ctl_host, 0, sizeof(StepCtl));
    h->ctl_host->t_end = INFINITY;
    if (cudaMemcpyAsync(h->ctl, h->ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return bail(set_error(EMG_ERR_CUDA, "control block upload failed"));
    plan_sweeps(h);
    for (int d = 0; d < 3; d++)
        if (h->active[d] && (h->sweepGrid[d].y > 65535u || h->sweepGrid[d].z > 65535u))
            return bail(set_error(EMG_ERR_INVALID, "mesh too large for the sweep grid (an axis above 65535 pencils)"));
    setup_tma(h);
    int rc = emg_uniform_upload(h, u_aos, len);
    if (rc) return bail(rc);
    if ((opts->flags & EMG_OPT_AUTOTUNE) && (rc = autotune_sweeps(h))) return bail(rc);
    *out = h;
    return EMG_OK;
}

int emg_uniform_destroy(emg_uniform* h) {
    if (!h) return EMG_OK;
    cudaSetDevice(h->device);
    // the state buffers go back to the library's pool (stream-ordered), the rest is freed
    if (h->stream) {
        for (double* p : {h->u, h->sa, h->sb, h->rhs, h->staging})
            if (p) cudaFreeAsync(p, h->stream);
        cudaStreamSynchronize(h->stream);
    }
    cudaGetLastError();
    cudaFree(h->partial);
    cudaFree(h->ctl);
    if (h->ctl_host) cudaFreeHost(h->ctl_host);
    for (auto& r : h->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : h->pool) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return EMG_OK;
}

int emg_uniform_upload(emg_uniform* h, const double* u_aos, size_t len) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!u_aos || len != (size_t)h->ncell) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    const size_t bytes = (size_t)h->ncell * 5 * sizeof(double);
    EMG_CUDA(cudaMemcpyAsync(h->staging, u_aos, bytes, cudaMemcpyHostToDevice, h->stream));
    aos_to_soa<<<kernel_grid(h->ncell, 256), 256, 0, h->stream>>>(h->staging, h->u, h->ncell);
    EMG_CUDA(cudaGetLastError());
    h->launches++;
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    h->rate_valid = false;
    return EMG_OK;
}

int emg_uniform_download(emg_uniform* h, double* u_aos, size_t len) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!u_aos || len != (size_t)h->ncell) return set_error(EMG_ERR_INVALID, "state length does not match the padded mesh");
    soa_to_aos<<<kernel_grid(h->ncell, 256), 256, 0, h->stream>>>(h->u, h->staging, h->ncell);
    EMG_CUDA(cudaGetLastError());
    h->launches++;
    EMG_CUDA(cudaMemcpyAsync(u_aos, h->staging, (size_t)h->ncell * 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_uniform_step(emg_uniform* h, double dt) {
    int rc = check_handle(h);
    if (rc) return rc;
    ctl_begin_host<<<1, 1, 0, h->stream>>>(h->ctl, dt);
    EMG_CUDA(cudaGetLastError());
    h->launches++;
    rc = launch_step_body(h);
    if (rc) return rc;
    h->rate_valid = true;
    rc = sync_ctl(h);
    if (rc) return rc;
    return check_status(h);
}

int emg_uniform_dt_cfl(emg_uniform* h, double* dt) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!dt) return set_error(EMG_ERR_INVALID, "null dt");
    rc = ensure_rate(h);
    if (rc) return rc;
    rc = sync_ctl(h);
    if (rc) return rc;
    if ((rc = check_status(h))) return rc;
    const double rate = bits_to_double(h->ctl_host->rate_bits);
    *dt = h->opts.cfl / rate;
    return EMG_OK;
}

int emg_uniform_advance(emg_uniform* h, uint64_t nsteps, double t_end, uint64_t* taken) {
    int rc = check_handle(h);
    if (rc) return rc;
    rc = ensure_rate(h);
    if (rc) return rc;
    // arm device-driven stepping (not from an inadmissible state)
    rc = sync_ctl(h);
    if (rc) return rc;
    if ((rc = check_status(h))) return rc;
    StepCtl c = *h->ctl_host;
    c.t_end = t_end;
    c.done = 0;
    c.status = 0;
    const uint64_t steps0 = c.steps;
    EMG_CUDA(cudaMemcpyAsync(h->ctl, &c, sizeof(StepCtl), cudaMemcpyHostToDevice, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    const bool bounded = !std::isinf(t_end);
    uint64_t issued = 0;
    while (issued < nsteps) {
        const uint64_t batch = bounded ? std::min<uint64_t>(nsteps - issued, 8) : nsteps - issued;
        for (uint64_t s = 0; s < batch; s++) {
            ctl_begin_device<<<1, 1, 0, h->stream>>>(h->ctl, h->opts.cfl);
            EMG_CUDA(cudaGetLastError());
            h->launches++;
            rc = launch_step_body(h);
            if (rc) return rc;
        }
        issued += batch;
        if (bounded) {
            rc = sync_ctl(h);
            if (rc) return rc;
            if (h->ctl_host->done) break;
        }
    }
    rc = sync_ctl(h);
    if (rc) return rc;
    // face statistics were counted for every issued step; correct for skipped ones
    const uint64_t done_steps = h->ctl_host->steps - steps0;
    if (issued > done_steps) {
        uint64_t f = 0;
        for (int d = 0; d < 3; d++)
            if (h->active[d]) f += (uint64_t)(h->cells / h->mesh.n[d]) * (uint64_t)(h->mesh.n[d] + 1);
        h->faces -= 3 * f * (issued - done_steps);
        if (h->opts.mode == EMG_MODE_WENO) h->weno_faces -= 3 * f * (issued - done_steps);
    }
    if (taken) *taken = done_steps;
    h->rate_valid = true;
    return check_status(h);
}

int emg_uniform_run_to(emg_uniform* h, double t_end, uint64_t* steps) {
    if (!std::isfinite(t_end)) return set_error(EMG_ERR_INVALID, "t_end must be finite");
    uint64_t taken = 0;
    int rc = emg_uniform_advance(h, UINT64_MAX / 2, t_end, &taken);
    if (steps) *steps = taken;
    return rc;
}

int emg_uniform_totals(emg_uniform* h, double out[5]) {
    int rc = check_handle(h);
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
    const int nb = (int)std::min<int64_t>(4095, std::max<int64_t>(1, (h->cells + 255) / 256));
    totals_partial<<<nb, 256, 0, h->stream>>>(h->u, h->ncell, cr, vol, h->partial);
    EMG_CUDA(cudaGetLastError());
    totals_final<<<1, 32, 0, h->stream>>>(h->partial, nb, h->partial + 5 * 4095);
    EMG_CUDA(cudaGetLastError());
    h->launches += 2;
    EMG_CUDA(cudaMemcpyAsync(out, h->partial + 5 * 4095, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_uniform_counters(emg_uniform* h, uint64_t out[4]) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!out) return set_error(EMG_ERR_INVALID, "null out");
    rc = sync_ctl(h);
    if (rc) return rc;
    out[0] = h->faces;
    out[1] = h->weno_faces + h->ctl_host->counters[1];  // WENO mode counted on the host, hybrid on the device
    out[2] = h->ctl_host->counters[2];
    out[3] = h->ctl_host->counters[3];
    return EMG_OK;
}

int emg_uniform_get_time(emg_uniform* h, double* t) {
    int rc = check_handle(h);
    if (rc) return rc;
    if (!t) return set_error(EMG_ERR_INVALID, "null t");
    rc = sync_ctl(h);
    if (rc) return rc;
    *t = h->ctl_host->t;
    return EMG_OK;
}

int emg_uniform_set_time(emg_uniform* h, double t) {
    int rc = check_handle(h);
    if (rc) return rc;
    rc = sync_ctl(h);
    if (rc) return rc;
    h->ctl_host->t = t;
    EMG_CUDA(cudaMemcpyAsync(h->ctl, h->ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, h->stream));
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_uniform_synchronize(emg_uniform* h) {
    int rc = check_handle(h);
    if (rc) return rc;
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_uniform_stream(emg_uniform* h, void** stream) {
    if (!h || !stream) return set_error(EMG_ERR_INVALID, "null argument");
    *stream = (void*)h->stream;
    return EMG_OK;
}

int emg_uniform_set_profiling(emg_uniform* h, int on) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    h->profiling = on != 0;
    return EMG_OK;
}

int emg_uniform_kernel_times(emg_uniform* h, double* ms, uint64_t* launches) {
    int rc = check_handle(h);
    if (rc) return rc;
    EMG_CUDA(cudaStreamSynchronize(h->stream));
    for (auto& r : h->recs) {
        float t = 0.f;
        cudaEventElapsedTime(&t, r.a, r.b);
        h->prof_ms[r.kind] += t;
        h->prof_n[r.kind] += 1;
        h->pool.push_back(r.a);
        h->pool.push_back(r.b);
    }
    h->recs.clear();
    for (int k = 0; k < EMG_K_COUNT; k++) {
        if (ms) ms[k] = h->prof_ms[k];
        if (launches) launches[k] = h->prof_n[k];
        h->prof_ms[k] = 0.0;
        h->prof_n[k] = 0;
    }
    return EMG_OK;
}

int emg_uniform_features(emg_uniform* h, uint32_t* flags) {
    if (!h || !flags) return set_error(EMG_ERR_INVALID, "null argument");
    *flags = h->tma ? EMG_FEATURE_TMA : 0u;
    return EMG_OK;
}

int emg_uniform_launch_count(emg_uniform* h, uint64_t* launches) {
    if (!h || !launches) return set_error(EMG_ERR_INVALID, "null argument");
    *launches = h->launches;
    return EMG_OK;
}

// Allocation-free step: the emg_uniform object lives on the host stack and
// its device buffers point into g_noalloc_scratch; nothing is allocated.
int emg_uniform_step_noalloc(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                             const double* u_in, double* u_out, double dt, void* stream) {
    if (!mesh || !eos || !bc || !opts || !u_in || !u_out) return set_error(EMG_ERR_INVALID, "null argument");
    int ndim = 0;
    size_t padded = 0;
    if (int rc = check_uniform_args(mesh, bc, opts, &ndim, &padded)) return rc;
    if (padded > (size_t)EMG_NOALLOC_MAX_CELLS)
        return set_error(EMG_ERR_INVALID, "grid exceeds EMG_NOALLOC_MAX_CELLS padded cells (131072)");
    const int64_t ncell = (int64_t)padded;
    {
        // u_out is written while u_in is still read: no shared byte allowed
        const uintptr_t a0 = (uintptr_t)u_in, b0 = (uintptr_t)u_out, nb = (uintptr_t)padded * 5 * sizeof(double);
        if (a0 < b0 + nb && b0 < a0 + nb) return set_error(EMG_ERR_INVALID, "u_in and u_out must not overlap");
    }
    if (!(std::isfinite(dt) && dt > 0.0)) return set_error(EMG_ERR_INVALID, "dt must be finite and > 0");
    int dev = 0;
    EMG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_error(EMG_ERR_INVALID, "device index out of range");
    // The sweep kernels' shared-memory attribute is set once per device (the
    // first call on a device; make it before any stream capture). The scratch
    // address is looked up on every call, with this device current: a cached
    // address would not survive a device reset or a new primary context.
    static std::mutex prep_mu;
    static bool prepared[64] = {false};
    {
        std::lock_guard<std::mutex> lock(prep_mu);
        if (!prepared[dev]) {
            cudaError_t e = sweep_prepare_device();
            if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("sweep setup: ") + cudaGetErrorString(e));
            prepared[dev] = true;
        }
    }
    double* base = nullptr;
    {
        cudaError_t e = cudaGetSymbolAddress((void**)&base, g_noalloc_scratch);
        if (e != cudaSuccess || !base)
            return set_error(EMG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    }
    emg_uniform h;
    h.device = dev;
    h.stream = (cudaStream_t)stream;
    h.mesh = *mesh;
    h.eos = *eos;
    for (int i = 0; i < 6; i++) h.bc[i] = bc[i];
    h.opts = *opts;
    h.ndim = ndim;
    for (int d = 0; d < 3; d++) {
        h.active[d] = mesh->n[d] > 1;
        h.m[d] = h.active[d] ? mesh->n[d] + 2 * mesh->ng : 1;
    }
    h.stride[2] = 1;
    h.stride[1] = h.m[2];
    h.stride[0] = h.m[1] * h.m[2];
    h.ncell = ncell;
    h.cells = mesh->n[0] * mesh->n[1] * mesh->n[2];
    for (int d = 0; d < 3; d++)
        if (h.active[d] && mesh->n[d] < mesh->ng &&
            (bc[2 * d].kind == EMG_BC_REFLECT || bc[2 * d + 1].kind == EMG_BC_REFLECT))
            h.deep = true;
    h.ctl = reinterpret_cast<StepCtl*>(base);
    h.sa = base + NOALLOC_CTL_DOUBLES;
    h.sb = h.sa + 5 * (size_t)EMG_NOALLOC_MAX_CELLS;
    h.rhs = h.sb + 5 * (size_t)EMG_NOALLOC_MAX_CELLS;
    h.u = u_out;
    plan_sweeps(&h);
    for (int d = 0; d < 3; d++)
        if (h.active[d] && (h.sweepGrid[d].y > 65535u || h.sweepGrid[d].z > 65535u))
            return set_error(EMG_ERR_INVALID, "mesh too large for the sweep grid");
    // u_out starts as a copy of u_in; the stage kernels then work in place on
    // it (ghosts filled at stage 1, the stage-3 update written back)
    EMG_CUDA(cudaMemcpyAsync(u_out, u_in, (size_t)ncell * 5 * sizeof(double), cudaMemcpyDeviceToDevice, h.stream));
    ctl_reset_all<<<1, 128, 0, h.stream>>>(h.ctl, dt);
    EMG_CUDA(cudaGetLastError());
    for (int stage = 1; stage <= 3; stage++) {
        int rc = launch_stage(&h, stage);
        if (rc) return rc;
    }
    EMG_CUDA(cudaGetLastError());
    return EMG_OK;
}

}  // extern "C"
