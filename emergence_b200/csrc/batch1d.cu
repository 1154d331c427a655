// Batched independent 1-D lines (emg_batch1d_*): thousands of Riemann
// problems of different lengths advanced together. Each RK stage is one ghost
// launch and one fused-sweep launch over the segments of all instances
// (sweep.cuh, KIND_BATCH); each instance keeps its own time, CFL time step
// (C/solver.rs:478-523) and stopping rule (C/solver.rs:758-768) on the
// device, so a whole run needs no host round trip per step.
//
// The discrete adjoint of a batched run (emg_batch1d_record / _objective /
// _backward) keeps every instance's time steps and the limiter's blend
// weights of a recorded FP64 run, checkpoints the whole batch every K batch
// steps and reverses each batch step with one adjoint-sweep launch per stage
// over the line segments of all instances that stepped (adjoint.cu).
//
// Built with -fmad=false.
#include "../../include/emergence_b200.h"
#include "adjoint.cuh"
#include "adjoint_launch.h"
#include "sweep_launch.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace emg {
int set_error(int code, const std::string& msg);
}
using namespace emg;

#define B_CUDA(call)                                                                               \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            return set_error(EMG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));  \
    } while (0)

namespace {

constexpr int NG = 6;
// cells per segment (one lane of a sweep CTA): short segments keep the CTAs
// of unfinished instances evenly spread as instances finish at different
// batch steps (4096 Riemann problems: 24 cells 2.8 s, 32 cells 2.9 s, 64 cells
// 3.7 s per run, FP64; the 5 halo midpoints per segment cost less than the
// imbalance of long ones)
constexpr int SEG = 24;

struct Inst {
    int64_t off;   // flat index of the instance's first padded cell
    int64_t n;     // interior cells
    double dx;
    double t;
    double dt;
    double rate_dummy;
    unsigned long long rate_bits;
    unsigned long long steps;
    int done;
    int status;
};

// Ghost layers of every instance (C/solver.rs:278-348 on a 1-D mesh).
__global__ void batch_ghosts(double* u, int64_t ntot, Inst* inst, int ninst, int kind_lo, int kind_hi, EosD eos,
                             const double* st_lo, const double* st_hi) {
    const int i = blockIdx.x;
    if (i >= ninst || inst[i].done) return;
    const int64_t off = inst[i].off, n = inst[i].n;
    for (int t = threadIdx.x; t < 2 * NG; t += blockDim.x) {
        const int side = t / NG, gi = t % NG;
        const int kind = side ? kind_hi : kind_lo;
        int64_t src;
        bool flip = false;
        if (kind == EMG_BC_PERIODIC) {
            if (n >= NG)
                src = side ? NG + gi : n + gi;
            else
                src = side ? NG + gi % n : NG + (gi + n - NG % n) % n;
        } else if (kind == EMG_BC_OUTFLOW) {
            src = side ? n + NG - 1 : NG;
        } else if (kind == EMG_BC_REFLECT) {
            src = side ? n + NG - 1 - gi : 2 * NG - 1 - gi;
            flip = true;
        } else {
            src = -1;  // Dirichlet
        }
        const int64_t dst = off + (side ? n + NG + gi : gi);
        for (int k = 0; k < 5; k++) {
            double v = src >= 0 ? u[k * ntot + off + src] : (side ? st_hi[k] : st_lo[k]);
            if (flip && k == 1) v = -v;
            u[k * ntot + dst] = v;
        }
    }
}

// CFL rate of each instance and its dt (C/solver.rs:478-523, :758-768)
__global__ void batch_begin(const double* __restrict__ u, int64_t ntot, Inst* inst, double* dtv, int ninst, double cfl,
                            double t_end, EosD eosd) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    Inst& I = inst[i];
    __shared__ double sr[32];
    if (I.done) {
        if (threadIdx.x == 0) dtv[i] = 0.0;
        return;
    }
    const Eos<double> e = Eos<double>::from(eosd);
    double rate = 0.0;
    for (int64_t c = threadIdx.x; c < I.n; c += blockDim.x) {
        double q[5], w[5];
        for (int k = 0; k < 5; k++) q[k] = u[k * ntot + I.off + NG + c];
        to_prim(e, q, w);
        const double cs = sound_speed(e, w[0], w[4]);
        double acc = -0.0;
        acc = acc + (fabs(w[1]) + cs) / I.dx;
        rate = fmax(rate, acc);
    }
    for (int o = 16; o > 0; o >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, o));
    if ((threadIdx.x & 31) == 0) sr[threadIdx.x >> 5] = rate;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = sr[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = fmax(r, sr[w]);
        double dt = 0.0;
        if (!(I.t < t_end - 1e-10 * fabs(t_end))) {
            I.done = 1;
        } else {
            dt = fmin(cfl / r, t_end - I.t);
            if (!(isfinite(dt) && dt > 1e-12 * fmax(fabs(t_end), 1e-300))) {
                I.status = EMG_ERR_DT_COLLAPSED;
                I.done = 1;
                dt = 0.0;
            }
        }
        I.dt = dt;
        dtv[i] = dt;
    }
}

__global__ void batch_end(Inst* inst, int ninst, int* active) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ninst) return;
    Inst& I = inst[i];
    if (!I.done && I.dt > 0.0) {
        I.t = I.t + I.dt;
        I.steps += 1;
        atomicAdd(active, 1);
    }
}

__global__ void batch_pack(const double* __restrict__ aos, double* u, int64_t ntot, const Inst* inst, int ninst,
                           const int64_t* __restrict__ coff) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    for (int64_t c = threadIdx.x; c < inst[i].n; c += blockDim.x)
        for (int k = 0; k < 5; k++) u[k * ntot + inst[i].off + NG + c] = aos[(coff[i] + c) * 5 + k];
}
__global__ void batch_unpack(const double* __restrict__ u, double* aos, int64_t ntot, const Inst* inst, int ninst,
                             const int64_t* __restrict__ coff) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    for (int64_t c = threadIdx.x; c < inst[i].n; c += blockDim.x)
        for (int k = 0; k < 5; k++) aos[(coff[i] + c) * 5 + k] = u[k * ntot + inst[i].off + NG + c];
}

// ---- discrete adjoint of batched runs

// done = (no step) for the recorded time steps of one batch step, so that the
// ghost fill of a recomputed step treats every instance as it did then
__global__ void batch_set_done(Inst* inst, const double* __restrict__ dt, int ninst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < ninst) inst[i].done = dt[i] > 0.0 ? 0 : 1;
}

// Reverse of stage 3 (Uⁿ⁺¹ = Uⁿ/3 + ⅔(U² + dt·R)) on interior cells: ān = ⅓ȳ,
// x̄ = ⅔ȳ; an instance that took no step passes ȳ through (ān = ȳ, x̄ = 0).
__global__ void batch_adj_rk3(const double* __restrict__ ybar, double* an, double* ax, int64_t ntot, const Inst* inst,
                              const double* __restrict__ dt, int ninst) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    const bool act = dt[i] > 0.0;
    for (int64_t c = threadIdx.x; c < inst[i].n; c += blockDim.x)
        for (int k = 0; k < 5; k++) {
            const int64_t g = k * ntot + inst[i].off + NG + c;
            const double y = ybar[g];
            an[g] = act ? (1.0 / 3.0) * y : y;
            ax[g] = act ? (2.0 / 3.0) * y : 0.0;
        }
}
// Reverse of stage 2 (U² = ¾Uⁿ + ¼(U¹ + dt·R)): ān += ¾x̄, ȳ₁ = ¼x̄.
__global__ void batch_adj_rk2(const double* __restrict__ ax, double* ay, double* an, int64_t ntot, const Inst* inst,
                              int ninst) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    for (int64_t c = threadIdx.x; c < inst[i].n; c += blockDim.x)
        for (int k = 0; k < 5; k++) {
            const int64_t g = k * ntot + inst[i].off + NG + c;
            an[g] = an[g] + 0.75 * ax[g];
            ay[g] = 0.25 * ax[g];
        }
}
// Reverse of stage 1 (U¹ = Uⁿ + dt·R), direct part: ān += ȳ₁.
__global__ void batch_adj_rk1(const double* __restrict__ ay, double* an, int64_t ntot, const Inst* inst, int ninst) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    for (int64_t c = threadIdx.x; c < inst[i].n; c += blockDim.x)
        for (int k = 0; k < 5; k++) {
            const int64_t g = k * ntot + inst[i].off + NG + c;
            an[g] = an[g] + ay[g];
        }
}

// Reverse of batch_ghosts: each ghost's cotangent moves to its source cell
// (normal momentum negated for reflecting walls, dropped for Dirichlet).
__global__ void batch_adj_ghosts(double* xb, int64_t ntot, const Inst* inst, int ninst, int kind_lo, int kind_hi) {
    // one thread per (instance, field): the ghost cotangents of both sides are
    // loaded together and cleared, then each side adds them into its source
    // cells (an outflow side sums its layers first; periodic and reflecting
    // sources of one side are distinct cells when n >= NG); the sides go one
    // after the other, as their sources may coincide on a short line
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ninst * 5) return;
    const int i = t / 5, k = t % 5;
    const int64_t n = inst[i].n;
    double* x = xb + k * ntot + inst[i].off;
    double g[2][NG];
#pragma unroll
    for (int gi = 0; gi < NG; gi++) {
        g[0][gi] = x[gi];
        g[1][gi] = x[n + NG + gi];
    }
#pragma unroll
    for (int gi = 0; gi < NG; gi++) {
        x[gi] = 0.0;
        x[n + NG + gi] = 0.0;
    }
    for (int side = 0; side < 2; side++) {
        const int kind = side ? kind_hi : kind_lo;
        auto src = [&](int gi) -> int64_t {
            if (kind == EMG_BC_PERIODIC) return side ? NG + gi : n + gi;
            if (kind == EMG_BC_OUTFLOW) return side ? n + NG - 1 : NG;
            if (kind == EMG_BC_REFLECT) return side ? n + NG - 1 - gi : 2 * NG - 1 - gi;
            return -1;
        };
        const double sg = (kind == EMG_BC_REFLECT && k == 1) ? -1.0 : 1.0;
        if (kind == EMG_BC_OUTFLOW) {
            double acc = 0.0;
#pragma unroll
            for (int gi = 0; gi < NG; gi++) acc += g[side][gi];
            x[src(0)] += acc;
        } else if ((kind == EMG_BC_PERIODIC || kind == EMG_BC_REFLECT) && n >= NG) {
            double sv[NG];
#pragma unroll
            for (int gi = 0; gi < NG; gi++) sv[gi] = x[src(gi)];
#pragma unroll
            for (int gi = 0; gi < NG; gi++) x[src(gi)] = sv[gi] + sg * g[side][gi];
        } else if (kind == EMG_BC_PERIODIC || kind == EMG_BC_REFLECT) {
            for (int gi = 0; gi < NG; gi++) x[src(gi)] += sg * g[side][gi];
        }
    }
}

// Per-instance box objective over cells with centre (c+½)·dx in [xlo, xhi]:
// kind 0 = Σ p·dx, kind 1 = Σ E·dx; writes ∂J/∂U and J per instance.
__global__ void batch_objective(const double* __restrict__ u, double* abar, int64_t ntot, const Inst* inst, int ninst,
                                int kind, double xlo, double xhi, EosD eosd, double* J) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    __shared__ double sj[32];
    const Eos<double> e = Eos<double>::from(eosd);
    const double dx = inst[i].dx;
    double acc = 0.0, gdummy = 0.0;
    for (int64_t c = threadIdx.x; c < inst[i].n; c += blockDim.x) {
        const int64_t g = inst[i].off + NG + c;
        const double x = ((double)c + 0.5) * dx;
        double ub[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        if (x >= xlo && x <= xhi) {
            double q[5], w[5];
            for (int k = 0; k < 5; k++) q[k] = u[k * ntot + g];
            if (kind == 0) {
                to_prim(e, q, w);
                acc += w[4] * dx;
                const double wb[5] = {0.0, 0.0, 0.0, 0.0, dx};
                adj::to_prim_vjp(e, q, wb, ub, gdummy);
            } else {
                acc += q[4] * dx;
                ub[4] = dx;
            }
        }
        for (int k = 0; k < 5; k++) abar[k * ntot + g] = ub[k];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sj[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) a += sj[w];
        J[i] = a;
    }
}

// Initial primitive cotangent w̄ = (∂U/∂w)ᵀŪ per cell (optional AoS output)
// and its sums over the cells left / right of x_split: per instance
// [ρ_L, u_L, p_L, ρ_R, u_R, p_R].
__global__ void batch_grad6(const double* __restrict__ u0, const double* __restrict__ abar, int64_t ntot, const Inst* inst,
                            int ninst, const int64_t* __restrict__ coff, double xsplit, EosD eosd, double* wbar_aos,
                            double* grad6) {
    const int i = blockIdx.x;
    if (i >= ninst) return;
    __shared__ double sg[6][32];
    const Eos<double> e = Eos<double>::from(eosd);
    double acc[6] = {0, 0, 0, 0, 0, 0}, gdummy = 0.0;
    for (int64_t c = threadIdx.x; c < inst[i].n; c += blockDim.x) {
        const int64_t g = inst[i].off + NG + c;
        double q[5], qb[5], w[5], wb[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (int k = 0; k < 5; k++) {
            q[k] = u0[k * ntot + g];
            qb[k] = abar[k * ntot + g];
        }
        to_prim(e, q, w);
        adj::to_cons_vjp(e, w, qb, wb, gdummy);
        if (wbar_aos)
            for (int k = 0; k < 5; k++) wbar_aos[(coff[i] + c) * 5 + k] = wb[k];
        const int side = ((double)c + 0.5) * inst[i].dx < xsplit ? 0 : 3;
        acc[side] += wb[0];
        acc[side + 1] += wb[1];
        acc[side + 2] += wb[4];
    }
    for (int q = 0; q < 6; q++) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sg[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += sg[threadIdx.x][w];
        grad6[6 * i + threadIdx.x] = v;
    }
}

}  // namespace

struct emg_batch1d {
    int device = 0;
    cudaStream_t stream = nullptr;
    emg_eos eos{};
    emg_opts opts{};
    emg_bc bc[2]{};
    int ninst = 0;
    int64_t ntot = 0, ncells = 0;
    std::vector<Inst> hinst;
    std::vector<int64_t> coff;
    Inst* inst = nullptr;
    double* dtv = nullptr;
    double* dxv = nullptr;
    int64_t* dcoff = nullptr;
    BatchSeg* segs = nullptr;
    int nseg = 0;
    double *u = nullptr, *sa = nullptr, *sb = nullptr, *state = nullptr;
    double* dstate = nullptr;  // Dirichlet states
    int* active = nullptr;
    StepCtl* ctl = nullptr;
    // ---- discrete adjoint of a recorded FP64 run
    double* u0 = nullptr;          // initial state (padded SoA)
    double* ufin = nullptr;        // final state of the recorded run
    double* theta_rec[3]{};        // when set, the stages record the limiter's blend weights
    uint64_t rec_B = 0, rec_K = 0; // batch steps recorded, checkpoint interval
    double* rec_dt = nullptr;      // per batch step the time step of every instance
    uint64_t rec_cap = 0;
    std::vector<double*> ckpt;     // batch state before batch steps 0, K, 2K, ...
    double* seg = nullptr;         // stage inputs and blend weights of up to K batch steps
    uint64_t seg_cap = 0;
    double *a_next = nullptr, *a_n = nullptr, *a_x = nullptr, *a_y = nullptr;
    AdjLane* lanes = nullptr;
    int nlanes = 0;
    bool recorded = false, seeded = false;
    double adj_ms[3]{};            // device ms: recorded forward, checkpoint recompute, reverse

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        for (double* b : {u0, ufin, rec_dt, seg, a_next, a_n, a_x, a_y})
            if (b) cudaFree(b);
        for (double* c : ckpt) cudaFree(c);
        if (lanes) cudaFree(lanes);
        cudaFree(inst);
        cudaFree(dtv);
        cudaFree(dxv);
        cudaFree(dcoff);
        cudaFree(segs);
        cudaFree(u);
        cudaFree(sa);
        cudaFree(sb);
        cudaFree(dstate);
        cudaFree(active);
        cudaFree(ctl);
        if (stream) cudaStreamDestroy(stream);
    }

    int stage(int s) {
        double* in = s == 1 ? u : (s == 2 ? sa : sb);
        batch_ghosts<<<ninst, 32, 0, stream>>>(in, ntot, inst, ninst, bc[0].kind, bc[1].kind,
                                                EosD{eos.gamma, eos.p_inf, eos.b, eos.q}, dstate, dstate + 5);
        B_CUDA(cudaGetLastError());
        SweepParams p{};
        p.uin = in;
        p.ctl = ctl;
        p.ncell = ntot;
        p.sd = 1;
        p.sl = 0;
        p.so = 0;
        p.nd = SEG;
        p.nl = 1;
        p.no = 1;
        p.d = 0;
        p.seg = SEG;
        p.first = 1;
        p.last = 1;
        p.stage = s;
        p.rows_contig = 1;
        p.ndim = 1.0;
        p.positivity = opts.positivity ? 1 : 0;
        p.tol = opts.tol;
        p.eos = EosD{eos.gamma, eos.p_inf, eos.b, eos.q};
        p.dx = 1.0;
        p.lw = 32;
        p.segs = segs;
        p.nseg = nseg;
        p.inst_dx = dxv;
        p.inst_dt = dtv;
        p.theta_rec = theta_rec[s - 1];
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
        const dim3 grid((unsigned)((nseg + 31) / 32), 1, 1);
        cudaError_t e = opts.precision == EMG_PRECISION_MIXED      ? sweep_launch_batch_mixed(opts.mode, p, grid, stream)
                        : opts.precision == EMG_PRECISION_F64_FAST ? sweep_launch_batch_fast(opts.mode, p, grid, stream)
                                                                   : sweep_launch_batch_f64(opts.mode, p, grid, stream);
        if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("batch sweep: ") + cudaGetErrorString(e));
        return EMG_OK;
    }

    // ---- discrete adjoint
    size_t state_bytes() const { return (size_t)ntot * 5 * sizeof(double); }
    size_t step_doubles() const { return (size_t)ntot * 18; }  // 3 stage inputs + 3 blend-weight arrays
    double* seg_x(uint64_t slot, int stage) { return seg + slot * step_doubles() + (size_t)(stage - 1) * 5 * ntot; }
    double* seg_theta(uint64_t slot, int stage) { return seg + slot * step_doubles() + (size_t)(15 + stage - 1) * ntot; }

    int ensure_adjoint_buffers() {
        if (a_next) return EMG_OK;
        for (double** b : {&a_next, &a_n, &a_x, &a_y, &ufin}) B_CUDA(cudaMalloc(b, state_bytes()));
        // lanes: segments of ADJ_L owned rows over rows [NG − 5, NG + n + 5) of every instance
        std::vector<AdjLane> ln;
        for (int i = 0; i < ninst; i++)
            for (int c0 = NG - 5; c0 < NG + hinst[i].n + 5; c0 += ADJ_L) {
                AdjLane a{};
                a.base = hinst[i].off;
                a.n = (int)hinst[i].n;
                a.c0 = c0;
                a.inst = i;
                ln.push_back(a);
            }
        nlanes = (int)ln.size();
        B_CUDA(cudaMalloc(&lanes, ln.size() * sizeof(AdjLane)));
        B_CUDA(cudaMemcpyAsync(lanes, ln.data(), ln.size() * sizeof(AdjLane), cudaMemcpyHostToDevice, stream));
        return EMG_OK;
    }

    // a recorded batch step b (slot s): stage inputs and blend weights
    int record_step(uint64_t b, uint64_t slot) {
        const double* dtb = rec_dt + b * ninst;
        batch_set_done<<<(ninst + 255) / 256, 256, 0, stream>>>(inst, dtb, ninst);
        B_CUDA(cudaMemcpyAsync(dtv, dtb, ninst * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        B_CUDA(cudaMemcpyAsync(seg_x(slot, 1), u, state_bytes(), cudaMemcpyDeviceToDevice, stream));
        for (int st = 1; st <= 3; st++) theta_rec[st - 1] = seg_theta(slot, st);
        int rc = EMG_OK;
        for (int st = 1; st <= 3 && !rc; st++) rc = stage(st);
        for (auto& t : theta_rec) t = nullptr;
        if (rc) return rc;
        B_CUDA(cudaMemcpyAsync(seg_x(slot, 2), sa, state_bytes(), cudaMemcpyDeviceToDevice, stream));
        B_CUDA(cudaMemcpyAsync(seg_x(slot, 3), sb, state_bytes(), cudaMemcpyDeviceToDevice, stream));
        return EMG_OK;
    }

    int adj_sweep(const double* X, const double* theta, const double* ybar, double beta, double* xbar,
                  const double* dtb) {
        AdjSweepParams p{};
        p.u = X;
        p.theta = opts.positivity ? theta : nullptr;
        p.ybar = ybar;
        p.xbar = xbar;
        p.gpart = nullptr;
        p.ncell = ntot;
        p.sd = 1;
        p.ng = NG;
        p.eos = EosD{eos.gamma, eos.p_inf, eos.b, eos.q};
        p.lanes = lanes;
        p.nlanes = nlanes;
        p.inst_dx = dxv;
        p.inst_dt = dtb;
        p.beta = beta;
        cudaError_t e = adj_sweep_launch_batch(p, stream);
        if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("batch adjoint sweep: ") + cudaGetErrorString(e));
        return EMG_OK;
    }

    // reverse of batch step b (slot s): a_next = Ūⁿ⁺¹ in, Ūⁿ out
    int reverse_step(uint64_t b, uint64_t slot) {
        const double* dtb = rec_dt + b * ninst;
        const int kl = bc[0].kind, kh = bc[1].kind;
        const int gg5 = (ninst * 5 + 127) / 128;  // reverse ghost fill: one thread per (instance, field)
        for (double* x : {a_n, a_x, a_y}) B_CUDA(cudaMemsetAsync(x, 0, state_bytes(), stream));
        batch_adj_rk3<<<ninst, 256, 0, stream>>>(a_next, a_n, a_x, ntot, inst, dtb, ninst);
        int rc = adj_sweep(seg_x(slot, 3), seg_theta(slot, 3), a_next, 2.0 / 3.0, a_x, dtb);
        if (rc) return rc;
        batch_adj_ghosts<<<gg5, 128, 0, stream>>>(a_x, ntot, inst, ninst, kl, kh);
        batch_adj_rk2<<<ninst, 256, 0, stream>>>(a_x, a_y, a_n, ntot, inst, ninst);
        if ((rc = adj_sweep(seg_x(slot, 2), seg_theta(slot, 2), a_x, 0.25, a_y, dtb))) return rc;
        batch_adj_ghosts<<<gg5, 128, 0, stream>>>(a_y, ntot, inst, ninst, kl, kh);
        batch_adj_rk1<<<ninst, 256, 0, stream>>>(a_y, a_n, ntot, inst, ninst);
        // the slot holds Uⁿ as it was before its ghost fill
        batch_set_done<<<(ninst + 255) / 256, 256, 0, stream>>>(inst, dtb, ninst);
        batch_ghosts<<<ninst, 32, 0, stream>>>(seg_x(slot, 1), ntot, inst, ninst, kl, kh,
                                                EosD{eos.gamma, eos.p_inf, eos.b, eos.q}, dstate, dstate + 5);
        if ((rc = adj_sweep(seg_x(slot, 1), seg_theta(slot, 1), a_y, 1.0, a_n, dtb))) return rc;
        batch_adj_ghosts<<<gg5, 128, 0, stream>>>(a_n, ntot, inst, ninst, kl, kh);
        B_CUDA(cudaGetLastError());
        std::swap(a_next, a_n);
        return EMG_OK;
    }
};

extern "C" {

int emg_batch1d_create(const emg_eos* eos, const emg_opts* opts, const emg_bc bc[2], size_t ninst, const int64_t* n,
                       const double* dx, const double* u, emg_batch1d** out) {
    if (!eos || !opts || !bc || !n || !dx || !u || !out || ninst == 0) return set_error(EMG_ERR_INVALID, "null argument");
    *out = nullptr;
    for (int s = 0; s < 2; s++)
        if (bc[s].kind < 0 || bc[s].kind > 3)
            return set_error(EMG_ERR_INVALID, "batched lines support periodic, outflow, reflect and Dirichlet boundaries");
    if ((bc[0].kind == EMG_BC_PERIODIC) != (bc[1].kind == EMG_BC_PERIODIC))
        return set_error(EMG_ERR_INVALID, "periodic boundaries must be paired");
    if (opts->mode < 0 || opts->mode > 2 || opts->precision < 0 || opts->precision > 2)
        return set_error(EMG_ERR_INVALID, "unknown mode or precision");
    for (size_t i = 0; i < ninst; i++) {
        if (n[i] < 2) return set_error(EMG_ERR_INVALID, "every instance needs at least 2 cells");
        if (n[i] < NG && (bc[0].kind == EMG_BC_REFLECT || bc[1].kind == EMG_BC_REFLECT))
            return set_error(EMG_ERR_INVALID, "reflecting instances need at least 6 cells");
        if (!(dx[i] > 0.0)) return set_error(EMG_ERR_INVALID, "dx must be > 0");
    }
    {
        int cnt = 0;
        if (cudaGetDeviceCount(&cnt) != cudaSuccess || cnt == 0) {
            cudaGetLastError();
            return set_error(EMG_ERR_NO_DEVICE, "no CUDA device visible");
        }
    }
    emg_batch1d* h = new emg_batch1d();
    auto bail = [&](int rc) {
        h->release();
        delete h;
        return rc;
    };
    h->eos = *eos;
    h->opts = *opts;
    h->bc[0] = bc[0];
    h->bc[1] = bc[1];
    h->ninst = (int)ninst;
    cudaGetDevice(&h->device);
    std::vector<BatchSeg> segs;
    int64_t off = 0, coff = 0;
    for (size_t i = 0; i < ninst; i++) {
        Inst I{};
        I.off = off;
        I.n = n[i];
        I.dx = dx[i];
        h->hinst.push_back(I);
        h->coff.push_back(coff);
        for (int64_t s0 = 0; s0 < n[i]; s0 += SEG) {
            BatchSeg sg{};
            sg.base = off + (NG - 5) + s0;
            sg.len = (int)std::min<int64_t>(SEG, n[i] - s0);
            sg.inst = (int)i;
            sg.tail = s0 + SEG >= n[i];
            segs.push_back(sg);
        }
        off += n[i] + 2 * NG;
        coff += n[i];
    }
    h->ntot = off;
    h->ncells = coff;
    h->nseg = (int)segs.size();
    std::vector<double> dxs(dx, dx + ninst);
    const size_t bytes = (size_t)h->ntot * 5 * sizeof(double);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->inst, ninst * sizeof(Inst)) != cudaSuccess || cudaMalloc(&h->dtv, ninst * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->dxv, ninst * sizeof(double)) != cudaSuccess || cudaMalloc(&h->dcoff, ninst * sizeof(int64_t)) != cudaSuccess ||
        cudaMalloc(&h->segs, segs.size() * sizeof(BatchSeg)) != cudaSuccess || cudaMalloc(&h->u, bytes) != cudaSuccess ||
        cudaMalloc(&h->sa, bytes) != cudaSuccess || cudaMalloc(&h->sb, bytes) != cudaSuccess ||
        cudaMalloc(&h->dstate, 10 * sizeof(double)) != cudaSuccess || cudaMalloc(&h->active, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&h->ctl, sizeof(StepCtl)) != cudaSuccess || cudaMalloc(&h->state, (size_t)h->ncells * 5 * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return bail(set_error(EMG_ERR_CUDA, "device allocation failed"));
    }
    if (sweep_prepare_device() != cudaSuccess) return bail(set_error(EMG_ERR_CUDA, "sweep setup failed"));
    StepCtl c{};
    c.dt = 1.0;  // the batched sweep reads per-instance dt; the control block only gates it
    double st[10];
    for (int s = 0; s < 2; s++)
        for (int k = 0; k < 5; k++) st[5 * s + k] = bc[s].state[k];
    cudaMemsetAsync(h->u, 0, bytes, h->stream);
    cudaMemsetAsync(h->sa, 0, bytes, h->stream);
    cudaMemsetAsync(h->sb, 0, bytes, h->stream);
    cudaMemcpyAsync(h->ctl, &c, sizeof c, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->dstate, st, sizeof st, cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->inst, h->hinst.data(), ninst * sizeof(Inst), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->dxv, dxs.data(), ninst * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->dcoff, h->coff.data(), ninst * sizeof(int64_t), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->segs, segs.data(), segs.size() * sizeof(BatchSeg), cudaMemcpyHostToDevice, h->stream);
    cudaMemcpyAsync(h->state, u, (size_t)h->ncells * 5 * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    batch_pack<<<h->ninst, 256, 0, h->stream>>>(h->state, h->u, h->ntot, h->inst, h->ninst, h->dcoff);
    if (cudaMalloc(&h->u0, bytes) != cudaSuccess) {
        cudaGetLastError();
        return bail(set_error(EMG_ERR_CUDA, "device allocation failed"));
    }
    cudaMemcpyAsync(h->u0, h->u, bytes, cudaMemcpyDeviceToDevice, h->stream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess)
        return bail(set_error(EMG_ERR_CUDA, "upload failed"));
    *out = h;
    return EMG_OK;
}

int emg_batch1d_destroy(emg_batch1d* h) {
    if (!h) return EMG_OK;
    h->release();
    delete h;
    return EMG_OK;
}

int emg_batch1d_run_to(emg_batch1d* h, double t_end, uint64_t* launched) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    if (!std::isfinite(t_end)) return set_error(EMG_ERR_INVALID, "t_end must be finite");
    cudaSetDevice(h->device);
    uint64_t issued = 0;
    const EosD e{h->eos.gamma, h->eos.p_inf, h->eos.b, h->eos.q};
    // reopen instances for the new t_end
    std::vector<Inst> hi(h->ninst);
    B_CUDA(cudaMemcpyAsync(hi.data(), h->inst, h->ninst * sizeof(Inst), cudaMemcpyDeviceToHost, h->stream));
    B_CUDA(cudaStreamSynchronize(h->stream));
    for (auto& I : hi) {
        I.done = 0;
        I.status = 0;
    }
    B_CUDA(cudaMemcpyAsync(h->inst, hi.data(), h->ninst * sizeof(Inst), cudaMemcpyHostToDevice, h->stream));
    for (;;) {
        // a batch of steps between checks on the host
        for (int k = 0; k < 16; k++) {
            batch_begin<<<h->ninst, 256, 0, h->stream>>>(h->u, h->ntot, h->inst, h->dtv, h->ninst, h->opts.cfl, t_end, e);
            for (int s = 1; s <= 3; s++) {
                int rc = h->stage(s);
                if (rc) return rc;
            }
            batch_end<<<(h->ninst + 255) / 256, 256, 0, h->stream>>>(h->inst, h->ninst, h->active);
            B_CUDA(cudaGetLastError());
        }
        issued += 16;
        int act = 0;
        B_CUDA(cudaMemcpyAsync(&act, h->active, sizeof act, cudaMemcpyDeviceToHost, h->stream));
        B_CUDA(cudaMemsetAsync(h->active, 0, sizeof(int), h->stream));
        B_CUDA(cudaStreamSynchronize(h->stream));
        if (act == 0) break;
        if (issued > 100000000ull) return set_error(EMG_ERR_DT_COLLAPSED, "run did not terminate");
    }
    B_CUDA(cudaMemcpyAsync(hi.data(), h->inst, h->ninst * sizeof(Inst), cudaMemcpyDeviceToHost, h->stream));
    B_CUDA(cudaStreamSynchronize(h->stream));
    uint64_t mx = 0;
    for (auto& I : hi) {
        if (I.status) return set_error(I.status, "time step collapsed in an instance");
        mx = std::max<uint64_t>(mx, I.steps);
    }
    if (BOUNDS_CHECK) {
        StepCtl c;
        B_CUDA(cudaMemcpy(&c, h->ctl, sizeof c, cudaMemcpyDeviceToHost));
        if (c.status == EMG_ERR_BOUNDS) return set_error(EMG_ERR_BOUNDS, "device index out of range (bounds-check build)");
    }
    if (launched) *launched = mx;
    return EMG_OK;
}

int emg_batch1d_download(emg_batch1d* h, double* u) {
    if (!h || !u) return set_error(EMG_ERR_INVALID, "null argument");
    cudaSetDevice(h->device);
    batch_unpack<<<h->ninst, 256, 0, h->stream>>>(h->u, h->state, h->ntot, h->inst, h->ninst, h->dcoff);
    B_CUDA(cudaGetLastError());
    B_CUDA(cudaMemcpyAsync(u, h->state, (size_t)h->ncells * 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    B_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_batch1d_status(emg_batch1d* h, double* t, uint64_t* steps) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    std::vector<Inst> hi(h->ninst);
    B_CUDA(cudaMemcpyAsync(hi.data(), h->inst, h->ninst * sizeof(Inst), cudaMemcpyDeviceToHost, h->stream));
    B_CUDA(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < h->ninst; i++) {
        if (t) t[i] = hi[i].t;
        if (steps) steps[i] = hi[i].steps;
    }
    return EMG_OK;
}

int emg_batch1d_stream(emg_batch1d* h, void** stream) {
    if (!h || !stream) return set_error(EMG_ERR_INVALID, "null argument");
    *stream = (void*)h->stream;
    return EMG_OK;
}

int emg_batch1d_record(emg_batch1d* h, double t_end, uint64_t checkpoint_every, uint64_t* batch_steps) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    if (!std::isfinite(t_end)) return set_error(EMG_ERR_INVALID, "t_end must be finite");
    if (h->opts.mode != EMG_MODE_WENO) return set_error(EMG_ERR_INVALID, "the adjoint supports the WENO flux mode");
    for (int s = 0; s < 2; s++)
        if (h->bc[s].kind == EMG_BC_PERIODIC)
            for (auto& I : h->hinst)
                if (I.n < NG) return set_error(EMG_ERR_INVALID, "periodic adjoint instances need at least 6 cells");
    cudaSetDevice(h->device);
    int rc = h->ensure_adjoint_buffers();
    if (rc) return rc;
    const uint64_t K = checkpoint_every ? checkpoint_every : 64;
    const EosD e{h->eos.gamma, h->eos.p_inf, h->eos.b, h->eos.q};
    // restart every instance from the initial state at t = 0
    B_CUDA(cudaMemcpyAsync(h->u, h->u0, h->state_bytes(), cudaMemcpyDeviceToDevice, h->stream));
    std::vector<Inst> hi = h->hinst;
    for (auto& I : hi) {
        I.t = 0.0;
        I.steps = 0;
        I.done = 0;
        I.status = 0;
    }
    B_CUDA(cudaMemcpyAsync(h->inst, hi.data(), h->ninst * sizeof(Inst), cudaMemcpyHostToDevice, h->stream));
    B_CUDA(cudaMemsetAsync(h->active, 0, sizeof(int), h->stream));
    cudaEvent_t ea, eb;
    cudaEventCreate(&ea);
    cudaEventCreate(&eb);
    cudaEventRecord(ea, h->stream);
    uint64_t b = 0;
    for (;;) {
        for (int k = 0; k < 16; k++, b++) {
            if (b + 1 > h->rec_cap) {
                // grow the time-step record (doubling), keeping what is there
                const uint64_t cap = std::max<uint64_t>(1024, 2 * h->rec_cap);
                double* nr = nullptr;
                B_CUDA(cudaMalloc(&nr, cap * h->ninst * sizeof(double)));
                if (h->rec_dt) {
                    B_CUDA(cudaMemcpyAsync(nr, h->rec_dt, h->rec_cap * h->ninst * sizeof(double), cudaMemcpyDeviceToDevice,
                                           h->stream));
                    B_CUDA(cudaStreamSynchronize(h->stream));
                    cudaFree(h->rec_dt);
                }
                h->rec_dt = nr;
                h->rec_cap = cap;
            }
            if (b % K == 0) {
                if (h->ckpt.size() <= b / K) {
                    double* c = nullptr;
                    B_CUDA(cudaMalloc(&c, h->state_bytes()));
                    h->ckpt.push_back(c);
                }
                B_CUDA(cudaMemcpyAsync(h->ckpt[b / K], h->u, h->state_bytes(), cudaMemcpyDeviceToDevice, h->stream));
            }
            batch_begin<<<h->ninst, 256, 0, h->stream>>>(h->u, h->ntot, h->inst, h->dtv, h->ninst, h->opts.cfl, t_end, e);
            B_CUDA(cudaMemcpyAsync(h->rec_dt + b * h->ninst, h->dtv, h->ninst * sizeof(double), cudaMemcpyDeviceToDevice,
                                   h->stream));
            for (int st = 1; st <= 3; st++)
                if ((rc = h->stage(st))) return rc;
            batch_end<<<(h->ninst + 255) / 256, 256, 0, h->stream>>>(h->inst, h->ninst, h->active);
            B_CUDA(cudaGetLastError());
        }
        int act = 0;
        B_CUDA(cudaMemcpyAsync(&act, h->active, sizeof act, cudaMemcpyDeviceToHost, h->stream));
        B_CUDA(cudaMemsetAsync(h->active, 0, sizeof(int), h->stream));
        B_CUDA(cudaStreamSynchronize(h->stream));
        if (act == 0) break;
        if (b > 100000000ull) return set_error(EMG_ERR_DT_COLLAPSED, "run did not terminate");
    }
    cudaEventRecord(eb, h->stream);
    B_CUDA(cudaMemcpyAsync(hi.data(), h->inst, h->ninst * sizeof(Inst), cudaMemcpyDeviceToHost, h->stream));
    B_CUDA(cudaStreamSynchronize(h->stream));
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ea, eb);
    cudaEventDestroy(ea);
    cudaEventDestroy(eb);
    h->adj_ms[0] = ms;
    uint64_t B = 0;
    for (auto& I : hi) {
        if (I.status) return set_error(I.status, "time step collapsed in an instance");
        B = std::max<uint64_t>(B, I.steps);  // an instance steps in every batch step until it is done
    }
    B_CUDA(cudaMemcpyAsync(h->ufin, h->u, h->state_bytes(), cudaMemcpyDeviceToDevice, h->stream));
    B_CUDA(cudaStreamSynchronize(h->stream));
    h->rec_B = B;
    h->rec_K = K;
    h->recorded = B > 0;
    h->seeded = false;
    if (batch_steps) *batch_steps = B;
    return EMG_OK;
}

int emg_batch1d_objective(emg_batch1d* h, int kind, double x_lo, double x_hi, double* J) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    if (!h->recorded) return set_error(EMG_ERR_INVALID, "no recorded run (emg_batch1d_record)");
    if (kind != EMG_OBJ_PRESSURE && kind != EMG_OBJ_ENERGY) return set_error(EMG_ERR_INVALID, "unknown objective");
    cudaSetDevice(h->device);
    double* dJ = nullptr;
    B_CUDA(cudaMalloc(&dJ, h->ninst * sizeof(double)));
    B_CUDA(cudaMemsetAsync(h->a_next, 0, h->state_bytes(), h->stream));
    batch_objective<<<h->ninst, 256, 0, h->stream>>>(h->ufin, h->a_next, h->ntot, h->inst, h->ninst, kind, x_lo, x_hi,
                                                      EosD{h->eos.gamma, h->eos.p_inf, h->eos.b, h->eos.q}, dJ);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess && J)
        err = cudaMemcpyAsync(J, dJ, h->ninst * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
    cudaFree(dJ);
    if (err != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("batch objective: ") + cudaGetErrorString(err));
    h->seeded = true;
    return EMG_OK;
}

int emg_batch1d_backward(emg_batch1d* h, double x_split, double* grad6, double* wbar) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    if (!h->recorded) return set_error(EMG_ERR_INVALID, "no recorded run (emg_batch1d_record)");
    if (!h->seeded) return set_error(EMG_ERR_INVALID, "no cotangent seeded (emg_batch1d_objective)");
    cudaSetDevice(h->device);
    const uint64_t K = h->rec_K, B = h->rec_B;
    if (K > h->seg_cap) {
        if (h->seg) cudaFree(h->seg);
        h->seg = nullptr;
        h->seg_cap = 0;
        B_CUDA(cudaMalloc(&h->seg, K * h->step_doubles() * sizeof(double)));
        h->seg_cap = K;
    }
    const uint64_t nseg = (B + K - 1) / K;
    std::vector<cudaEvent_t> ev(3 * nseg);
    for (auto& x : ev) cudaEventCreate(&x);
    for (uint64_t sg = nseg; sg-- > 0;) {
        const uint64_t b0 = sg * K, b1 = std::min(b0 + K, B);
        cudaEventRecord(ev[3 * sg], h->stream);
        B_CUDA(cudaMemcpyAsync(h->u, h->ckpt[sg], h->state_bytes(), cudaMemcpyDeviceToDevice, h->stream));
        for (uint64_t b = b0; b < b1; b++) {
            int rc = h->record_step(b, b - b0);
            if (rc) return rc;
        }
        cudaEventRecord(ev[3 * sg + 1], h->stream);
        for (uint64_t b = b1; b-- > b0;) {
            int rc = h->reverse_step(b, b - b0);
            if (rc) return rc;
        }
        cudaEventRecord(ev[3 * sg + 2], h->stream);
    }
    double* dg = nullptr;
    double* dw = nullptr;
    B_CUDA(cudaMalloc(&dg, (size_t)h->ninst * 6 * sizeof(double)));
    if (wbar) B_CUDA(cudaMalloc(&dw, (size_t)h->ncells * 5 * sizeof(double)));
    batch_grad6<<<h->ninst, 256, 0, h->stream>>>(h->u0, h->a_next, h->ntot, h->inst, h->ninst, h->dcoff, x_split,
                                                  EosD{h->eos.gamma, h->eos.p_inf, h->eos.b, h->eos.q}, dw, dg);
    cudaError_t err = cudaGetLastError();
    if (err == cudaSuccess && grad6)
        err = cudaMemcpyAsync(grad6, dg, (size_t)h->ninst * 6 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (err == cudaSuccess && wbar)
        err = cudaMemcpyAsync(wbar, dw, (size_t)h->ncells * 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    // the batch state is back at the recorded run's end
    if (err == cudaSuccess) err = cudaMemcpyAsync(h->u, h->ufin, h->state_bytes(), cudaMemcpyDeviceToDevice, h->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(h->stream);
    cudaFree(dg);
    if (dw) cudaFree(dw);
    if (err != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("batch backward: ") + cudaGetErrorString(err));
    h->adj_ms[1] = h->adj_ms[2] = 0.0;
    for (uint64_t sg = 0; sg < nseg; sg++) {
        float a = 0.0f, c = 0.0f;
        cudaEventElapsedTime(&a, ev[3 * sg], ev[3 * sg + 1]);
        cudaEventElapsedTime(&c, ev[3 * sg + 1], ev[3 * sg + 2]);
        h->adj_ms[1] += a;
        h->adj_ms[2] += c;
    }
    for (auto& x : ev) cudaEventDestroy(x);
    h->seeded = false;
    return EMG_OK;
}

int emg_batch1d_adjoint_times(emg_batch1d* h, double ms[3]) {
    if (!h || !ms) return set_error(EMG_ERR_INVALID, "null argument");
    for (int k = 0; k < 3; k++) ms[k] = h->adj_ms[k];
    return EMG_OK;
}

}  // extern "C"
