// Batched independent 1-D lines (emg_batch1d_*): thousands of Riemann
// problems of different lengths advanced together. Each RK stage is one ghost
// launch and one fused-sweep launch over the segments of all instances
// (sweep.cuh, KIND_BATCH); each instance keeps its own time, CFL time step
// (C/solver.rs:478-523) and stopping rule (C/solver.rs:758-768) on the
// device, so a whole run needs no host round trip per step.
//
// Built with -fmad=false.
#include "../../include/emergence_b200.h"
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
constexpr int SEG = 64;

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

    void release() {
        if (stream) cudaStreamSynchronize(stream);
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
        cudaError_t e = opts.precision == EMG_PRECISION_MIXED ? sweep_launch_batch_mixed(opts.mode, p, grid, stream)
                                                               : sweep_launch_batch_f64(opts.mode, p, grid, stream);
        if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("batch sweep: ") + cudaGetErrorString(e));
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
    if (opts->mode < 0 || opts->mode > 2 || (opts->precision != 0 && opts->precision != 1))
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
    static bool prepared = false;
    if (!prepared) {
        cudaError_t e = sweep_prepare_f64();
        if (e == cudaSuccess) e = sweep_prepare_mixed();
        if (e != cudaSuccess) return bail(set_error(EMG_ERR_CUDA, "sweep setup failed"));
        prepared = true;
    }
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

}  // extern "C"
