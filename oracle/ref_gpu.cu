// Same-box GPU baseline: measurement infrastructure, not the product.
//
// The reference's own CUDA kernels of the uniform solver
// (fluid/crates/compressible-cuda/src/kernels.cu, included unmodified from
// where it lies; the reference compiles it at run time with NVRTC for sm_86)
// built by nvcc for sm_100a and launched in the order of GpuSolver<f64> for
// the Euler system (fluid/crates/compressible-cuda/src/lib.rs:186-447):
//
//   step(dt):  u0 ← u; 3 × [ghost per active axis (lib.rs:274-304), prim
//              (:306-315), then per active axis theta, midflux (not in
//              Central mode), flux, accum (:317-379); rk (:381-388)] with
//              (α, β) = (0, 1), (¾, ¼), (⅓, ⅔) (:391-401)
//   dt_cfl():  ghost, prim, rate over 256 blocks of 256 threads, a host max
//              over the 2·256 block results, dt = cfl / r1 (:404-432)
//
// Every other launch is 1-D with 128 threads per block (`cfg`, lib.rs:151-153).
// The scratch arrays (w, TH, MF, MU, F, UF, rhs) are sized as in from_cpu
// (lib.rs:186-239). oracle/Makefile builds this file into oracle/_ref/ (target
// `refgpu`); only bench.py's reference-GPU leg loads the result.
#include REF_KERNELS_CU

#include "../include/emergence_b200.h"

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

namespace {

constexpr int BLOCK = 128;        // lib.rs:22
constexpr int RATE_BLOCKS = 256;  // lib.rs:23
constexpr int NV_MAX = 7;         // FiveEq (Euler: 5)

thread_local std::string g_err;

int fail(const std::string& m) {
    g_err = m;
    return 1;
}

unsigned grid_of(int64_t len) { return (unsigned)std::max<int64_t>((len + BLOCK - 1) / BLOCK, 1); }

}  // namespace

struct refgpu {
    emg_mesh mesh;
    Geo geo;
    int bc[3][2];
    double cfl = 0.5, tol = 1e-3;
    int mode = EMG_MODE_WENO, positivity = 1;
    double t = 0.0;
    double e[8];
    int kap = 0;
    int nv = 5;         // 5: Euler, 7: FiveEq (GpuSystem::nv, lib.rs:64-69)
    bool five = false;
    int64_t m[3], g[3], len = 1, cells = 1;
    cudaStream_t stream = nullptr;
    double *u = nullptr, *u0 = nullptr, *w = nullptr, *rhs = nullptr, *f = nullptr, *uf = nullptr, *th = nullptr,
           *mf = nullptr, *mu = nullptr, *rates = nullptr;
    double* dir[3][2] = {};
    unsigned long long* counters = nullptr;
    int* bl0 = nullptr;
    std::vector<double> host_rates;

    bool active(int d) const { return mesh.n[d] > 1; }
};

#define RG_CUDA(x)                                                          \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) return fail(std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)
#define RG_LAUNCHED() RG_CUDA(cudaGetLastError())
#define EOSV(h) h->e[0], h->e[1], h->e[2], h->e[3], h->e[4], h->e[5], h->e[6], h->e[7], h->kap
// the entry point of the handle's system: NAME_euler_f64 or NAME_five_f64
#define SYS_LAUNCH(h, NAME, GRID, BLK, ...)                                      \
    do {                                                                        \
        if ((h)->five)                                                          \
            NAME##_five_f64<<<GRID, BLK, 0, (h)->stream>>>(__VA_ARGS__);        \
        else                                                                    \
            NAME##_euler_f64<<<GRID, BLK, 0, (h)->stream>>>(__VA_ARGS__);       \
    } while (0)

namespace {

int fill_ghosts(refgpu* h) {
    for (int d = 0; d < 3; d++) {
        if (!h->active(d)) continue;
        int e0 = (d + 1) % 3, e1 = (d + 2) % 3;
        if (e0 > e1) std::swap(e0, e1);
        const int64_t np = h->m[e0] * h->m[e1] * h->g[d];
        // momentum index of axis d (GpuSystem::mom, lib.rs:70-75)
        const int mom = (h->five ? 2 : 1) + d;
        SYS_LAUNCH(h, ghost, grid_of(np), BLOCK, EOSV(h), h->u, h->geo, d, h->bc[d][0], h->bc[d][1], mom, h->dir[d][0],
                   h->dir[d][1]);
        RG_LAUNCHED();
    }
    return 0;
}

int prim(refgpu* h) {
    SYS_LAUNCH(h, prim, grid_of(h->len), BLOCK, EOSV(h), h->u, h->w, h->geo, h->bl0);
    RG_LAUNCHED();
    return 0;
}

int rhs(refgpu* h, double dt) {
    int rc = fill_ghosts(h);
    if (rc) return rc;
    if ((rc = prim(h))) return rc;
    double ndim = 0;
    for (int d = 0; d < 3; d++) ndim += h->active(d) ? 1.0 : 0.0;
    int first = 1;
    for (int d = 0; d < 3; d++) {
        if (!h->active(d)) continue;
        const double dx = h->mesh.dx[d];
        const double lambda = h->positivity ? ndim * dt / dx : 0.0;
        const int64_t cross = (int64_t)h->mesh.n[(d + 1) % 3] * h->mesh.n[(d + 2) % 3];
        const int64_t nf = (h->mesh.n[d] + 1) * cross;
        const int64_t nm = (h->mesh.n[d] + 5) * cross;
        SYS_LAUNCH(h, theta, grid_of(nf), BLOCK, EOSV(h), h->w, h->geo, h->bl0, d, h->mode, h->tol, h->th);
        RG_LAUNCHED();
        if (h->mode != EMG_MODE_CENTRAL) {
            SYS_LAUNCH(h, midflux, grid_of(nm), BLOCK, EOSV(h), h->w, h->geo, h->bl0, d, h->th, h->mf, h->mu, h->counters);
            RG_LAUNCHED();
        }
        SYS_LAUNCH(h, flux, grid_of(nf), BLOCK, EOSV(h), h->w, h->geo, h->bl0, d, lambda, h->th, h->mf, h->mu, h->f, h->uf,
                   h->counters);
        RG_LAUNCHED();
        SYS_LAUNCH(h, accum, grid_of(h->cells), BLOCK, EOSV(h), h->w, h->geo, h->bl0, d, dx, h->f, h->uf, h->rhs, first);
        RG_LAUNCHED();
        first = 0;
    }
    return 0;
}

int rk(refgpu* h, double al, double be, double dt) {
    SYS_LAUNCH(h, rk, grid_of(h->cells), BLOCK, h->u, h->u0, h->rhs, h->geo, h->bl0, al, be, dt);
    RG_LAUNCHED();
    return 0;
}

}  // namespace

extern "C" {

const char* refgpu_last_error(void) { return g_err.c_str(); }

int refgpu_destroy(refgpu* h) {
    if (!h) return 0;
    if (h->stream) cudaStreamSynchronize(h->stream);
    double* bufs[] = {h->u, h->u0, h->w, h->rhs, h->f, h->uf, h->th, h->mf, h->mu, h->rates};
    for (double* b : bufs)
        if (b) cudaFree(b);
    for (auto& pair : h->dir)
        for (double* b : pair)
            if (b) cudaFree(b);
    if (h->counters) cudaFree(h->counters);
    if (h->bl0) cudaFree(h->bl0);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return 0;
}

// GpuSolver::from_cpu (lib.rs:186-258) in f64: u_aos is the ghost-padded AoS
// state of the CPU solver (len cells of nv values); ev the EOS arguments of
// GpuSystem::eos_args (lib.rs:76-81); bc kinds and their nv-value states.
static int create_any(const emg_mesh* mesh, const double ev[8], int kap, int nv, const int kinds[6],
                      const double* const states[6], const emg_opts* opts, const double* u_aos, size_t len,
                      refgpu** out) {
    *out = nullptr;
    refgpu* h = new refgpu();
    h->nv = nv;
    h->five = nv == 7;
    h->kap = kap;
    h->mesh = *mesh;
    for (int d = 0; d < 3; d++) {
        if (mesh->n[d] < 1) {
            delete h;
            return fail("mesh extents must be >= 1");
        }
        h->g[d] = h->active(d) ? mesh->ng : 0;
        h->m[d] = mesh->n[d] + 2 * h->g[d];
        h->len *= h->m[d];
        h->cells *= mesh->n[d];
        h->bc[d][0] = kinds[2 * d];
        h->bc[d][1] = kinds[2 * d + 1];
    }
    if ((size_t)h->len != len) {
        delete h;
        return fail("state length does not match the padded mesh");
    }
    for (int d = 0; d < 3; d++) {
        h->geo.m[d] = (int)h->m[d];
        h->geo.n[d] = (int)mesh->n[d];
        h->geo.g[d] = (int)h->g[d];
    }
    h->geo.stride[0] = (long)(h->m[1] * h->m[2]);
    h->geo.stride[1] = (long)h->m[2];
    h->geo.stride[2] = 1;
    h->geo.ncell = (long)h->len;
    h->geo.ntot = (long)h->len;
    h->geo.rtot = (long)h->cells;
    h->geo.nb = 1;
    h->geo.s0 = 0;
    memcpy(h->e, ev, sizeof h->e);
    h->cfl = opts->cfl;
    h->tol = opts->tol;
    h->mode = opts->mode;
    h->positivity = opts->positivity;
    auto bail = [&](int rc) {
        refgpu_destroy(h);
        return rc;
    };
    int64_t maxf = 1, maxm = 1;
    for (int d = 0; d < 3; d++) {
        if (!h->active(d)) continue;
        const int64_t cross = (int64_t)mesh->n[(d + 1) % 3] * mesh->n[(d + 2) % 3];
        maxf = std::max<int64_t>(maxf, (mesh->n[d] + 1) * cross);
        maxm = std::max<int64_t>(maxm, (mesh->n[d] + 5) * cross);
    }
    const size_t sb = (size_t)h->nv * h->len * sizeof(double);
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&h->u, sb) != cudaSuccess || cudaMalloc(&h->u0, sb) != cudaSuccess ||
        cudaMalloc(&h->w, sb) != cudaSuccess ||
        cudaMalloc(&h->rhs, (size_t)h->nv * h->cells * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->f, (size_t)h->nv * maxf * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->uf, (size_t)maxf * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->th, (size_t)maxf * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->mf, (size_t)h->nv * maxm * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->mu, (size_t)maxm * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->counters, 4 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc(&h->rates, 2 * RATE_BLOCKS * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&h->bl0, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return bail(fail("device allocation failed"));
    }
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++) {
            double vals[NV_MAX] = {0, 0, 0, 0, 0, 0, 0};
            const int k = kinds[2 * d + s];
            if (k == EMG_BC_DIRICHLET || k == EMG_BC_CHARACTERISTIC)
                for (int q = 0; q < nv; q++) vals[q] = states[2 * d + s][q];
            if (cudaMalloc(&h->dir[d][s], nv * sizeof(double)) != cudaSuccess ||
                cudaMemcpy(h->dir[d][s], vals, nv * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
                return bail(fail("boundary state upload failed"));
        }
    // SoA upload (lib.rs:204-213); the other arrays start at zero (alloc_zeros)
    std::vector<double> soa((size_t)h->nv * h->len);
    for (int64_t c = 0; c < h->len; c++)
        for (int q = 0; q < nv; q++) soa[(size_t)q * h->len + c] = u_aos[(size_t)nv * c + q];
    const int zero = 0;
    if (cudaMemcpy(h->u, soa.data(), sb, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(h->u0, 0, sb) != cudaSuccess || cudaMemset(h->w, 0, sb) != cudaSuccess ||
        cudaMemset(h->rhs, 0, (size_t)h->nv * h->cells * sizeof(double)) != cudaSuccess ||
        cudaMemset(h->counters, 0, 4 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMemcpy(h->bl0, &zero, sizeof zero, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail("state upload failed"));
    h->host_rates.resize(2 * RATE_BLOCKS);
    *out = h;
    return 0;
}

// Euler system (GpuSystem::Euler): eos_args = [γ, p∞, b, q, 1.4, 0, 0, 0], kapila 0
int refgpu_create(const emg_mesh* mesh, const emg_eos* eos, const emg_bc bc[6], const emg_opts* opts,
                  const double* u_aos, size_t len, refgpu** out) {
    if (!mesh || !eos || !bc || !opts || !u_aos || !out) return fail("null argument");
    const double ev[8] = {eos->gamma, eos->p_inf, eos->b, eos->q, 1.4, 0.0, 0.0, 0.0};  // lib.rs:77-79
    int kinds[6];
    const double* states[6];
    for (int i = 0; i < 6; i++) {
        kinds[i] = bc[i].kind;
        states[i] = bc[i].state;
    }
    return create_any(mesh, ev, 0, 5, kinds, states, opts, u_aos, len, out);
}

// Five-equation system (GpuSystem::FiveEq): eos_args = both phases' [γ, p∞, b, q], kapila
int refgpu_five_create(const emg_mesh* mesh, const emg_five_system* sys, const emg_bc7 bc[6], const emg_opts* opts,
                       const double* u_aos, size_t len, refgpu** out) {
    if (!mesh || !sys || !bc || !opts || !u_aos || !out) return fail("null argument");
    const double ev[8] = {sys->eos[0].gamma, sys->eos[0].p_inf, sys->eos[0].b, sys->eos[0].q,
                          sys->eos[1].gamma, sys->eos[1].p_inf, sys->eos[1].b, sys->eos[1].q};  // lib.rs:80
    int kinds[6];
    const double* states[6];
    for (int i = 0; i < 6; i++) {
        kinds[i] = bc[i].kind;
        states[i] = bc[i].state;
    }
    return create_any(mesh, ev, sys->kapila ? 1 : 0, 7, kinds, states, opts, u_aos, len, out);
}

// GpuSolver::step (lib.rs:391-401)
int refgpu_step(refgpu* h, double dt) {
    if (!h) return fail("null handle");
    RG_CUDA(cudaMemcpyAsync(h->u0, h->u, (size_t)h->nv * h->len * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    int rc;
    if ((rc = rhs(h, dt)) || (rc = rk(h, 0.0, 1.0, dt))) return rc;
    if ((rc = rhs(h, dt)) || (rc = rk(h, 0.75, 0.25, dt))) return rc;
    if ((rc = rhs(h, dt)) || (rc = rk(h, 1.0 / 3.0, 2.0 / 3.0, dt))) return rc;
    h->t += dt;
    return 0;
}

// GpuSolver::dt_cfl (lib.rs:404-432): one device→host copy and a host max per call
int refgpu_dt_cfl(refgpu* h, double* dt) {
    if (!h || !dt) return fail("null argument");
    int rc = fill_ghosts(h);
    if (rc) return rc;
    if ((rc = prim(h))) return rc;
    SYS_LAUNCH(h, rate, RATE_BLOCKS, 256, EOSV(h), h->w, h->geo, h->bl0, h->mesh.dx[0], h->mesh.dx[1], h->mesh.dx[2],
               h->rates);
    RG_LAUNCHED();
    RG_CUDA(cudaMemcpyAsync(h->host_rates.data(), h->rates, 2 * RATE_BLOCKS * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream));
    RG_CUDA(cudaStreamSynchronize(h->stream));
    double r1 = 0.0, r2 = 0.0;
    for (int b = 0; b < RATE_BLOCKS; b++) {
        r1 = std::max(r1, h->host_rates[2 * b]);
        r2 = std::max(r2, h->host_rates[2 * b + 1]);
    }
    double d = h->cfl / r1;
    if (r2 > 0.0) d = std::min(d, 0.5 / r2);
    *dt = d;
    return 0;
}

// nsteps iterations of GpuSolver::run_to's loop body (lib.rs:435-447) without
// the t_end clamp: dt_cfl, the collapse check, step. taken counts the steps.
int refgpu_advance(refgpu* h, uint64_t nsteps, uint64_t* taken) {
    if (!h) return fail("null handle");
    uint64_t n = 0;
    for (; n < nsteps; n++) {
        double dt = 0.0;
        int rc = refgpu_dt_cfl(h, &dt);
        if (rc) return rc;
        if (!(dt > 0.0 && dt < INFINITY)) {
            if (taken) *taken = n;
            return fail("time step collapsed");
        }
        if ((rc = refgpu_step(h, dt))) return rc;
    }
    if (taken) *taken = n;
    return 0;
}

// GpuSolver::download (lib.rs:450-455): ghost-padded AoS
int refgpu_download(refgpu* h, double* u_aos, size_t len) {
    if (!h || !u_aos || len != (size_t)h->len) return fail("state length does not match the padded mesh");
    std::vector<double> soa((size_t)h->nv * h->len);
    RG_CUDA(cudaMemcpyAsync(soa.data(), h->u, soa.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    RG_CUDA(cudaStreamSynchronize(h->stream));
    for (int64_t c = 0; c < h->len; c++)
        for (int q = 0; q < h->nv; q++) u_aos[(size_t)h->nv * c + q] = soa[(size_t)q * h->len + c];
    return 0;
}

// GpuSolver::counters (lib.rs:458-461): shock-path faces, fallbacks, limited faces
int refgpu_counters(refgpu* h, uint64_t out[3]) {
    if (!h || !out) return fail("null argument");
    unsigned long long c[4];
    RG_CUDA(cudaMemcpyAsync(c, h->counters, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    RG_CUDA(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < 3; i++) out[i] = c[i];
    return 0;
}

void* refgpu_stream(refgpu* h) { return h ? (void*)h->stream : nullptr; }

int refgpu_synchronize(refgpu* h) {
    if (!h) return fail("null handle");
    RG_CUDA(cudaStreamSynchronize(h->stream));
    return 0;
}

}  // extern "C"
