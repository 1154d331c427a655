// Block-AMR kernels: box pipelines (prediction from the coarser level,
// restriction from the finer level), leaf ghost slabs, refluxing, the
// SSP-RK3 update with the fused CFL rate, and wavelet details. Each kernel
// follows the reference CPU operator it names (fluid/crates/compressible/
// src/amr.rs) in arithmetic order.
#pragma once
#include "amr_dev.cuh"
#include "sweep.cuh"

namespace emg {

// row-major cell index within a box of size s
// (box cells stay far below 2^31: 32-bit division, several times cheaper
// than the 64-bit one in these index-bound kernels)
__device__ __forceinline__ void box_coord(int64_t q, const int* s, int64_t* c) {
    const int qi = (int)q;
    const int a = qi / s[2];
    c[2] = qi - a * s[2];
    c[1] = a % s[1];
    c[0] = a / s[1];
}
__device__ __forceinline__ int64_t box_index(const int64_t* c, const int* s) { return (c[0] * s[1] + c[1]) * s[2] + c[2]; }

// size of a prediction box after `npass` separable passes (active axes in order)
__device__ __forceinline__ void pbox_size(const AmrDev& A, const PBox& b, int npass, int* s) {
    for (int d = 0; d < 3; d++) s[d] = b.csz[d];
    for (int i = 0; i < npass; i++) s[A.dims[i]] = b.fsz[A.dims[i]];
}
__device__ __forceinline__ void rbox_size(const AmrDev& A, const RBox& b, int npass, int* s) {
    for (int d = 0; d < 3; d++) s[d] = b.sz[d];
    for (int i = 0; i < npass; i++) s[A.dims[i]] = b.hi[A.dims[i]] - b.lo[A.dims[i]];
}

// gather_box(l−1) inner cells by sampling; cells beyond a non-periodic
// boundary are left invalid for bc_box (amr.rs:508-530). `off` is the box's
// cell offset in buf/ok.
template <int NV>
__device__ __forceinline__ void pbox_gather_cell(const AmrDev& A, const PBox& b, int64_t q, double* buf,
                                                 unsigned char* ok, int64_t off) {
    const int l = b.l - 1;
    int64_t c[3];
    box_coord(q, b.csz, c);
    int64_t g[3] = {b.cmin[0] + c[0], b.cmin[1] + c[1], b.cmin[2] + c[2]};
    bool out = false;
    for (int i = 0; i < A.ndims; i++) {
        const int d = A.dims[i];
        const int64_t nn = amr_nlevel(A, l, d);
        if ((g[d] < 0 || g[d] >= nn) && A.bc[d][g[d] >= nn ? 1 : 0] != EMG_BC_PERIODIC) out = true;
    }
    double* v = buf + (off + q) * NV;
    if (out) {
        ok[off + q] = 0;
    } else {
        amr_sample<NV>(A, l, g, v, 0);
        ok[off + q] = 1;
    }
}
template <int NV>
__global__ void pbox_gather(const AmrDev A, const PBox* __restrict__ boxes, double* buf, unsigned char* ok) {
    const PBox b = boxes[blockIdx.x];
    const int64_t n = (int64_t)b.csz[0] * b.csz[1] * b.csz[2];
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x)
        pbox_gather_cell<NV>(A, b, q, buf, ok, b.off);
}

// bc_box sweep along active axis dims[di] over a box at level l with global
// origin g0 (amr.rs:450-504): cells outside along that axis and inside along
// every later one copy their (flipped) source from the same box, or take the
// Dirichlet state.
template <int NV>
__device__ __forceinline__ void bc_cell(const AmrDev& A, int l, const int64_t* g0, const int* s, int64_t q, int di,
                                        double* buf, unsigned char* ok, int64_t off) {
    int64_t c[3];
    box_coord(q, s, c);
    const int64_t g[3] = {g0[0] + c[0], g0[1] + c[1], g0[2] + c[2]};
    const int d = A.dims[di];
    int64_t n[3];
    for (int e = 0; e < 3; e++) n[e] = amr_nlevel(A, l, e);
    auto outside = [&](int e) {
        return (g[e] < 0 || g[e] >= n[e]) && A.bc[e][g[e] >= n[e] ? 1 : 0] != EMG_BC_PERIODIC;
    };
    if (!outside(d)) return;
    for (int j = di + 1; j < A.ndims; j++)
        if (outside(A.dims[j])) return;
    const int side = g[d] >= n[d] ? 1 : 0;
    const int kind = A.bc[d][side];
    double* dst = buf + (off + q) * NV;
    if (kind == EMG_BC_DIRICHLET) {
        for (int k = 0; k < NV; k++) dst[k] = A.bcs[d][side][k];
        ok[off + q] = 1;
        return;
    }
    int64_t src_g;
    if (kind == EMG_BC_OUTFLOW)
        src_g = g[d] < 0 ? 0 : n[d] - 1;
    else  // reflect
        src_g = side == 0 ? -1 - g[d] : 2 * n[d] - 1 - g[d];
    int64_t sc[3] = {c[0], c[1], c[2]};
    sc[d] = src_g - g0[d];
    if (sc[d] < 0 || sc[d] >= s[d]) return;
    const int64_t sq = box_index(sc, s);
    if (!ok[off + sq]) return;
    const double* src = buf + (off + sq) * NV;
    for (int k = 0; k < NV; k++) dst[k] = src[k];
    if (kind == EMG_BC_REFLECT) dst[amr_iu<NV>() + d] = -dst[amr_iu<NV>() + d];
    ok[off + q] = 1;
}

template <int NV>
__global__ void pbox_bc(const AmrDev A, const PBox* __restrict__ boxes, double* buf, unsigned char* ok, int di) {
    const PBox b = boxes[blockIdx.x];
    if (!((b.bcmask >> di) & 1)) return;  // nothing of this box lies outside along dims[di]
    const int64_t n = (int64_t)b.csz[0] * b.csz[1] * b.csz[2];
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x)
        bc_cell<NV>(A, b.l - 1, b.cmin, b.csz, q, di, buf, ok, b.off);
}

// cells still invalid after bc_box are sampled (amr.rs:531-542)
template <int NV>
__device__ __forceinline__ void pbox_fallback_cell(const AmrDev& A, const PBox& b, int64_t q, double* buf,
                                                   unsigned char* ok, int64_t off) {
    if (ok[off + q]) return;
    int64_t c[3];
    box_coord(q, b.csz, c);
    const int64_t g[3] = {b.cmin[0] + c[0], b.cmin[1] + c[1], b.cmin[2] + c[2]};
    amr_sample<NV>(A, b.l - 1, g, buf + (off + q) * NV, 0);
    ok[off + q] = 1;
}
template <int NV>
__global__ void pbox_fallback(const AmrDev A, const PBox* __restrict__ boxes, double* buf, unsigned char* ok) {
    const PBox b = boxes[blockIdx.x];
    const int64_t n = (int64_t)b.csz[0] * b.csz[1] * b.csz[2];
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x)
        pbox_fallback_cell<NV>(A, b, q, buf, ok, b.off);
}

// one separable 6-point prediction pass along dims[di] (amr.rs:560-583): output
// cell q of the box after di+1 passes from the box after di passes
template <int NV>
__device__ __forceinline__ void pbox_pass_cell(const AmrDev& A, const PBox& b, int di, const int* si, const int* so,
                                               int64_t q, const double* in, double* outb, int64_t off) {
    const int d = A.dims[di];
    int64_t c[3];
    box_coord(q, so, c);
    const int64_t f = b.fmin[d] + c[d];
    const int par = (int)amr_erem(f, 2);
    const int64_t base = amr_ediv(f, 2) + (par == 1 ? -2 : -3) - b.cmin[d];
    double acc[NV] = {};
    for (int kk = 0; kk < 6; kk++) {
        int64_t sc[3] = {c[0], c[1], c[2]};
        sc[d] = base + kk;
        const double* v = in + (off + box_index(sc, si)) * NV;
        const double w = A.wp[par][kk];
        for (int k = 0; k < NV; k++) acc[k] = acc[k] + w * v[k];
    }
    double* o = outb + (off + q) * NV;
    for (int k = 0; k < NV; k++) o[k] = acc[k];
}
template <int NV>
__global__ void pbox_pass(const AmrDev A, const PBox* __restrict__ boxes, const double* in, double* outb, int di) {
    const PBox b = boxes[blockIdx.x];
    int si[3], so[3];
    pbox_size(A, b, di, si);
    pbox_size(A, b, di + 1, so);
    const int64_t n = (int64_t)so[0] * so[1] * so[2];
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x)
        pbox_pass_cell<NV>(A, b, di, si, so, q, in, outb, b.off);
}

// write the predicted fine box into its target block
template <int NV>
__device__ __forceinline__ void pbox_scatter_cell(const AmrDev& A, const PBox& b, int64_t q, const double* in,
                                                  int64_t off) {
    double* u = A.u + (int64_t)b.slot * A.bcell;
    int64_t c[3];
    box_coord(q, b.fsz, c);
    const int64_t cell = ((b.t0[0] + c[0]) * A.ext[1] + (b.t0[1] + c[1])) * A.ext[2] + (b.t0[2] + c[2]);
    const double* v = in + (off + q) * NV;
    for (int k = 0; k < NV; k++) u[(int64_t)k * A.ntot + cell] = v[k];
}
template <int NV>
__global__ void pbox_scatter(const AmrDev A, const PBox* __restrict__ boxes, const double* in) {
    const PBox b = boxes[blockIdx.x];
    const int64_t n = (int64_t)b.fsz[0] * b.fsz[1] * b.fsz[2];
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x)
        pbox_scatter_cell<NV>(A, b, q, in, b.off);
}

// The whole prediction pipeline of one box in shared memory (one CTA per
// box): gather, boundary fill per active axis, fallback sampling, one
// separable pass per active axis (ping-pong) and the scatter, with the same
// per-cell arithmetic as the multi-launch pipeline above. `cap` is the
// largest box stage in cells; dynamic shared memory 2·cap·NV doubles + cap bytes.
// 512 threads: one CTA per box fills an SM's shared memory, so the CTA's own
// warps are all the latency hiding the gathers get
constexpr int PBOX_THREADS = 512;
template <int NV>
__global__ void __launch_bounds__(PBOX_THREADS) pbox_fused(const AmrDev A, const PBox* __restrict__ boxes, int cap) {
    extern __shared__ __align__(16) double pb_smem[];
    double* bufs[2] = {pb_smem, pb_smem + (size_t)cap * NV};
    unsigned char* ok = reinterpret_cast<unsigned char*>(pb_smem + (size_t)2 * cap * NV);
    const PBox b = boxes[blockIdx.x];
    const int64_t nc = (int64_t)b.csz[0] * b.csz[1] * b.csz[2];
    // A coarse patch inside the domain that spans at most three blocks per
    // axis reads its blocks through a table of their pool slots, filled once
    // per box: no per-cell key division or block-map load. Cells of absent
    // blocks (and every other patch) take the general sample, which gives the
    // same value for cells inside the domain.
    __shared__ int s_slot[27];
    __shared__ int s_fast;
    __shared__ int64_t s_kmin[3];
    __shared__ int s_nk[3];
    const int L = b.l - 1;
    if (threadIdx.x == 0) {
        int fast = 1;
        for (int d = 0; d < 3; d++) {
            s_kmin[d] = 0;
            s_nk[d] = 1;
            if (!A.act[d]) continue;
            const int64_t n = amr_nlevel(A, L, d);
            if (b.cmin[d] < 0 || b.cmin[d] + b.csz[d] > n || b.csz[d] > 2 * A.bd[d] + 1) fast = 0;
            s_kmin[d] = amr_ediv(b.cmin[d], A.bd[d]);
            s_nk[d] = (int)(amr_ediv(b.cmin[d] + b.csz[d] - 1, A.bd[d]) - s_kmin[d] + 1);
        }
        s_fast = fast;
    }
    __syncthreads();
    if (s_fast) {
        const int nt = s_nk[0] * s_nk[1] * s_nk[2];
        if (threadIdx.x < nt) {
            const int t = threadIdx.x;
            const int64_t key[3] = {s_kmin[0] + t / (s_nk[1] * s_nk[2]), s_kmin[1] + (t / s_nk[2]) % s_nk[1], s_kmin[2] + t % s_nk[2]};
            s_slot[t] = amr_get(A, L, key);
        }
        __syncthreads();
        for (int64_t q = threadIdx.x; q < nc; q += blockDim.x) {
            int64_t c[3];
            box_coord(q, b.csz, c);
            int j[3];
            int64_t lc[3];
            for (int d = 0; d < 3; d++) {
                if (!A.act[d]) {
                    j[d] = 0;
                    lc[d] = 0;
                    continue;
                }
                const int o = (int)(b.cmin[d] - s_kmin[d] * A.bd[d] + c[d]);  // 0 <= o < 3·bd
                j[d] = o >= A.bd[d] ? (o >= 2 * A.bd[d] ? 2 : 1) : 0;
                lc[d] = o - j[d] * A.bd[d];
            }
            const int slot = s_slot[(j[0] * s_nk[1] + j[1]) * s_nk[2] + j[2]];
            double* v = bufs[0] + q * NV;
            if (slot >= 0) {
                amr_load<NV>(A, slot, amr_cell(A, lc), v);
            } else {
                const int64_t g[3] = {b.cmin[0] + c[0], b.cmin[1] + c[1], b.cmin[2] + c[2]};
                amr_sample<NV>(A, L, g, v, 0);
            }
            ok[q] = 1;
        }
    } else {
        for (int64_t q = threadIdx.x; q < nc; q += blockDim.x) pbox_gather_cell<NV>(A, b, q, bufs[0], ok, 0);
    }
    __syncthreads();
    for (int di = 0; di < A.ndims; di++) {
        if (!((b.bcmask >> di) & 1)) continue;  // the same for the whole CTA
        for (int64_t q = threadIdx.x; q < nc; q += blockDim.x) bc_cell<NV>(A, b.l - 1, b.cmin, b.csz, q, di, bufs[0], ok, 0);
        __syncthreads();
    }
    for (int64_t q = threadIdx.x; q < nc; q += blockDim.x) pbox_fallback_cell<NV>(A, b, q, bufs[0], ok, 0);
    __syncthreads();
    int cur = 0;
    for (int di = 0; di < A.ndims; di++) {
        int si[3], so[3];
        pbox_size(A, b, di, si);
        pbox_size(A, b, di + 1, so);
        const int64_t n = (int64_t)so[0] * so[1] * so[2];
        for (int64_t q = threadIdx.x; q < n; q += blockDim.x) pbox_pass_cell<NV>(A, b, di, si, so, q, bufs[cur], bufs[1 - cur], 0);
        __syncthreads();
        cur = 1 - cur;
    }
    const int64_t nf = (int64_t)b.fsz[0] * b.fsz[1] * b.fsz[2];
    for (int64_t q = threadIdx.x; q < nf; q += blockDim.x) pbox_scatter_cell<NV>(A, b, q, bufs[cur], 0);
}

// fine patch of a restriction box with validity (amr.rs:632-663). `rem`
// (optional) replays a batch of coarsenings in their sequential order: fine
// block id is absent for box seq when rem[id] < seq, i.e. it was removed by an
// earlier coarsening of the batch.
template <int NV>
__global__ void rbox_gather(const AmrDev A, const RBox* __restrict__ boxes, double* buf, unsigned char* ok,
                            const int* __restrict__ rem, int skip_fast) {
    const RBox b = boxes[blockIdx.x];
    if (skip_fast && b.fast) return;  // gathered inside rbox_gather_pass0
    const int lf = b.l + 1;
    const int64_t n = (int64_t)b.sz[0] * b.sz[1] * b.sz[2];
    // fine patch inside the domain spanning at most four blocks per axis: the
    // pool slots of its blocks (after the removal mask) from a table built by
    // each CTA, instead of a key division and a block-map load per cell
    __shared__ int s_slot[64];
    __shared__ int s_fast;
    __shared__ int64_t s_kmin[3];
    __shared__ int s_nk[3];
    if (threadIdx.x == 0) {
        int fast = 1;
        for (int d = 0; d < 3; d++) {
            s_kmin[d] = 0;
            s_nk[d] = 1;
            if (!A.act[d]) continue;
            const int64_t nf = amr_nlevel(A, lf, d);
            if (b.f0[d] < 0 || b.f0[d] + b.sz[d] > nf || b.sz[d] > 3 * A.bd[d] + 1) fast = 0;
            s_kmin[d] = amr_ediv(b.f0[d], A.bd[d]);
            s_nk[d] = (int)(amr_ediv(b.f0[d] + b.sz[d] - 1, A.bd[d]) - s_kmin[d] + 1);
        }
        s_fast = fast;
    }
    __syncthreads();
    if (s_fast) {
        const int nt = s_nk[0] * s_nk[1] * s_nk[2];
        if (threadIdx.x < nt) {
            const int t = threadIdx.x;
            const int64_t key[3] = {s_kmin[0] + t / (s_nk[1] * s_nk[2]), s_kmin[1] + (t / s_nk[2]) % s_nk[1], s_kmin[2] + t % s_nk[2]};
            int id = amr_get(A, lf, key);
            if (id >= 0 && rem != nullptr && b.seq >= 0 && rem[id] < b.seq) id = -1;
            s_slot[t] = id;
        }
        __syncthreads();
        for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
            int64_t c[3];
            box_coord(q, b.sz, c);
            int j[3];
            int64_t lc[3];
            for (int d = 0; d < 3; d++) {
                if (!A.act[d]) {
                    j[d] = 0;
                    lc[d] = 0;
                    continue;
                }
                const int o = (int)(b.f0[d] - s_kmin[d] * A.bd[d] + c[d]);  // 0 <= o < 4·bd
                j[d] = o / A.bd[d];
                lc[d] = o - j[d] * A.bd[d];
            }
            const int id = s_slot[(j[0] * s_nk[1] + j[1]) * s_nk[2] + j[2]];
            double* v = buf + (b.off + q) * NV;
            if (id >= 0) {
                amr_load<NV>(A, id, amr_cell(A, lc), v);
            } else {
                for (int k = 0; k < NV; k++) v[k] = 0.0;
            }
            ok[b.off + q] = id >= 0 ? 1 : 0;
        }
        return;
    }
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(q, b.sz, c);
        int64_t gw[3];
        bool out = false;
        for (int d = 0; d < 3; d++) {
            const int64_t g = b.f0[d] + c[d];
            gw[d] = g;
            if (A.act[d]) {
                const int64_t nf = amr_nlevel(A, lf, d);
                if (g < 0 || g >= nf) {
                    if (A.bc[d][g >= nf ? 1 : 0] == EMG_BC_PERIODIC)
                        gw[d] = amr_erem(g, nf);
                    else
                        out = true;
                }
            }
        }
        double* v = buf + (b.off + q) * NV;
        unsigned char o = 0;
        if (!out) {
            int64_t key[3], lc[3];
            for (int d = 0; d < 3; d++) {
                key[d] = A.act[d] ? amr_ediv(gw[d], A.bd[d]) : 0;
                lc[d] = A.act[d] ? amr_erem(gw[d], A.bd[d]) : 0;
            }
            int id = amr_get(A, lf, key);
            if (id >= 0 && rem != nullptr && b.seq >= 0 && rem[id] < b.seq) id = -1;
            if (id >= 0) {
                amr_load<NV>(A, id, amr_cell(A, lc), v);
                o = 1;
            }
        }
        if (!o)
            for (int k = 0; k < NV; k++) v[k] = 0.0;
        ok[b.off + q] = o;
    }
}

template <int NV>
__global__ void rbox_bc(const AmrDev A, const RBox* __restrict__ boxes, double* buf, unsigned char* ok, int di,
                        const int* __restrict__ sel) {
    const RBox b = boxes[sel ? sel[blockIdx.x] : blockIdx.x];
    const int64_t n = (int64_t)b.sz[0] * b.sz[1] * b.sz[2];
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x)
        bc_cell<NV>(A, b.l + 1, b.f0, b.sz, q, di, buf, ok, b.off);
}

// one restriction pass along dims[di] with the shifted stencils and the
// child-average fallback (amr.rs:674-727)
template <int NV>
__global__ void __launch_bounds__(256, 4) rbox_pass(const AmrDev A, const RBox* __restrict__ boxes, const double* in,
                                                   const unsigned char* okin,
                          double* outb, unsigned char* okout, int di, int skip_fast) {
    const RBox b = boxes[blockIdx.x];
    if (skip_fast && b.fast) return;  // first pass done by rbox_gather_pass0
    const int d = A.dims[di];
    int si[3], so[3];
    rbox_size(A, b, di, si);
    rbox_size(A, b, di + 1, so);
    const int shifts[5] = {0, -1, 1, -2, 2};
    const int64_t n = (int64_t)so[0] * so[1] * so[2];
    // stride of d in the box's row-major layout, and its extent
    const int64_t str = d == 0 ? (int64_t)si[1] * si[2] : (d == 1 ? si[2] : 1);
    const int sid = d == 0 ? si[0] : (d == 1 ? si[1] : si[2]);
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(q, so, c);
        const int cd = (int)(d == 0 ? c[0] : (d == 1 ? c[1] : c[2]));
        int64_t c0[3] = {c[0], c[1], c[2]};
        if (d == 0) c0[0] = 0;
        else if (d == 1) c0[1] = 0;
        else c0[2] = 0;
        const int64_t row0 = b.off + box_index(c0, si);  // source index at position 0 along d
        const int base = 2 * cd + 2;
        // positions base − 2 .. base + 7 (every stencil the shifts reach): index
        // and validity, position i = shift + 2 + kk of the unrolled stencils
        int64_t at[10];
        bool okp[10];
#pragma unroll
        for (int i = 0; i < 10; i++) {
            const int x = base - 2 + i;
            at[i] = row0 + (int64_t)x * str;
            okp[i] = x >= 0 && x < sid && okin[at[i]];
        }
        double acc[NV] = {};
        bool done = false;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const int sh = shifts[m];
            const int st = base + sh;
            if (!done && st >= 0 && st + 5 < sid) {
                bool all = true;
#pragma unroll
                for (int kk = 0; kk < 6; kk++) all = all && okp[sh + 2 + kk];
                if (all) {
#pragma unroll
                    for (int kk = 0; kk < 6; kk++) {
                        const double* v = in + at[sh + 2 + kk] * NV;
#pragma unroll
                        for (int k = 0; k < NV; k++) acc[k] = acc[k] + A.wrs[m][kk] * v[k];
                    }
                    done = true;
                }
            }
        }
        unsigned char o = done ? 1 : 0;
        if (!done && okp[4] && okp[5]) {  // positions base + 2, base + 3: the child average
            const int64_t pa = at[4], pb = at[5];
            for (int k = 0; k < NV; k++) acc[k] = 0.5 * (in[pa * NV + k] + in[pb * NV + k]);
            o = 1;
        }
        double* ov = outb + (b.off + q) * NV;
        for (int k = 0; k < NV; k++) ov[k] = acc[k];
        okout[b.off + q] = o;
    }
}

// Gather and first restriction pass (along dims[0]) in one kernel for boxes
// whose fine patch lies inside the domain (RBox::fast): the fine values come
// straight from the pool through a per-CTA table of the patch's block slots,
// so the gathered patch never goes through global scratch. Same stencil
// choice, validity and summation order as rbox_gather + rbox_pass.
template <int NV>
__global__ void __launch_bounds__(256, 4) rbox_gather_pass0(const AmrDev A, const RBox* __restrict__ boxes, double* outb,
                                                           unsigned char* okout,
                                  const int* __restrict__ rem) {
    const RBox b = boxes[blockIdx.x];
    if (!b.fast) return;
    const int lf = b.l + 1;
    __shared__ int s_slot[64];
    __shared__ int64_t s_kmin[3];
    __shared__ int s_nk[3];
    if (threadIdx.x == 0) {
        for (int d = 0; d < 3; d++) {
            s_kmin[d] = A.act[d] ? amr_ediv(b.f0[d], A.bd[d]) : 0;
            s_nk[d] = A.act[d] ? (int)(amr_ediv(b.f0[d] + b.sz[d] - 1, A.bd[d]) - s_kmin[d] + 1) : 1;
        }
    }
    __syncthreads();
    const int nt = s_nk[0] * s_nk[1] * s_nk[2];
    if (threadIdx.x < nt) {
        const int t = threadIdx.x;
        const int64_t key[3] = {s_kmin[0] + t / (s_nk[1] * s_nk[2]), s_kmin[1] + (t / s_nk[2]) % s_nk[1], s_kmin[2] + t % s_nk[2]};
        int id = amr_get(A, lf, key);
        if (id >= 0 && rem != nullptr && b.seq >= 0 && rem[id] < b.seq) id = -1;
        s_slot[t] = id;
    }
    __syncthreads();
    const int d = A.dims[0];
    int so[3];
    rbox_size(A, b, 1, so);
    const int sid = b.sz[d];
    const int shifts[5] = {0, -1, 1, -2, 2};
    const int64_t n = (int64_t)so[0] * so[1] * so[2];
    const int bdd = A.bd[d];
    const int64_t sd = d == 0 ? (int64_t)A.ext[1] * A.ext[2] : (d == 1 ? A.ext[2] : 1);  // pool stride along d
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(q, so, c);
        const int base = 2 * (int)c[d] + 2;
        // the block and local cell along the two other axes are the same for
        // every position of the stencil: resolve them once, then step along d
        int jt[3] = {0, 0, 0};
        int64_t lt[3] = {0, 0, 0};
        for (int e = 0; e < 3; e++) {
            if (e == d || !A.act[e]) continue;
            const int o = (int)(b.f0[e] - s_kmin[e] * A.bd[e] + c[e]);
            jt[e] = o / A.bd[e];
            lt[e] = o - jt[e] * A.bd[e];
        }
        // positions base − 2 .. base + 7 along d (every stencil the shifts can
        // reach): block index along d and local coordinate of the first one
        const int o0 = (int)(b.f0[d] - s_kmin[d] * bdd) + base - 2;
        const int jd0 = o0 >= 0 ? o0 / bdd : -((-o0 + bdd - 1) / bdd);  // floor (o0 ≥ −2)
        const int ld0 = o0 - jd0 * bdd;
        // slot table index of block jd along d (the other two block indices fixed)
        const int tstr = d == 0 ? s_nk[1] * s_nk[2] : (d == 1 ? s_nk[2] : 1);
        const int nkd = d == 0 ? s_nk[0] : (d == 1 ? s_nk[1] : s_nk[2]);
        const int tbase = (d == 0 ? 0 : jt[0] * s_nk[1] * s_nk[2]) + (d == 1 ? 0 : jt[1] * s_nk[2]) + (d == 2 ? 0 : jt[2]);
        auto slot_at = [&](int jd) -> int { return (jd < 0 || jd >= nkd) ? -1 : s_slot[tbase + jd * tstr]; };
        int64_t lcb[3] = {lt[0], lt[1], lt[2]};
        lcb[d] = 0;
        const int64_t cell0 = amr_cell(A, lcb);  // local cell at coordinate 0 along d
        int pslot[10];
        int64_t pcell[10];
        bool okp[10];
        {
            int jd = jd0, ld = ld0, sl = slot_at(jd0);
#pragma unroll
            for (int i = 0; i < 10; i++) {
                const int x = base - 2 + i;
                pslot[i] = sl;
                pcell[i] = cell0 + (int64_t)ld * sd;
                okp[i] = x >= 0 && x < sid && sl >= 0;
                if (++ld == bdd) {
                    ld = 0;
                    sl = slot_at(++jd);
                }
            }
        }
        // slot and local cell of the fine cell at position x along d
        // the stencils in the order of the shifts, the first whole one used;
        // unrolled, so that every position index is a constant and the
        // tables stay in registers (position i = shift + 2 + kk)
        double acc[NV] = {};
        bool done = false;
#pragma unroll
        for (int m = 0; m < 5; m++) {
            const int sh = shifts[m];
            const int st = base + sh;
            if (!done && st >= 0 && st + 5 < sid) {
                bool all = true;
#pragma unroll
                for (int kk = 0; kk < 6; kk++) all = all && okp[sh + 2 + kk];
                if (all) {
                    double v[6][NV];
#pragma unroll
                    for (int kk = 0; kk < 6; kk++) amr_load<NV>(A, pslot[sh + 2 + kk], pcell[sh + 2 + kk], v[kk]);
#pragma unroll
                    for (int kk = 0; kk < 6; kk++)
#pragma unroll
                        for (int k = 0; k < NV; k++) acc[k] = acc[k] + A.wrs[m][kk] * v[kk][k];
                    done = true;
                }
            }
        }
        unsigned char o = done ? 1 : 0;
        if (!done && okp[4] && okp[5]) {  // positions base + 2, base + 3: the child average
            double va[NV], vb[NV];
            amr_load<NV>(A, pslot[4], pcell[4], va);
            amr_load<NV>(A, pslot[5], pcell[5], vb);
            for (int k = 0; k < NV; k++) acc[k] = 0.5 * (va[k] + vb[k]);
            o = 1;
        }
        double* ov = outb + (b.off + q) * NV;
        for (int k = 0; k < NV; k++) ov[k] = acc[k];
        okout[b.off + q] = o;
    }
}

// write the restricted box into the ancestor's interior cells [lo, hi)
template <int NV>
__global__ void rbox_scatter(const AmrDev A, const RBox* __restrict__ boxes, const double* in) {
    const RBox b = boxes[blockIdx.x];
    int so[3];
    for (int d = 0; d < 3; d++) so[d] = b.hi[d] - b.lo[d];
    const int64_t n = (int64_t)so[0] * so[1] * so[2];
    double* u = A.u + (int64_t)b.slot * A.bcell;
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(q, so, c);
        const int64_t ic[3] = {b.lo[0] + c[0], b.lo[1] + c[1], b.lo[2] + c[2]};
        const int64_t cell = amr_cell(A, ic);
        const double* v = in + (b.off + q) * NV;
        for (int k = 0; k < NV; k++) u[(int64_t)k * A.ntot + cell] = v[k];
    }
}

// Same-level ghost slab copy (fill_scratch, amr.rs:1176-1187): task =
// (leaf slot, neighbour slot, direction o[3]).
struct CopyTask {
    int slot, src;
    int o[3];
};
// one CTA per task; the source cell is the destination cell shifted by one
// block along the task's direction (o = 0 on inactive axes)
constexpr int COPY_THREADS = 128;
template <int NV>
__global__ void __launch_bounds__(COPY_THREADS) ghost_copy(const AmrDev A, const CopyTask* __restrict__ tasks) {
    const CopyTask t = tasks[blockIdx.x];
    int rs[3], sz[3];
    for (int d = 0; d < 3; d++) {
        if (!A.act[d]) {
            rs[d] = 0;
            sz[d] = 1;
        } else if (t.o[d] == -1) {
            rs[d] = 0;
            sz[d] = A.ng;
        } else if (t.o[d] == 0) {
            rs[d] = A.ng;
            sz[d] = A.bd[d];
        } else {
            rs[d] = A.ng + A.bd[d];
            sz[d] = A.ng;
        }
    }
    const int e1 = A.ext[1], e2 = A.ext[2];
    const int shift = ((t.o[0] * A.bd[0]) * e1 + t.o[1] * A.bd[1]) * e2 + t.o[2] * A.bd[2];
    const int n = sz[0] * sz[1] * sz[2];
    double* dst = A.u + (int64_t)t.slot * A.bcell;
    const double* src = A.u + (int64_t)t.src * A.bcell;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const int a = q / sz[2];
        const int c2 = q - a * sz[2], c1 = a % sz[1], c0 = a / sz[1];
        const int de = ((rs[0] + c0) * e1 + rs[1] + c1) * e2 + rs[2] + c2;
        const int se = de - shift;
#pragma unroll
        for (int k = 0; k < NV; k++) dst[(int64_t)k * A.ntot + de] = src[(int64_t)k * A.ntot + se];
    }
}

// bc_box over the ghost-extended box of a leaf touching the domain boundary
// (fill_scratch → bc_box, amr.rs:1205-1217), one active axis per launch,
// restricted to the face slabs along that axis.
template <int NV>
__global__ void ghost_bc(const AmrDev A, const int* __restrict__ leaves, const int* __restrict__ level,
                         const int64_t* __restrict__ idx, int di) {
    const int slot = leaves[blockIdx.x];
    const int l = level[slot];
    const int64_t n = (int64_t)A.ext[0] * A.ext[1] * A.ext[2];
    int64_t g0[3];
    for (int d = 0; d < 3; d++) g0[d] = idx[3 * slot + d] * A.bd[d] - A.gof[d];
    int64_t nl[3];
    for (int e = 0; e < 3; e++) nl[e] = amr_nlevel(A, l, e);
    const int d = A.dims[di];
    double* u = A.u + (int64_t)slot * A.bcell;
    // the two face slabs along d over the interior lanes (the only ghost cells
    // that are read); other ghost cells are left as they are
    int span[3];
    for (int e = 0; e < 3; e++) span[e] = e == d ? 2 * A.gof[d] : (A.act[e] ? A.bd[e] : 1);
    const int64_t ns = (int64_t)span[0] * span[1] * span[2];
    (void)n;
    for (int64_t t = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; t < ns; t += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(t, span, c);
        for (int e = 0; e < 3; e++) {
            if (e == d)
                c[e] = c[e] < A.gof[d] ? c[e] : c[e] + A.bd[d];
            else if (A.act[e])
                c[e] += A.gof[e];
        }
        const int64_t q = (c[0] * A.ext[1] + c[1]) * A.ext[2] + c[2];
        const int64_t g[3] = {g0[0] + c[0], g0[1] + c[1], g0[2] + c[2]};
        auto outside = [&](int e) {
            return (g[e] < 0 || g[e] >= nl[e]) && A.bc[e][g[e] >= nl[e] ? 1 : 0] != EMG_BC_PERIODIC;
        };
        if (!outside(d)) continue;
        bool later = false;
        for (int j = di + 1; j < A.ndims; j++) later = later || outside(A.dims[j]);
        if (later) continue;
        const int side = g[d] >= nl[d] ? 1 : 0;
        const int kind = A.bc[d][side];
        if (kind == EMG_BC_DIRICHLET) {
            for (int k = 0; k < NV; k++) u[(int64_t)k * A.ntot + q] = A.bcs[d][side][k];
            continue;
        }
        const int64_t sg = kind == EMG_BC_OUTFLOW ? (g[d] < 0 ? 0 : nl[d] - 1) : (side == 0 ? -1 - g[d] : 2 * nl[d] - 1 - g[d]);
        int64_t sc[3] = {c[0], c[1], c[2]};
        sc[d] = sg - g0[d];
        if (sc[d] < 0 || sc[d] >= A.ext[d]) {  // source outside the box: needs sampling
            atomicOr(A.err, 2u);
            continue;
        }
        const int64_t sq = (sc[0] * A.ext[1] + sc[1]) * A.ext[2] + sc[2];
        for (int k = 0; k < NV; k++) {
            double v = u[(int64_t)k * A.ntot + sq];
            if (kind == EMG_BC_REFLECT && k == amr_iu<NV>() + d) v = -v;
            u[(int64_t)k * A.ntot + q] = v;
        }
    }
}

// Refluxing (amr.rs:1327-1406): one thread per corrected coarse cell applies
// its corrections in the CPU's order. A task names the coarse face (slot, d,
// side, pencil) and up to four fine faces.
// (flat index, block id) edits of the device block map
__global__ void map_scatter(int* map, const int64_t* __restrict__ pairs, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) map[pairs[2 * i]] = (int)pairs[2 * i + 1];
}

// One coarse face of a leaf whose same-level neighbour is refined
// (reflux, amr.rs:1327-1406): fine[qa][qb] are the leaf children of that
// neighbour covering quadrant (qa, qb) of the face (−1: none).
struct RefluxFace {
    int slot, d, side;
    int fine[2][2];
    double dx;
};
// Corrections of every face of one (d, side) bucket: one CTA per face, one
// thread per face pen. Each cell receives at most one correction per bucket,
// and the buckets run in the reference's (d, side) order, so every cell sums
// its corrections in the reference's order.
template <int NV>
__global__ void reflux_faces(const AmrDev A, double* rhs, const double* __restrict__ face, int npen,
                             const RefluxFace* __restrict__ tasks) {
    const RefluxFace tk = tasks[blockIdx.x];
    const int d = tk.d;
    const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
    const int b0 = A.bd[e0], b1 = A.bd[e1];
    for (int pen = threadIdx.x; pen < b0 * b1; pen += blockDim.x) {
        const int a = pen / b1, bb = pen % b1;
        double sum[NV] = {};
        double cnt = 0.0;
        for (int fa = 0; fa < (A.act[e0] ? 2 : 1); fa++)
            for (int fb = 0; fb < (A.act[e1] ? 2 : 1); fb++) {
                const int qa = A.act[e0] ? (2 * a + fa) / b0 : 0, qb = A.act[e1] ? (2 * bb + fb) / b1 : 0;
                const int cid = tk.fine[qa][qb];
                if (cid < 0) continue;
                const int la = A.act[e0] ? (2 * a + fa) % b0 : 0, lb = A.act[e1] ? (2 * bb + fb) % b1 : 0;
                const double* fv = face + ((((int64_t)cid * 3 + d) * 2 + (1 - tk.side)) * NV) * npen + la * b1 + lb;
                for (int k = 0; k < NV; k++) sum[k] = sum[k] + fv[(int64_t)k * npen];
                cnt = cnt + 1.0;
            }
        if (cnt == 0.0) continue;
        const double* fc = face + ((((int64_t)tk.slot * 3 + d) * 2 + tk.side) * NV) * npen + pen;
        int64_t c[3];
        c[d] = tk.side == 1 ? A.bd[d] - 1 : 0;
        c[e0] = a;
        c[e1] = bb;
        double* r = rhs + (int64_t)tk.slot * A.bcell + amr_cell(A, c);
        for (int k = 0; k < NV; k++) {
            const double df = sum[k] / cnt - fc[(int64_t)k * npen];
            const double dr = tk.side == 1 ? -df / tk.dx : df / tk.dx;
            r[(int64_t)k * A.ntot] = r[(int64_t)k * A.ntot] + dr;
        }
    }
}

// The physical system of the AMR kernels that need more than linear
// operations on the conserved variables: primitives, a failed state, the
// CFL speed and the regrid sensors (system.rs / multiphase.rs).
struct AmrEulerPh {
    static constexpr int NV = 5, NS = 2;
    struct Ctx {
        Eos<double> e;
    };
    __device__ static Ctx ctx(const AmrDev& A) { return Ctx{Eos<double>::from(A.eos)}; }
    __device__ static void prim(const Ctx& c, const double* u, double* w) { to_prim(c.e, u, w); }
    // inadmissible (C/eos.rs:71-80): the admissible set of the scheme
    __device__ static bool bad(const Ctx& c, const double* w) { return !admissible(c.e, w[0], w[4]); }
    __device__ static double sound(const Ctx& c, const double* w) { return sound_speed(c.e, w[0], w[4]); }
    __device__ static double vel(const double* w, int d) { return w[1 + d]; }
    // ln ρ, ln(p + p∞) (system.rs sensor)
    __device__ static void sensor(const Ctx& c, const double* w, double* s) {
        s[0] = log(fmax(w[0], 1e-300));
        s[1] = log(fmax(w[4] + c.e.p_inf, 1e-300));
    }
};
struct AmrFivePh {
    static constexpr int NV = 7, NS = 3;
    struct Ctx {
        Five f;
    };
    __device__ static Ctx ctx(const AmrDev& A) { return Ctx{Five::from(A.fsys)}; }
    __device__ static void prim(const Ctx& c, const double* u, double* w) { c.f.to_prim(u, w); }
    // a failed state: a non-finite value or a non-positive density (the
    // reference steps on through states slightly outside the model's
    // admissible set, which only the limiter keeps the one-sided updates in)
    __device__ static bool bad(const Ctx&, const double* w) {
        bool b = !(Five::rho(w) > 0.0);
#pragma unroll
        for (int k = 0; k < NF; k++) b = b || !isfinite(w[k]);
        return b;
    }
    __device__ static double sound(const Ctx& c, const double* w) { return c.f.sound_speed(w); }
    __device__ static double vel(const double* w, int d) { return w[F_IU + d]; }
    // ln ρ, ln(p + p∞ of the mixture), α1 (multiphase.rs:386-391)
    __device__ static void sensor(const Ctx& c, const double* w, double* s) {
        s[0] = log(fmax(Five::rho(w), 1e-300));
        s[1] = log(fmax(w[F_IP] + c.f.p_inf_mix(w), 1e-300));
        s[2] = w[F_IA];
    }
};

// SSP-RK3 stage update of the leaves (amr.rs:1476-1498) and, after the third
// stage, the CFL rate of the new state (amr.rs:1409-1427).
// `sc`: the coefficient form of the subcycled level step (amr.rs:1869-1877,
// a0·u0 + a1·(u + dt·r) with (a0, a1) = (0, 1), (3/4, 1/4), (1/3, 2/3)),
// which rounds differently from the global step's in stages 1 and 3. Its
// lists hold covered ancestors too, whose restricted data may leave the
// admissible set at sharp interfaces (6th-order restriction overshoots)
// without harm, so the sc form skips the stage-3 rate and admissibility
// reduction; the leaves are checked by amr_cfl after the step.
template <class PH>
__global__ void amr_rk(const AmrDev A, double* u0, const double* __restrict__ rhs, const int* __restrict__ leaves,
                       const int* __restrict__ level, const double* __restrict__ dxl, int stage, StepCtl* ctl,
                       int sc) {
    constexpr int NV = PH::NV;
    const int slot = leaves[blockIdx.x];
    const int l = level[slot];
    const double dt = ctl->dt;
    const int64_t n = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    const typename PH::Ctx e = PH::ctx(A);
    double rate = 0.0;
    int bad = 0;  // a non-finite or inadmissible new leaf state (stage 3)
    // a block holds at most 32³ cells: 32-bit index arithmetic
    const unsigned b2 = (unsigned)A.bd[2], b12 = (unsigned)A.bd[1] * b2;
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        const unsigned qq = (unsigned)q;
        const unsigned c0 = qq / b12, r12 = qq - c0 * b12, c1 = r12 / b2;
        const int64_t c[3] = {(int64_t)c0, (int64_t)c1, (int64_t)(r12 - c1 * b2)};
        const int64_t cell = (int64_t)slot * A.bcell + amr_cell(A, c);
        if constexpr (BOUNDS_CHECK) {
            if (slot < 0 || cell < 0 || cell >= A.ntot) {
                atomicOr(A.err, 4u);
                continue;
            }
        }
        // every operand first (the pool, u0 and the residual may alias as far
        // as the compiler knows, so loads would otherwise wait on stores)
        double un[NV], uu[NV], r[NV], b0[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const int64_t o = (int64_t)k * A.ntot + cell;
            uu[k] = A.u[o];
            r[k] = rhs[o];
            b0[k] = stage == 1 ? 0.0 : u0[o];
        }
#pragma unroll
        for (int k = 0; k < NV; k++) {
            const int64_t o = (int64_t)k * A.ntot + cell;
            double v;
            if (stage == 1) {
                u0[o] = uu[k];
                v = sc ? 0.0 * uu[k] + 1.0 * (uu[k] + dt * r[k]) : uu[k] + dt * r[k];
            } else if (stage == 2) {
                v = 0.75 * b0[k] + 0.25 * (uu[k] + dt * r[k]);
            } else {
                v = sc ? (1.0 / 3.0) * b0[k] + 2.0 / 3.0 * (uu[k] + dt * r[k]) : b0[k] / 3.0 + 2.0 / 3.0 * (uu[k] + dt * r[k]);
            }
            A.u[o] = v;
            un[k] = v;
        }
        if (stage == 3 && !sc) {
            double w[NV];
            PH::prim(e, un, w);
            if (PH::bad(e, w)) bad = 1;
            const double cs = PH::sound(e, w);
            double s = -0.0;
            for (int i = 0; i < A.ndims; i++) {
                const int d = A.dims[i];
                s = s + (fabs(PH::vel(w, d)) + cs) / dxl[3 * l + d];
            }
            rate = fmax(rate, s);
        }
    }
    if (stage == 3 && !sc) {
        for (int o = 16; o > 0; o >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, o));
        __shared__ double sr[32];
        if ((threadIdx.x & 31) == 0) sr[threadIdx.x >> 5] = rate;
        const int any_bad = __syncthreads_or(bad);
        if (threadIdx.x == 0) {
            double v = sr[0];
            for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = fmax(v, sr[w]);
            if (!isnan(v) && v > 0.0) atomicMax(&ctl->rate_bits, (unsigned long long)__double_as_longlong(v));
            if (any_bad) atomicCAS(&ctl->status, 0, (int)EMG_ERR_INADMISSIBLE);
        }
    }
}

// CFL rate of the current leaves (amr.rs:1409-1427)
template <class PH>
__global__ void amr_cfl(const AmrDev A, const int* __restrict__ leaves, const int* __restrict__ level,
                        const double* __restrict__ dxl, StepCtl* ctl) {
    constexpr int NV = PH::NV;
    const int slot = leaves[blockIdx.x];
    const int l = level[slot];
    const int64_t n = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    const typename PH::Ctx e = PH::ctx(A);
    double rate = 0.0;
    int bad = 0;  // a non-finite or inadmissible leaf cell
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(q, A.bd, c);
        double uu[NV], w[NV];
        amr_load<NV>(A, slot, amr_cell(A, c), uu);
        PH::prim(e, uu, w);
        if (PH::bad(e, w)) bad = 1;
        const double cs = PH::sound(e, w);
        double s = -0.0;
        for (int i = 0; i < A.ndims; i++) {
            const int d = A.dims[i];
            s = s + (fabs(PH::vel(w, d)) + cs) / dxl[3 * l + d];
        }
        rate = fmax(rate, s);
    }
    for (int o = 16; o > 0; o >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, o));
    __shared__ double sr[32];
    if ((threadIdx.x & 31) == 0) sr[threadIdx.x >> 5] = rate;
    const int any_bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        double v = sr[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = fmax(v, sr[w]);
        if (!isnan(v) && v > 0.0) atomicMax(&ctl->rate_bits, (unsigned long long)__double_as_longlong(v));
        if (any_bad) atomicCAS(&ctl->status, 0, (int)EMG_ERR_INADMISSIBLE);
    }
}

// Dilatation limit of the five-equation CFL step over the leaves
// (dt_cfl, amr.rs:1426-1461): per cell the rate ρc²|∇·u| / (p + p∞ head)
// with ∇·u from the primitive velocities of the two neighbours along each
// active axis, read in the block or, across a block face, sampled from the
// hierarchy (the block's neighbour or its prediction). Max into *src_bits.
// A neighbour contributes only its velocity u_d = (ρu)_d/(α1ρ1 + α2ρ2), the
// value its primitive recovery computes (multiphase.rs:131-146), so a sampled
// neighbour predicts those three fields only. The cells of the block's
// interior (no neighbour outside the block) and those of its faces run in
// two kernels, so that a warp's sampled neighbours take the same branch.
// EDGE false: every neighbour lies in the block (the interior kernel)
template <bool EDGE>
__device__ __forceinline__ double five_cell_dilatation(const AmrDev& A, const Five& f, int slot, int l,
                                                       const int64_t* __restrict__ idx, const double* __restrict__ dxl,
                                                       const int64_t* c) {
    double uu[NF], w[NF];
    amr_load<NF>(A, slot, amr_cell(A, c), uu);
    f.to_prim(uu, w);
    double divu = 0.0;
    for (int i = 0; i < A.ndims; i++) {
        const int d = A.dims[i];
        double vv[2];
        for (int hi = 0; hi < 2; hi++) {
            int64_t cc[3] = {c[0], c[1], c[2]};
            cc[d] += hi ? 1 : -1;
            if (!EDGE || (cc[d] >= 0 && cc[d] < A.bd[d])) {
                const int64_t cell = amr_cell(A, cc);
                if (BOUNDS_CHECK && (cell < 0 || cell >= A.bcell || (int64_t)slot * A.bcell + cell >= A.ntot)) {
                    atomicOr(A.err, 4u);
                    vv[hi] = 0.0;
                    continue;
                }
                const double* p = A.u + (int64_t)slot * A.bcell + cell;
                vv[hi] = p[(int64_t)(F_IU + d) * A.ntot] / (p[0] + p[A.ntot]);
            } else if constexpr (EDGE) {
                int64_t g[3];
                for (int e = 0; e < 3; e++) g[e] = idx[3 * slot + e] * A.bd[e] + cc[e];
                const int qs[3] = {0, 1, F_IU + d};
                double v[3];
                amr_sample3_t<AMR_PREDICT_DEPTH, NF>(A, l, g, qs, v);
                vv[hi] = v[2] / (v[0] + v[1]);
            }
        }
        divu = divu + fabs(vv[1] - vv[0]) / (2.0 * dxl[3 * l + d]);
    }
    return f.dilatation_rate(w, divu);
}

__device__ __forceinline__ void five_src_max(double src, unsigned long long* src_bits) {
    for (int o = 16; o > 0; o >>= 1) src = fmax(src, __shfl_xor_sync(0xffffffffu, src, o));
    __shared__ double sr[32];
    if ((threadIdx.x & 31) == 0) sr[threadIdx.x >> 5] = src;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = sr[0];
        for (int w2 = 1; w2 < (int)(blockDim.x >> 5); w2++) v = fmax(v, sr[w2]);
        if (!isnan(v) && v > 0.0) atomicMax(src_bits, (unsigned long long)__double_as_longlong(v));
    }
}

// cells whose neighbours along every active axis lie in the block
__global__ void amr_dilatation_five(const AmrDev A, const int* __restrict__ leaves, const int* __restrict__ level,
                                    const int64_t* __restrict__ idx, const double* __restrict__ dxl,
                                    unsigned long long* src_bits) {
    const int slot = leaves[blockIdx.x];
    const int l = level[slot];
    int ni[3];
    for (int d = 0; d < 3; d++) ni[d] = A.act[d] ? A.bd[d] - 2 : 1;
    const int64_t n = (int64_t)ni[0] * ni[1] * ni[2];
    const Five f = Five::from(A.fsys);
    double src = 0.0;
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(q, ni, c);
        for (int d = 0; d < 3; d++)
            if (A.act[d]) c[d] += 1;
        src = fmax(src, five_cell_dilatation<false>(A, f, slot, l, idx, dxl, c));
    }
    five_src_max(src, src_bits);
}

// the cells of face blockIdx.y (axis dims[y/2], low or high side): cells on
// an edge belong to two or three faces and are evaluated once per face
__global__ void __launch_bounds__(128, 3) amr_dilatation_five_faces(const AmrDev A, const int* __restrict__ leaves, const int* __restrict__ level,
                                          const int64_t* __restrict__ idx, const double* __restrict__ dxl,
                                          unsigned long long* src_bits) {
    const int slot = leaves[blockIdx.x];
    const int l = level[slot];
    const int df = A.dims[blockIdx.y >> 1];
    const int side = blockIdx.y & 1;
    int nf[3];
    for (int d = 0; d < 3; d++) nf[d] = d == df ? 1 : (A.act[d] ? A.bd[d] : 1);
    const int64_t n = (int64_t)nf[0] * nf[1] * nf[2];
    const Five f = Five::from(A.fsys);
    double src = 0.0;
    for (int64_t q = blockIdx.z * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.z * blockDim.x) {
        int64_t c[3];
        box_coord(q, nf, c);
        c[df] = side ? A.bd[df] - 1 : 0;
        src = fmax(src, five_cell_dilatation<true>(A, f, slot, l, idx, dxl, c));
    }
    five_src_max(src, src_bits);
}

// ---------------------------------------------------------------- subcycling
// (amr.rs:1654-1954). One CTA per block of a level list, threads over the
// block's interior cells.

// step size of the level step in flight (read by the sweeps' limiter and the RK update)
__global__ void sc_set_dt(StepCtl* ctl, double dt) { ctl->dt = dt; }

// Level-l data as its linear interpolation in time, u ← (1−θ)·u0 + θ·u, the
// current data kept in `usave` (set_time_view, amr.rs:1702-1716); the ghost
// prediction of level l+1 reads block interiors only.
template <int NV>
__global__ void sc_time_view(const AmrDev A, const int* __restrict__ blist, const double* __restrict__ u0,
                             double* __restrict__ usave, double th) {
    const int slot = blist[blockIdx.x];
    const int64_t n = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    for (int64_t q = threadIdx.x; q < n; q += blockDim.x) {
        int64_t c[3];
        box_coord(q, A.bd, c);
        const int64_t cell = (int64_t)slot * A.bcell + amr_cell(A, c);
        if constexpr (BOUNDS_CHECK) {
            if (slot < 0 || cell < 0 || cell >= A.ntot) {
                atomicOr(A.err, 4u);
                continue;
            }
        }
        for (int k = 0; k < NV; k++) {
            const int64_t o = (int64_t)k * A.ntot + cell;
            const double uu = A.u[o];
            usave[o] = uu;
            A.u[o] = (1.0 - th) * u0[o] + th * uu;
        }
    }
}

// restore_time_view (amr.rs:1718-1723)
template <int NV>
__global__ void sc_restore(const AmrDev A, const int* __restrict__ blist, const double* __restrict__ usave) {
    const int slot = blist[blockIdx.x];
    const int64_t n = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    for (int64_t q = threadIdx.x; q < n; q += blockDim.x) {
        int64_t c[3];
        box_coord(q, A.bd, c);
        const int64_t cell = (int64_t)slot * A.bcell + amr_cell(A, c);
        if constexpr (BOUNDS_CHECK) {
            if (slot < 0 || cell < 0 || cell >= A.ntot) {
                atomicOr(A.err, 4u);
                continue;
            }
        }
        for (int k = 0; k < NV; k++) A.u[(int64_t)k * A.ntot + cell] = usave[(int64_t)k * A.ntot + cell];
    }
}

// A coarse–fine face of a level-l leaf whose same-level neighbour across
// (d, side) is refined (amr.rs:1725-1760, kind 0): its flux registers are rows
// `reg` of the register arrays (NV fields × npen face cells), fine[qa][qb] the
// adjacent level-(l+1) leaves per quarter of the face (−1: none).
struct ScFace {
    int slot, d, side, reg;
    double dx;
    int fine[2][2];
};

// coarse side: creg += w·F over the face (amr.rs:1774-1781)
template <int NV>
__global__ void sc_reg_coarse(const AmrDev A, const ScFace* __restrict__ tasks, const double* __restrict__ face, int npen,
                              double* creg, double w) {
    const ScFace tk = tasks[blockIdx.x];
    const int e0 = tk.d == 0 ? 1 : 0, e1 = tk.d == 2 ? 1 : 2;
    const int nf = A.bd[e0] * A.bd[e1];
    for (int pen = threadIdx.x; pen < nf; pen += blockDim.x) {
        const double* f = face + ((((int64_t)tk.slot * 3 + tk.d) * 2 + tk.side) * NV) * npen + pen;
        double* r = creg + (int64_t)tk.reg * NV * npen + pen;
        for (int k = 0; k < NV; k++) r[(int64_t)k * npen] = r[(int64_t)k * npen] + w * f[(int64_t)k * npen];
    }
}

// fine side: freg += w·F/nsub for the 2^(D−1) fine faces of each coarse face
// cell, in the order of the fine block's face loop (amr.rs:1782-1800)
template <int NV>
__global__ void sc_reg_fine(const AmrDev A, const ScFace* __restrict__ tasks, const double* __restrict__ face, int npen,
                            double* freg, double w, double nsub) {
    const ScFace tk = tasks[blockIdx.x];
    const int d = tk.d;
    const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
    const int b0 = A.bd[e0], b1 = A.bd[e1];
    for (int pen = threadIdx.x; pen < b0 * b1; pen += blockDim.x) {
        const int a = pen / b1, bb = pen % b1;
        double* r = freg + (int64_t)tk.reg * NV * npen + pen;
        for (int fa = 0; fa < (A.act[e0] ? 2 : 1); fa++)
            for (int fb = 0; fb < (A.act[e1] ? 2 : 1); fb++) {
                const int qa = A.act[e0] ? (2 * a + fa) / b0 : 0, qb = A.act[e1] ? (2 * bb + fb) / b1 : 0;
                const int cid = tk.fine[qa][qb];
                if (cid < 0) continue;
                const int la = A.act[e0] ? (2 * a + fa) % b0 : 0, lb = A.act[e1] ? (2 * bb + fb) % b1 : 0;
                const double* fv = face + ((((int64_t)cid * 3 + d) * 2 + (1 - tk.side)) * NV) * npen + la * b1 + lb;
                for (int k = 0; k < NV; k++) r[(int64_t)k * npen] = r[(int64_t)k * npen] + w * fv[(int64_t)k * npen] / nsub;
            }
    }
}

// reflux_level (amr.rs:1809-1834): u += ±(freg − creg)/dx on the face cells
// that received fine fluxes; launched per (d, side) bucket in order
template <int NV>
__global__ void sc_reflux(const AmrDev A, const ScFace* __restrict__ tasks, const double* __restrict__ creg,
                          const double* __restrict__ freg, int npen) {
    const ScFace tk = tasks[blockIdx.x];
    const int d = tk.d;
    const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
    const int b0 = A.bd[e0], b1 = A.bd[e1];
    for (int pen = threadIdx.x; pen < b0 * b1; pen += blockDim.x) {
        const int a = pen / b1, bb = pen % b1;
        const int qa = A.act[e0] ? (2 * a) / b0 : 0, qb = A.act[e1] ? (2 * bb) / b1 : 0;
        if (tk.fine[qa][qb] < 0) continue;
        int64_t c[3];
        c[d] = tk.side == 1 ? A.bd[d] - 1 : 0;
        c[e0] = a;
        c[e1] = bb;
        const int64_t cell = (int64_t)tk.slot * A.bcell + amr_cell(A, c);
        if constexpr (BOUNDS_CHECK) {
            if (tk.slot < 0 || cell < 0 || cell >= A.ntot) {
                atomicOr(A.err, 4u);
                continue;
            }
        }
        const double* fr = freg + (int64_t)tk.reg * NV * npen + pen;
        const double* cr = creg + (int64_t)tk.reg * NV * npen + pen;
        for (int k = 0; k < NV; k++) {
            const double df = fr[(int64_t)k * npen] - cr[(int64_t)k * npen];
            double* uo = A.u + (int64_t)k * A.ntot + cell;
            *uo = *uo + (tk.side == 1 ? -df / tk.dx : df / tk.dx);
        }
    }
}

// CFL rate of every block of a list (leaves and ancestors), reduced per level
// (dt_cfl_level, amr.rs:1657-1679)
template <class PH>
__global__ void sc_cfl_levels(const AmrDev A, const int* __restrict__ blist, const int* __restrict__ level,
                              const double* __restrict__ dxl, unsigned long long* rate_bits) {
    constexpr int NV = PH::NV;
    const int slot = blist[blockIdx.x];
    const int l = level[slot];
    const int64_t n = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    const typename PH::Ctx e = PH::ctx(A);
    double rate = 0.0;
    for (int64_t q = threadIdx.x; q < n; q += blockDim.x) {
        int64_t c[3];
        box_coord(q, A.bd, c);
        double uu[NV], w[NV];
        amr_load<NV>(A, slot, amr_cell(A, c), uu);
        PH::prim(e, uu, w);
        const double cs = PH::sound(e, w);
        double sp = -0.0;
        for (int i = 0; i < A.ndims; i++) {
            const int d = A.dims[i];
            sp = sp + (fabs(PH::vel(w, d)) + cs) / dxl[3 * l + d];
        }
        rate = fmax(rate, sp);
    }
    for (int o = 16; o > 0; o >>= 1) rate = fmax(rate, __shfl_xor_sync(0xffffffffu, rate, o));
    __shared__ double sr[32];
    if ((threadIdx.x & 31) == 0) sr[threadIdx.x >> 5] = rate;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = sr[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = fmax(v, sr[w]);
        if (!isnan(v) && v > 0.0) atomicMax(&rate_bits[l], (unsigned long long)__double_as_longlong(v));
    }
}

// Largest relative wavelet detail of each leaf on the system's sensors
// (block_detail, amr.rs:823-867), over its filled ghost-extended box.
template <class PH>
__device__ __forceinline__ void amr_sensor(const AmrDev& A, const typename PH::Ctx& e, const double* u, int64_t cell,
                                           double* s) {
    double q[PH::NV], w[PH::NV];
    for (int k = 0; k < PH::NV; k++) q[k] = u[(int64_t)k * A.ntot + cell];
    PH::prim(e, q, w);
    PH::sensor(e, w, s);
}
template <class PH>
__global__ void amr_detail(const AmrDev A, const int* __restrict__ leaves, unsigned long long* det_bits) {
    constexpr int NS = PH::NS;
    const int slot = leaves[blockIdx.x];
    const int64_t n = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    const typename PH::Ctx e = PH::ctx(A);
    const double* u = A.u + (int64_t)slot * A.bcell;
    const int offs[6] = {-5, -3, -1, 1, 3, 5};
    double mx = 0.0;
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.y * blockDim.x) {
        int64_t c[3];
        box_coord(q, A.bd, c);
        const int64_t cell = amr_cell(A, c);
        double s0[NS];
        amr_sensor<PH>(A, e, u, cell, s0);
        for (int i = 0; i < A.ndims; i++) {
            const int d = A.dims[i];
            const int64_t stride = d == 0 ? (int64_t)A.ext[1] * A.ext[2] : (d == 1 ? A.ext[2] : 1);
            double pred[NS];
            for (int k = 0; k < NS; k++) pred[k] = 0.0;
            for (int m = 0; m < 6; m++) {
                double sv[NS];
                amr_sensor<PH>(A, e, u, cell + offs[m] * stride, sv);
                for (int k = 0; k < NS; k++) pred[k] = pred[k] + A.wr[m] * sv[k];
            }
            for (int k = 0; k < NS; k++) {
                const double dd = fabs(s0[k] - pred[k]);
                mx = isfinite(dd) ? fmax(mx, dd) : INFINITY;
            }
        }
    }
    // max over the CTA; +inf orders above every finite bit pattern
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __shared__ double sr[32];
    if ((threadIdx.x & 31) == 0) sr[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = sr[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) v = fmax(v, sr[w]);
        atomicMax(&det_bits[slot], (unsigned long long)__double_as_longlong(v));
    }
}

// block moves (to, from) of the swap-removes of a batch of coarsenings
// (amr.rs:1024-1031): every source lies above every
// destination, so the moves are independent. grid = (moves, chunks of cells)
template <int NV>
__global__ void pool_move_list(const AmrDev A, const int* __restrict__ moves) {
    const int to = moves[2 * blockIdx.x], from = moves[2 * blockIdx.x + 1];
    for (int64_t q = blockIdx.y * (int64_t)blockDim.x + threadIdx.x; q < A.bcell; q += (int64_t)gridDim.y * blockDim.x)
        for (int k = 0; k < NV; k++)
            A.u[(int64_t)k * A.ntot + (int64_t)to * A.bcell + q] = A.u[(int64_t)k * A.ntot + (int64_t)from * A.bcell + q];
}

// interior cells of one block from host AoS data (initial condition)
template <int NV>
__global__ void pool_put_interior(const AmrDev A, int slot, const double* __restrict__ aos) {
    const int64_t n = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        int64_t c[3];
        box_coord(q, A.bd, c);
        const int64_t cell = (int64_t)slot * A.bcell + amr_cell(A, c);
        for (int k = 0; k < NV; k++) A.u[(int64_t)k * A.ntot + cell] = aos[NV * q + k];
    }
}

// interior cells of all blocks into AoS [block][cell][NV]
template <int NV>
__global__ void pool_get_interior(const AmrDev A, int nblocks, double* __restrict__ aos) {
    const int64_t nb = (int64_t)A.bd[0] * A.bd[1] * A.bd[2];
    const int64_t n = nb * nblocks;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t slot = t / nb, q = t % nb;
        int64_t c[3];
        box_coord(q, A.bd, c);
        const int64_t cell = slot * A.bcell + amr_cell(A, c);
        for (int k = 0; k < NV; k++) aos[NV * t + k] = A.u[(int64_t)k * A.ntot + cell];
    }
}

}  // namespace emg
