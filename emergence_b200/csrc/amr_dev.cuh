// Device side of the block-AMR solver: the hierarchy view used by the
// kernels, sampling with 6th-order prediction, and the box pipelines that
// predict fine boxes from the coarser level and restrict ancestors from the
// finer one.
//
// Every operator reproduces the arithmetic and order of the reference CPU
// solver (fluid/crates/compressible/src/amr.rs): `sample` (:384-439),
// `predict` (:589-613), `gather_box` + `bc_box` (:450-545), `predict_box`
// (:548-586) and `restrict_box` (:622-731), so that the device hierarchy
// evolves bit for bit like the CPU one.
#pragma once
#include "five_physics.cuh"
#include "physics.cuh"
#include <stdint.h>

namespace emg {

constexpr int AMR_MAX_LEVELS = 12;

// Hierarchy view (pointers into device memory owned by the host object).
struct AmrDev {
    double* u;             // pool: u[q*ntot + slot*bcell + ext cell]
    int64_t ntot;          // field stride
    int64_t bcell;         // cells per pool block (ghost-extended)
    int ext[3], bd[3], gof[3];
    int act[3];
    int ndims, dims[3];
    int ng;
    int levels;
    int64_t nb0[3];        // level-0 blocks per side
    const int* map;        // dense per-level block index (−1: absent)
    int64_t mapoff[AMR_MAX_LEVELS];
    int bc[3][2];
    double bcs[3][2][7];   // Dirichlet states (nv values)
    double wp[2][6];       // prediction weights by parity (amr.rs:307)
    double wr[6];          // centred restriction weights (amr.rs:308)
    double wrs[5][6];      // restriction weights by shift m (amr.rs:670-671)
    EosD eos;              // Euler system
    FiveSysD fsys;         // five-equation system
    int id_limit;          // block ids at or above it read as absent (predictions replaying a regrid's order)
    unsigned int* err;     // error word (depth overflow)
};

__device__ __forceinline__ int64_t amr_ediv(int64_t a, int64_t b) {
    int64_t q = a / b;
    return (a % b < 0) ? q - 1 : q;
}
__device__ __forceinline__ int64_t amr_erem(int64_t a, int64_t b) {
    int64_t r = a % b;
    return r < 0 ? r + b : r;
}

__device__ __forceinline__ int64_t amr_nbl(const AmrDev& A, int l, int d) { return A.act[d] ? (A.nb0[d] << l) : 1; }
__device__ __forceinline__ int64_t amr_nlevel(const AmrDev& A, int l, int d) {
    return A.act[d] ? A.nb0[d] * A.bd[d] * ((int64_t)1 << l) : 1;
}

// pool slot of block (l, key), or −1
__device__ __forceinline__ int amr_get(const AmrDev& A, int l, const int64_t* k) {
    if (l < 0 || l >= A.levels) return -1;
    int64_t s = 0;
    for (int d = 0; d < 3; d++) {
        const int64_t n = amr_nbl(A, l, d);
        if (k[d] < 0 || k[d] >= n) return -1;
        s = s * n + k[d];
    }
    const int id = A.map[A.mapoff[l] + s];
    return id < A.id_limit ? id : -1;
}

__device__ __forceinline__ int64_t amr_cell(const AmrDev& A, const int64_t* c) {
    return ((c[0] + A.gof[0]) * A.ext[1] + (c[1] + A.gof[1])) * A.ext[2] + (c[2] + A.gof[2]);
}

// NV: conserved variables per cell (5 Euler, 7 five-equation); the first
// momentum component is at amr_iu<NV>()
template <int NV> __host__ __device__ constexpr int amr_iu() { return NV == 5 ? 1 : 2; }

template <int NV = 5>
__device__ __forceinline__ void amr_load(const AmrDev& A, int slot, int64_t cell, double* v) {
    if constexpr (BOUNDS_CHECK) {
        // bounds-check build: a pool index outside the pool sets bit 4 of the error word
        const int64_t i = (int64_t)slot * A.bcell + cell;
        if (slot < 0 || cell < 0 || cell >= A.bcell || i >= A.ntot) {
            atomicOr(A.err, 4u);
#pragma unroll
            for (int q = 0; q < NV; q++) v[q] = 0.0;
            return;
        }
    }
    const double* p = A.u + (int64_t)slot * A.bcell + cell;
#pragma unroll
    for (int q = 0; q < NV; q++) v[q] = p[(int64_t)q * A.ntot];
}

template <int DEPTH, int NV> __device__ void amr_predict_t(const AmrDev& A, int l, const int64_t* g, double* out);

// Conserved value of global cell g at level l (amr.rs:384-439). Boundary
// kinds: periodic, outflow, reflect, Dirichlet (the characteristic kind is
// rejected when the solver is built). DEPTH bounds the chain of predictions
// from coarser levels (the reference recurses; with 2:1 balance and kept
// ancestors one level suffices in practice) so that no kernel recurses; a
// chain deeper than DEPTH sets the error word.
template <int DEPTH, int NV>
__device__ __forceinline__ void amr_sample_t(const AmrDev& A, int l, const int64_t* g_in, double* v) {
    int64_t g[3] = {g_in[0], g_in[1], g_in[2]};
    bool flip[3] = {false, false, false};
#pragma unroll
    for (int d = 2; d >= 0; d--) {
        if (!A.act[d]) {
            g[d] = 0;
            continue;
        }
        const int64_t n = amr_nlevel(A, l, d);
        if (g[d] < 0 || g[d] >= n) {
            const int side = g[d] >= n ? 1 : 0;
            const int kind = A.bc[d][side];
            if (kind == EMG_BC_PERIODIC) {
                g[d] = amr_erem(g[d], n);
            } else if (kind == EMG_BC_OUTFLOW) {
                g[d] = g[d] < 0 ? 0 : n - 1;
            } else if (kind == EMG_BC_REFLECT) {
                g[d] = side == 0 ? -1 - g[d] : 2 * n - 1 - g[d];
                flip[d] = true;
            } else {
#pragma unroll
                for (int q = 0; q < NV; q++) v[q] = A.bcs[d][side][q];
                return;
            }
        }
    }
    int64_t key[3], c[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        key[d] = A.act[d] ? amr_ediv(g[d], A.bd[d]) : 0;
        c[d] = A.act[d] ? amr_erem(g[d], A.bd[d]) : 0;
    }
    const int id = amr_get(A, l, key);
    if (id >= 0) {
        amr_load<NV>(A, id, amr_cell(A, c), v);
    } else {
        amr_predict_t<DEPTH, NV>(A, l, g, v);
    }
#pragma unroll
    for (int d = 0; d < 3; d++)
        if (flip[d]) v[amr_iu<NV>() + d] = -v[amr_iu<NV>() + d];
}

// Direct 6^D prediction of cell g (level l) from level l − 1 (amr.rs:589-613).
template <int DEPTH, int NV> __device__ void amr_predict_t(const AmrDev& A, int l, const int64_t* g, double* out) {
#pragma unroll
    for (int q = 0; q < NV; q++) out[q] = 0.0;
    if constexpr (DEPTH <= 0) {
        atomicOr(A.err, 1u);
        return;
    } else {
        if (l <= 0) {
            atomicOr(A.err, 1u);
            return;
        }
        int total = 1;
        for (int i = 0; i < A.ndims; i++) total *= 6;
        for (int s = 0; s < total; s++) {
            double w = 1.0;
            int64_t c[3] = {0, 0, 0};
            int rem = s;
            for (int i = 0; i < A.ndims; i++) {
                const int d = A.dims[i];
                const int k = rem % 6;
                rem /= 6;
                const int odd = (int)amr_erem(g[d], 2);
                const int64_t base = amr_ediv(g[d], 2) + (odd == 1 ? -2 : -3);
                c[d] = base + k;
                w = w * A.wp[odd][k];
            }
            double v[NV];
            amr_sample_t<DEPTH - 1, NV>(A, l - 1, c, v);
#pragma unroll
            for (int q = 0; q < NV; q++) out[q] = out[q] + w * v[q];
        }
    }
}

// The same sample and prediction for three of the NV fields only (indices
// qs[0..2]): each field's prediction is its own weighted sum in the same
// order, so the three values are those of amr_sample_t.
template <int DEPTH, int NV> __device__ void amr_predict3_t(const AmrDev& A, int l, const int64_t* g, const int* qs, double* out);

template <int DEPTH, int NV>
__device__ __forceinline__ void amr_sample3_t(const AmrDev& A, int l, const int64_t* g_in, const int* qs, double* v) {
    int64_t g[3] = {g_in[0], g_in[1], g_in[2]};
    bool flip[3] = {false, false, false};
#pragma unroll
    for (int d = 2; d >= 0; d--) {
        if (!A.act[d]) {
            g[d] = 0;
            continue;
        }
        const int64_t n = amr_nlevel(A, l, d);
        if (g[d] < 0 || g[d] >= n) {
            const int side = g[d] >= n ? 1 : 0;
            const int kind = A.bc[d][side];
            if (kind == EMG_BC_PERIODIC) {
                g[d] = amr_erem(g[d], n);
            } else if (kind == EMG_BC_OUTFLOW) {
                g[d] = g[d] < 0 ? 0 : n - 1;
            } else if (kind == EMG_BC_REFLECT) {
                g[d] = side == 0 ? -1 - g[d] : 2 * n - 1 - g[d];
                flip[d] = true;
            } else {
#pragma unroll
                for (int j = 0; j < 3; j++) v[j] = A.bcs[d][side][qs[j]];
                return;
            }
        }
    }
    int64_t key[3], c[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        key[d] = A.act[d] ? amr_ediv(g[d], A.bd[d]) : 0;
        c[d] = A.act[d] ? amr_erem(g[d], A.bd[d]) : 0;
    }
    const int id = amr_get(A, l, key);
    if (id >= 0) {
        const int64_t cell = amr_cell(A, c);
        if (BOUNDS_CHECK && (cell < 0 || cell >= A.bcell || (int64_t)id * A.bcell + cell >= A.ntot)) {
            atomicOr(A.err, 4u);
#pragma unroll
            for (int j = 0; j < 3; j++) v[j] = 0.0;
            return;
        }
        const double* p = A.u + (int64_t)id * A.bcell + cell;
#pragma unroll
        for (int j = 0; j < 3; j++) v[j] = p[(int64_t)qs[j] * A.ntot];
    } else {
        amr_predict3_t<DEPTH, NV>(A, l, g, qs, v);
    }
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int m = qs[j] - amr_iu<NV>();
        if (m >= 0 && m < 3 && flip[m]) v[j] = -v[j];
    }
}

template <int DEPTH, int NV> __device__ void amr_predict3_t(const AmrDev& A, int l, const int64_t* g, const int* qs, double* out) {
#pragma unroll
    for (int j = 0; j < 3; j++) out[j] = 0.0;
    if constexpr (DEPTH <= 0) {
        atomicOr(A.err, 1u);
        return;
    } else {
        if (l <= 0) {
            atomicOr(A.err, 1u);
            return;
        }
        // Fast path: the 6^D coarse stencil lies inside the domain and every
        // level-(l − 1) block it touches exists (at most two per axis, since a
        // block has at least 6 cells), so each coarse value is a plain load
        // from one of those blocks: the same values, weights and summation
        // order as the general loop below, without a key division and map
        // lookup per stencil point.
        {
            int64_t base[3] = {0, 0, 0}, kmin[3] = {0, 0, 0};
            int odd[3] = {0, 0, 0}, two[3] = {0, 0, 0};
            bool inside = true;
            for (int d = 0; d < 3; d++) {
                if (!A.act[d]) continue;
                odd[d] = (int)amr_erem(g[d], 2);
                base[d] = amr_ediv(g[d], 2) + (odd[d] == 1 ? -2 : -3);
                if (base[d] < 0 || base[d] + 5 >= amr_nlevel(A, l - 1, d)) inside = false;
                kmin[d] = amr_ediv(base[d], A.bd[d]);
                two[d] = amr_ediv(base[d] + 5, A.bd[d]) > kmin[d] ? 1 : 0;
            }
            int slot8[8];
            for (int t = 0; t < 8 && inside; t++) {
                const int j0 = t & 1, j1 = (t >> 1) & 1, j2 = t >> 2;
                if (j0 > two[0] || j1 > two[1] || j2 > two[2]) {
                    slot8[t] = -1;
                    continue;
                }
                const int64_t key[3] = {kmin[0] + j0, kmin[1] + j1, kmin[2] + j2};
                slot8[t] = amr_get(A, l - 1, key);
                if (slot8[t] < 0) inside = false;
            }
            if (inside) {
                int total = 1;
                for (int i = 0; i < A.ndims; i++) total *= 6;
                for (int s = 0; s < total; s++) {
                    double w = 1.0;
                    int jj[3] = {0, 0, 0};
                    int64_t lc[3] = {0, 0, 0};
                    int rem = s;
                    for (int i = 0; i < A.ndims; i++) {
                        const int d = A.dims[i];
                        const int k = rem % 6;
                        rem /= 6;
                        const int64_t c = base[d] + k - kmin[d] * A.bd[d];  // in [0, 2·bd)
                        jj[d] = c >= A.bd[d] ? 1 : 0;
                        lc[d] = c - jj[d] * A.bd[d];
                        w = w * A.wp[odd[d]][k];
                    }
                    const int slot = slot8[jj[0] + 2 * jj[1] + 4 * jj[2]];
                    const int64_t cell = amr_cell(A, lc);
                    if (BOUNDS_CHECK && (cell < 0 || cell >= A.bcell || (int64_t)slot * A.bcell + cell >= A.ntot)) {
                        atomicOr(A.err, 4u);
                        continue;
                    }
                    const double* p = A.u + (int64_t)slot * A.bcell + cell;
#pragma unroll
                    for (int j = 0; j < 3; j++) out[j] = out[j] + w * p[(int64_t)qs[j] * A.ntot];
                }
                return;
            }
        }
        int total = 1;
        for (int i = 0; i < A.ndims; i++) total *= 6;
        for (int s = 0; s < total; s++) {
            double w = 1.0;
            int64_t c[3] = {0, 0, 0};
            int rem = s;
            for (int i = 0; i < A.ndims; i++) {
                const int d = A.dims[i];
                const int k = rem % 6;
                rem /= 6;
                const int odd = (int)amr_erem(g[d], 2);
                const int64_t base = amr_ediv(g[d], 2) + (odd == 1 ? -2 : -3);
                c[d] = base + k;
                w = w * A.wp[odd][k];
            }
            double v[3];
            amr_sample3_t<DEPTH - 1, NV>(A, l - 1, c, qs, v);
#pragma unroll
            for (int j = 0; j < 3; j++) out[j] = out[j] + w * v[j];
        }
    }
}

constexpr int AMR_PREDICT_DEPTH = 3;
template <int NV = 5>
__device__ __forceinline__ void amr_sample(const AmrDev& A, int l, const int64_t* g, double* v, int) {
    amr_sample_t<AMR_PREDICT_DEPTH, NV>(A, l, g, v);
}

// ------------------------------------------------------------------ box pipelines
// A box is a row-major array of cells with its own size per axis; buffers
// ping-pong between passes. `val` holds NV doubles per cell (AoS within the
// box), `ok` one byte.

// Prediction of the level-l fine box [fmin, fmax] from level l − 1
// (predict_box, amr.rs:548-586), written to a target pool block.
struct PBox {
    int l;               // fine level
    int slot;            // target pool slot
    int64_t fmin[3];     // fine box, global cell coordinates at level l
    int64_t cmin[3];     // gathered coarse patch origin (level l − 1)
    int csz[3];          // coarse patch size
    int fsz[3];          // fine box size
    int t0[3];           // ext-local coordinates of fmin in the target block
    int64_t off;         // scratch offset (cells) of this box's buffers
    int64_t cap;         // cells per buffer
    int bcmask;          // bit di: the coarse patch crosses a non-periodic side along dims[di]
};

// Restriction of ancestor (l, idx) cells [lo, hi) from level l + 1
// (restrict_box, amr.rs:622-731), written into the ancestor's interior.
struct RBox {
    int l;               // coarse level
    int slot;            // ancestor pool slot
    int lo[3], hi[3];    // local cell box
    int64_t f0[3];       // fine patch origin (level l + 1)
    int sz[3];           // fine patch size
    int64_t off;         // scratch offset (cells)
    int64_t cap;         // cells per buffer
    int seq;             // position in a batch of coarsenings (-1: none)
    int fast;            // fine patch inside the domain over at most four blocks per axis
};

// thread → (box, cell) over a prefix-sum of box sizes
__device__ __forceinline__ int find_box(const int64_t* start, int nbox, int64_t t) {
    int lo = 0, hi = nbox;  // start[lo] <= t < start[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (start[mid] <= t)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

}  // namespace emg
