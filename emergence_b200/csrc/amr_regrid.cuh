// Regrid decisions and hierarchy edits on the device (Amr::regrid,
// fluid/crates/compressible/src/amr.rs:870-1106): refinement flags from the
// wavelet details, the one-block buffer, refinement with 2:1 balance, and the
// coarsening batches with their swap-remove compaction, applied to a device
// copy of the tree (level, key and leaf flag per block id, and the dense block
// map). The flags, the buffer, the coarsening candidates and the coarsening
// checks are one thread per block or candidate; the refinements and the edits
// of a coarsening batch keep the reference's sequential order (block ids
// follow the order of its recursive refine_block and of its swap-removes) and
// run on one thread of one CTA, with the block map in shared memory when it
// fits. Every loop is bounded by the block capacity (one block id per map
// slot) and the refinement recursion by the level count.
#pragma once
#include "amr_dev.cuh"

namespace emg {

constexpr int RG_MAX_STACK = AMR_MAX_LEVELS + 1;

// The device tree. `cap` = total map slots over all levels: a block id per
// slot at most, so appended blocks never exceed it.
struct RgTree {
    int* level;     // [cap]
    int64_t* idx;   // [cap][3]
    int* leaf;      // [cap]
    int* map;       // the device block map (A.map, writable)
    int* count;     // [0] blocks, [1] refinement events, [3] error (0: none), [4] coarsening
                    // candidates, [5] parents of the decided batch, [6] moves of the applied batch
    int cap;
};

struct RgGeom {
    int act[3];
    int64_t nb0[3];
    int levels;
    int64_t mapoff[AMR_MAX_LEVELS];
    int64_t mapsize;
    int periodic[3];
};

__device__ __forceinline__ int64_t rg_nbl(const RgGeom& G, int l, int d) { return G.act[d] ? (G.nb0[d] << l) : 1; }

// map slot of (l, key) or −1
__device__ __forceinline__ int64_t rg_slot(const RgGeom& G, int l, const int64_t* k) {
    if (l < 0 || l >= G.levels) return -1;
    int64_t s = 0;
    for (int d = 0; d < 3; d++) {
        const int64_t n = rg_nbl(G, l, d);
        if (k[d] < 0 || k[d] >= n) return -1;
        s = s * n + k[d];
    }
    return G.mapoff[l] + s;
}

// neighbour o (0..26, the reference's a, b, c loop order) of key k at level l
// with periodic wrap; false when o is the centre, moves along an inactive axis
// or leaves the domain through a non-periodic side (neighbours, amr.rs:918-947)
__device__ __forceinline__ bool rg_neighbour(const RgGeom& G, int l, const int64_t* k, int o, int64_t* nk) {
    const int off[3] = {o / 9 - 1, (o / 3) % 3 - 1, o % 3 - 1};
    if (off[0] == 0 && off[1] == 0 && off[2] == 0) return false;
    for (int d = 0; d < 3; d++) {
        if (!G.act[d] && off[d] != 0) return false;
        nk[d] = k[d] + off[d];
        const int64_t n = rg_nbl(G, l, d);
        if (nk[d] < 0 || nk[d] >= n) {
            if (!G.periodic[d]) return false;
            nk[d] = amr_erem(nk[d], n);
        }
    }
    return true;
}

// child c (0 .. 2^D − 1, the reference's children order: lower axes vary
// slowest) of key k
__device__ __forceinline__ void rg_child(const RgGeom& G, const int64_t* k, int c, int64_t* ck) {
    int bit = 0;
    int o[3] = {0, 0, 0};
    for (int d = 2; d >= 0; d--)
        if (G.act[d]) o[d] = (c >> bit++) & 1;
    for (int d = 0; d < 3; d++) ck[d] = G.act[d] ? 2 * k[d] + o[d] : 0;
}

__device__ __forceinline__ int rg_nkids(const RgGeom& G) { return 1 << (G.act[0] + G.act[1] + G.act[2]); }

// flags (amr.rs:877-892) from the detail bits of each block
__global__ void rg_flags(RgTree T, const unsigned long long* __restrict__ det_bits, int nb, int levels, double eps,
                         signed char* f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const double det = __longlong_as_double((long long)det_bits[i]);
    signed char v = 0;
    if (T.leaf[i]) {
        if (det > eps && T.level[i] + 1 < levels)
            v = 1;
        else if (det < eps / 128.0)
            v = -1;
    }
    f[i] = v;
}

// the refinement wish list with its one-block buffer (amr.rs:1051-1063): a
// block flagged for refinement and every same-level leaf neighbour of one
__global__ void rg_want(RgTree T, RgGeom G, const signed char* __restrict__ f, int nb, signed char* want) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nb) return;
    signed char w = f[j] > 0;
    if (!w && T.leaf[j]) {
        const int l = T.level[j];
        const int64_t* k = T.idx + 3 * j;
        for (int o = 0; o < 27 && !w; o++) {
            int64_t nk[3];
            if (!rg_neighbour(G, l, k, o, nk)) continue;
            const int64_t s = rg_slot(G, l, nk);
            const int i = s < 0 ? -1 : T.map[s];
            if (i >= 0 && f[i] > 0) w = 1;
        }
    }
    want[j] = w;
}

struct RgMap {
    int* m;
    __device__ __forceinline__ int get(const RgGeom& G, int l, const int64_t* k) const {
        const int64_t s = rg_slot(G, l, k);
        return s < 0 ? -1 : m[s];
    }
    __device__ __forceinline__ void set(const RgGeom& G, int l, const int64_t* k, int id) const {
        const int64_t s = rg_slot(G, l, k);
        if (s >= 0) m[s] = id;
    }
};

// the block map in dynamic shared memory when it fits (copied in and out by the CTA)
__device__ __forceinline__ RgMap rg_map_begin(const RgTree& T, const RgGeom& G, int* smem, bool in_smem) {
    if (!in_smem) return RgMap{T.map};
    for (int64_t s = threadIdx.x; s < G.mapsize; s += blockDim.x) smem[s] = T.map[s];
    __syncthreads();
    return RgMap{smem};
}
__device__ __forceinline__ void rg_map_end(const RgTree& T, const RgGeom& G, const int* smem, bool in_smem) {
    __syncthreads();
    if (!in_smem) return;
    for (int64_t s = threadIdx.x; s < G.mapsize; s += blockDim.x) T.map[s] = smem[s];
}

// Refinements (amr.rs:952-1011, 1064-1076): every wanted block of the
// original hierarchy (ids < nb0) in (level, key) order, each with the
// recursive refinement of coarser neighbours that keeps the 2:1 balance.
// Appends the children (leaves) and writes one event (parent id, first
// child id, parent level) per refinement. One working thread.
__global__ void rg_refine(RgTree T, RgGeom G, const signed char* __restrict__ want, int nb0, int in_smem,
                          int* events) {
    extern __shared__ int rg_smem[];
    const RgMap M = rg_map_begin(T, G, rg_smem, in_smem != 0);
    if (threadIdx.x == 0) {
        int nb = T.count[0];
        int nev = 0;
        const int nk = rg_nkids(G);
        struct Frame {
            int id, l, nbr;
            int64_t k[3];
        };
        Frame st[RG_MAX_STACK];
        for (int l = 0; l + 1 < G.levels; l++) {
            const int64_t n = rg_nbl(G, l, 0) * rg_nbl(G, l, 1) * rg_nbl(G, l, 2);
            for (int64_t s = 0; s < n; s++) {
                const int id = M.m[G.mapoff[l] + s];
                if (id < 0 || id >= nb0 || !want[id]) continue;
                int sp = 0;
                st[sp++] = Frame{id, l, 0, {T.idx[3 * id], T.idx[3 * id + 1], T.idx[3 * id + 2]}};
                while (sp > 0) {
                    Frame& F = st[sp - 1];
                    if (F.nbr == 0 && !T.leaf[F.id]) {  // refine_block: a non-leaf returns at once
                        sp--;
                        continue;
                    }
                    bool pushed = false;
                    if (F.l > 0) {
                        while (F.nbr < 27 && !pushed) {
                            int64_t nkey[3];
                            const int o = F.nbr++;
                            if (!rg_neighbour(G, F.l, F.k, o, nkey)) continue;
                            if (M.get(G, F.l, nkey) >= 0) continue;
                            for (int m = F.l - 1; m >= 0; m--) {
                                int64_t pk[3];
                                for (int d = 0; d < 3; d++) pk[d] = G.act[d] ? (nkey[d] >> (F.l - m)) : 0;
                                const int pid = M.get(G, m, pk);
                                if (pid >= 0) {
                                    if (sp < RG_MAX_STACK)
                                        st[sp++] = Frame{pid, m, 0, {pk[0], pk[1], pk[2]}};
                                    else
                                        T.count[3] = 1;  // deeper than the level count: cannot happen
                                    pushed = true;
                                    break;
                                }
                            }
                        }
                    }
                    if (pushed) continue;
                    Frame& G2 = st[sp - 1];
                    const int pid = M.get(G, G2.l, G2.k);
                    if (pid >= 0 && T.leaf[pid] && nb + nk <= T.cap) {
                        const int first = nb;
                        for (int c = 0; c < nk; c++) {
                            int64_t ck[3];
                            rg_child(G, G2.k, c, ck);
                            T.level[nb] = G2.l + 1;
                            for (int d = 0; d < 3; d++) T.idx[3 * nb + d] = ck[d];
                            T.leaf[nb] = 1;
                            nb++;
                        }
                        T.leaf[pid] = 0;
                        for (int c = 0; c < nk; c++) M.set(G, G2.l + 1, T.idx + 3 * (first + c), first + c);
                        events[3 * nev] = pid;
                        events[3 * nev + 1] = first;
                        events[3 * nev + 2] = G2.l;
                        nev++;
                    } else if (pid >= 0 && T.leaf[pid]) {
                        T.count[3] = 2;  // capacity (cannot happen: one id per map slot)
                    }
                    sp--;
                }
            }
        }
        T.count[0] = nb;
        T.count[1] = nev;
    }
    rg_map_end(T, G, rg_smem, in_smem != 0);
}

// Coarsening candidates (amr.rs:1077-1094) of the refined hierarchy: the
// ancestors whose children are all unprotected leaves flagged −1, with
// `prot(j)` = j < nb0 and want[j] (the wish list of the refinement pass).
// One thread per block marks them; rg_compact lists their keys
// [level, k0, k1, k2] in id order (ids move during the edits) and their count
// in T.count[4].
__global__ void rg_candidate_flags(RgTree T, RgGeom G, const signed char* __restrict__ f,
                                   const signed char* __restrict__ want, int nb0, signed char* mark) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int nb = T.count[0];
    if (b >= nb) return;
    const RgMap M{T.map};
    const int nk = rg_nkids(G);
    bool ok = !T.leaf[b];
    for (int c = 0; c < nk && ok; c++) {
        int64_t ck[3];
        rg_child(G, T.idx + 3 * b, c, ck);
        const int j = M.get(G, T.level[b] + 1, ck);
        ok = j >= 0 && T.leaf[j] && f[j] < 0 && !(j < nb0 && want[j]);
    }
    mark[b] = ok ? 1 : 0;
}

// Keys of the marked blocks in id order (one CTA: a contiguous range of ids
// per thread, an exclusive scan of the per-thread counts).
constexpr int RG_SCAN_T = 1024;
__global__ void __launch_bounds__(RG_SCAN_T) rg_compact(RgTree T, const signed char* __restrict__ mark, int64_t* ckey) {
    __shared__ int cnt[RG_SCAN_T];
    const int nb = T.count[0];
    const int per = (nb + RG_SCAN_T - 1) / RG_SCAN_T;
    const int b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
    int n = 0;
    for (int b = b0; b < b1; b++) n += mark[b];
    cnt[threadIdx.x] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int t = 0; t < RG_SCAN_T; t++) {
            const int v = cnt[t];
            cnt[t] = acc;
            acc += v;
        }
        T.count[4] = acc;
    }
    __syncthreads();
    int o = cnt[threadIdx.x];
    for (int b = b0; b < b1; b++) {
        if (!mark[b]) continue;
        ckey[4 * o] = T.level[b];
        for (int d = 0; d < 3; d++) ckey[4 * o + 1 + d] = T.idx[3 * b + d];
        o++;
    }
}

// Whether each level-l candidate may coarsen: no neighbour has a refined
// child (amr.rs:1097-1102), on the hierarchy as it is before the level's
// batch; one thread per candidate.
__global__ void rg_decide_flags(RgTree T, RgGeom G, const int64_t* __restrict__ ckey, int l, signed char* okc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.count[4]) return;
    if (ckey[4 * i] != l) {
        okc[i] = 0;
        return;
    }
    const RgMap M{T.map};
    const int nk = rg_nkids(G);
    const int64_t* key = ckey + 4 * i + 1;
    bool ok = true;
    for (int o = 0; o < 27 && ok; o++) {
        int64_t nkey[3];
        if (!rg_neighbour(G, l, key, o, nkey)) continue;
        for (int c = 0; c < nk && ok; c++) {
            int64_t ck[3];
            rg_child(G, nkey, c, ck);
            const int j = M.get(G, l + 1, ck);
            if (j >= 0 && !T.leaf[j]) ok = false;
        }
    }
    okc[i] = ok && M.get(G, l, key) >= 0;
}

// The coarsening batch of level l (amr.rs:1095-1104, in candidate order):
// the candidates that rg_decide_flags let through. Writes per batch parent
// (pre-batch id, k0, k1, k2) to `par`, and rem[id] = the batch position of
// the parent that removes fine block id (INT32_MAX: kept), for the
// restrictions, which run on the pool as it is before the batch. The count
// to T.count[5].
__global__ void rg_decide(RgTree T, RgGeom G, const int64_t* __restrict__ ckey, const signed char* __restrict__ okc,
                          int l, int64_t* par, int* rem) {
    const int nb = T.count[0];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) rem[i] = 0x7fffffff;
    __syncthreads();
    if (threadIdx.x == 0) {
        const RgMap M{T.map};
        const int nk = rg_nkids(G);
        const int nc = T.count[4];
        int n = 0;
        for (int i = 0; i < nc; i++) {
            if (!okc[i]) continue;
            const int64_t* key = ckey + 4 * i + 1;
            const int pid = M.get(G, l, key);
            par[4 * n] = pid;
            for (int d = 0; d < 3; d++) par[4 * n + 1 + d] = key[d];
            for (int c = 0; c < nk; c++) {
                int64_t ck[3];
                rg_child(G, key, c, ck);
                const int j = M.get(G, l + 1, ck);
                if (j >= 0) rem[j] = n;
            }
            n++;
        }
        T.count[5] = n;
    }
}

// The edits of a decided batch (amr.rs:1014-1032): each parent becomes a
// leaf and its children are swap-removed in descending id order; the moves
// (to, from) of the compaction go to `moves`, their count to T.count[6].
__device__ void rg_apply_serial(const RgTree& T, const RgGeom& G, const RgMap& M, const int64_t* __restrict__ par, int l,
                                int* orig, int* moves) {
    int nb = T.count[0];
    const int n0 = nb;
    const int npar = T.count[5];
    const int nk = rg_nkids(G);
    for (int i = 0; i < n0; i++) orig[i] = i;
    for (int q = 0; q < npar; q++) {
        const int64_t* key = par + 4 * q + 1;
        const int pid = M.get(G, l, key);
        if (pid < 0) continue;
        T.leaf[pid] = 1;
        int ids[8];
        for (int c = 0; c < nk; c++) {
            int64_t ck[3];
            rg_child(G, key, c, ck);
            ids[c] = M.get(G, l + 1, ck);
        }
        for (int a = 1; a < nk; a++)  // descending ids
            for (int b2 = a; b2 > 0 && ids[b2] > ids[b2 - 1]; b2--) {
                const int t = ids[b2];
                ids[b2] = ids[b2 - 1];
                ids[b2 - 1] = t;
            }
        for (int c = 0; c < nk; c++) {
            const int i = ids[c];
            if (i < 0) continue;
            M.set(G, T.level[i], T.idx + 3 * i, -1);
            const int last = nb - 1;
            if (i != last) {
                T.level[i] = T.level[last];
                for (int d = 0; d < 3; d++) T.idx[3 * i + d] = T.idx[3 * last + d];
                T.leaf[i] = T.leaf[last];
                orig[i] = orig[last];
            }
            nb--;
            if (i < nb) M.set(G, T.level[i], T.idx + 3 * i, i);
        }
    }
    int nm = 0;
    for (int s2 = 0; s2 < nb; s2++)
        if (orig[s2] != s2) {
            moves[2 * nm] = s2;
            moves[2 * nm + 1] = orig[s2];
            nm++;
        }
    T.count[0] = nb;
    T.count[6] = nm;
}

__global__ void rg_apply(RgTree T, RgGeom G, const int64_t* __restrict__ par, int l, int in_smem, int* orig,
                         int* moves) {
    extern __shared__ int rg_smem[];
    const RgMap M = rg_map_begin(T, G, rg_smem, in_smem != 0);
    if (threadIdx.x == 0) rg_apply_serial(T, G, M, par, l, orig, moves);
    rg_map_end(T, G, rg_smem, in_smem != 0);
}

}  // namespace emg
