// Block-AMR solver: host object and C ABI (emg_amr_*), replacing
// compressible-cuda's GpuAmr (fluid/crates/compressible-cuda/src/amr.rs:95-858)
// for the Euler system.
//
// The block ids follow the reference CPU solver's (fluid/crates/compressible/
// src/amr.rs), so the device pool, indexed by block id, mirrors `Amr::blocks`.
// Regrid decisions and hierarchy edits (flags, buffer, 2:1-balanced
// refinement, coarsening with swap-remove compaction) run on the device
// (amr_regrid.cuh); the host keeps a mirror of the tree, read back after each
// regrid, from which it builds the launch lists. All numerical work —
// restriction of edge ancestors, the six face ghost slabs of every leaf
// (same-level copies, 6th-order prediction from the coarser level, boundary
// conditions; edge and corner ghost regions are never read), the fused WCNS
// sweeps of every leaf, refluxing, SSP-RK3, the CFL reduction, wavelet details
// and the data of refined / coarsened blocks — runs on the device; unlike the
// reference GPU path, a regrid never downloads the solution (only one detail
// value per block).
//
// Built with -fmad=false (FP64 arithmetic rounds as the reference CPU's).
#include "../../include/emergence_b200.h"
#include "amr_kernels.cuh"
#include "amr_regrid.cuh"
#include "five_launch.h"
#include "sweep_launch.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <set>
#include <string>
#include <tuple>
#include <vector>

namespace emg {
int set_error(int code, const std::string& msg);
}

using namespace emg;

// the instance of an AMR kernel template for a handle's system: NVK by the
// number of conserved variables, PHK by the system adapter
#define NVK(kern) (nv == 7 ? kern<7> : kern<5>)
#define PHK(kern) (nv == 7 ? kern<AmrFivePh> : kern<AmrEulerPh>)

#define AMR_CUDA(call)                                                                             \
    do {                                                                                           \
        cudaError_t _e = (call);                                                                   \
        if (_e != cudaSuccess)                                                                     \
            return set_error(EMG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e));  \
    } while (0)

namespace {

using Key = std::array<int64_t, 3>;

int64_t ediv(int64_t a, int64_t b) {
    int64_t q = a / b;
    return (a % b < 0) ? q - 1 : q;
}
int64_t erem(int64_t a, int64_t b) {
    int64_t r = a % b;
    return r < 0 ? r + b : r;
}

// C/amr.rs:41-47
std::array<double, 6> lagrange6(double x0, double x) {
    std::array<double, 6> w;
    for (int k = 0; k < 6; k++) {
        double xk = x0 + k, p = 1.0;
        for (int j = 0; j < 6; j++)
            if (j != k) p = p * ((x - (x0 + j)) / (xk - (x0 + j)));
        w[k] = p;
    }
    return w;
}

struct HBlock {
    int level;
    Key idx;
    bool leaf;
};

template <class T> struct DevVec {
    T* p = nullptr;
    size_t n = 0, cap = 0;
    // capacity for at least m elements (contents not kept)
    int grow(size_t m) {
        if (m <= cap) return EMG_OK;
        if (p) cudaFree(p);
        cap = std::max<size_t>(m, 2 * cap);
        if (cudaMalloc(&p, cap * sizeof(T)) != cudaSuccess) {
            p = nullptr;
            cap = n = 0;
            return set_error(EMG_ERR_CUDA, "device allocation failed");
        }
        return EMG_OK;
    }
    int put(const std::vector<T>& v, cudaStream_t s) {
        int rc = grow(v.size());
        if (rc) return rc;
        n = v.size();
        if (n && cudaMemcpyAsync(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice, s) != cudaSuccess)
            return set_error(EMG_ERR_CUDA, "upload failed");
        return EMG_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = cap = 0;
    }
};

}  // namespace

struct emg_amr {
    // ---- configuration
    emg_amr_config cfg{};
    emg_eos eos{};
    double lo[3]{}, hi[3]{};
    emg_bc7 bc[6]{};            // kinds and Dirichlet states (nv values)
    int nv = 5;                 // conserved variables per cell: 5 (Euler) or 7 (five-equation system)
    emg_five_system five{};     // the two phases of the five-equation system (nv = 7)
    emg_opts opts{};
    int act[3]{}, bd[3]{}, ext[3]{}, gof[3]{};
    std::vector<int> dims;
    int ng = 5;
    int64_t nb0[3]{};
    int levels = 1;
    std::vector<double> dxl;  // [level][3]
    double wp[2][6]{}, wr[6]{}, wrs[5][6]{};
    // ---- hierarchy (block ids as in the reference's Amr::blocks)
    std::vector<HBlock> blocks;
    std::vector<std::vector<int>> map;
    std::vector<int64_t> mapoff;
    double t = 0.0;
    int64_t steps = 0, regrid_interval = 0, next_regrid = 0;
    uint64_t faces = 0, weno_faces = 0;
    // ---- device
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t bcell = 0, cap = 0;  // pool capacity in blocks
    double *u = nullptr, *u0 = nullptr, *rhs = nullptr, *face = nullptr;
    int npen = 1;
    unsigned int* err = nullptr;
    StepCtl* ctl = nullptr;
    StepCtl* ctl_host = nullptr;
    double* scr[2] = {nullptr, nullptr};
    unsigned char* sok[2] = {nullptr, nullptr};
    int64_t scr_cap = 0;
    unsigned long long* det = nullptr;
    int64_t det_cap = 0;
    DevVec<int> dmap, dleaves, dlevel, dbcleaves;
    // chains of same-level leaves along each axis for the global sweeps
    DevVec<int> dchain_off[3], dchain_slot[3];
    int nchain[3] = {0, 0, 0};
    DevVec<int64_t> didx;
    DevVec<double> ddxl;
    DevVec<CopyTask> dcopy;
    DevVec<CopyTask> dcopy_sweep;  // the copies the chained sweeps read (no slab between two blocks of a chain)
    DevVec<PBox> dpbox;
    std::vector<DevVec<RBox>> drbox;  // per level
    DevVec<RefluxFace> dreflux;
    int rface_start[7]{};  // refluxing faces of bucket (d, side) = 2d + side: [rface_start[b], rface_start[b+1])
    DevVec<PBox> dtmp_pbox;    // one-off prediction boxes (refined children)
    DevVec<RBox> dtmp_rbox;    // one-off restriction boxes (coarsened parents)
    int amrP[3] = {0, 0, 0};      // tuned pencils per CTA of the sweeps (0: default)
    bool tuned = false;
    std::vector<PBox> pend_pbox;  // prediction boxes of refinements not yet launched
    int pend_level = -1;          // their parent level
    DevVec<double> dstage;     // host initial data of new blocks
    std::vector<int> rbox_count;
    int ncopy = 0, npbox = 0, nbcleaves = 0, nleaves = 0;
    int ncopy_sweep = 0;
    bool layout_valid = false, map_dirty = true;
    uint64_t launches = 0;
    double phase_ms[5]{};
    bool rate_valid = false;
    // ---- subcycling (C/amr.rs:1654-1954; host schedule in step_subcycled)
    struct ScLevel {
        int nblk = 0;                  // blocks of the level, leaves and ancestors, in id order
        DevVec<int> blist;
        DevVec<CopyTask> copies;       // face ghost slabs of those blocks
        DevVec<PBox> pboxes;
        DevVec<int> bcl;
        int ncopy = 0, npbox = 0, nbcl = 0;
        int64_t pmax = 0;
        DevVec<RBox> rfull;            // every ancestor of the level, whole block, chunk-relative offsets
        std::vector<int> rchunk;       // chunk starts into rfull (and its end)
        std::vector<int64_t> rchunk_max;
        DevVec<ScFace> faces;          // coarse–fine faces of its leaves (coarse side), by (d, side)
        DevVec<int> choff[3], chslot[3];  // chains of its blocks along each axis for the level's sweeps
        int nch[3] = {0, 0, 0};
        int face_start[7]{};
        int reg0 = 0;                  // their register rows [reg0, reg0 + nfaces)
    };
    std::vector<ScLevel> sc;
    uint64_t sc_gen = ~0ull;
    DevVec<int> dall;                  // every block, for the per-level CFL reduction
    double* usave = nullptr;           // time-view save area, pool-sized
    int64_t usave_cap = 0;
    double *creg = nullptr, *freg = nullptr;  // flux registers, nv × npen doubles per face
    int64_t reg_cap = 0;
    unsigned long long* level_rates = nullptr;
    std::vector<double> level_t0, level_dt;
    static constexpr int SC_RCHUNK = 256;  // whole-block restriction boxes per launch set

    // ---------------------------------------------------------------- geometry
    int64_t nbl(int l, int d) const { return act[d] ? nb0[d] << l : 1; }
    int64_t n_level(int l, int d) const { return act[d] ? nb0[d] * bd[d] * ((int64_t)1 << l) : 1; }
    int64_t bcells() const { return (int64_t)bd[0] * bd[1] * bd[2]; }
    int bckind(int d, int s) const { return bc[2 * d + s].kind; }

    // ---------------------------------------------------------------- index
    int64_t slot_of(int l, const Key& k) const {
        if (l < 0 || l >= levels) return -1;
        int64_t s = 0;
        for (int d = 0; d < 3; d++) {
            int64_t n = nbl(l, d);
            if (k[d] < 0 || k[d] >= n) return -1;
            s = s * n + k[d];
        }
        return s;
    }
    int get(int l, const Key& k) const {
        int64_t s = slot_of(l, k);
        return s < 0 ? -1 : map[l][s];
    }
    void insert(int l, const Key& k, int id) {
        int64_t s = slot_of(l, k);
        if (s >= 0) {
            map[l][s] = id;
            map_changed.push_back(mapoff[l] + s);
        }
        map_dirty = true;
        layout_valid = false;
    }
    void remove(int l, const Key& k) {
        int64_t s = slot_of(l, k);
        if (s >= 0) {
            map[l][s] = -1;
            map_changed.push_back(mapoff[l] + s);
        }
        map_dirty = true;
        layout_valid = false;
    }
    std::vector<int64_t> map_changed;  // flat map entries changed since the last upload
    bool map_uploaded = false;

    // same-level neighbour keys with periodic wrap (C/amr.rs:918-947)
    std::vector<Key> neighbours(int l, const Key& idx) const {
        std::vector<Key> out;
        int64_t nb[3];
        for (int d = 0; d < 3; d++) nb[d] = nbl(l, d);
        int r[3];
        for (int d = 0; d < 3; d++) r[d] = act[d] ? 1 : 0;
        for (int a = -r[0]; a <= r[0]; a++)
            for (int b = -r[1]; b <= r[1]; b++)
                for (int c = -r[2]; c <= r[2]; c++) {
                    if (!a && !b && !c) continue;
                    Key k = {idx[0] + a, idx[1] + b, idx[2] + c};
                    bool inside = true;
                    for (int d = 0; d < 3; d++)
                        if (k[d] < 0 || k[d] >= nb[d]) {
                            if (bckind(d, k[d] >= nb[d] ? 1 : 0) == EMG_BC_PERIODIC)
                                k[d] = erem(k[d], nb[d]);
                            else
                                inside = false;
                        }
                    if (inside) out.push_back(k);
                }
        return out;
    }
    // C/amr.rs:894-915
    std::vector<Key> children(const Key& idx) const {
        std::vector<Key> out = {Key{0, 0, 0}};
        for (int d = 0; d < 3; d++) {
            std::vector<Key> next;
            for (auto& c : out) {
                if (act[d]) {
                    for (int o = 0; o < 2; o++) {
                        Key cc = c;
                        cc[d] = 2 * idx[d] + o;
                        next.push_back(cc);
                    }
                } else {
                    Key cc = c;
                    cc[d] = 0;
                    next.push_back(cc);
                }
            }
            out = next;
        }
        return out;
    }
    bool is_edge_ancestor(int i) const {  // C/amr.rs:741-744
        const HBlock& b = blocks[i];
        if (b.leaf) return false;
        for (auto& nk : neighbours(b.level, b.idx)) {
            int j = get(b.level, nk);
            if (j < 0 || blocks[j].leaf) return true;
        }
        return false;
    }

    // ---------------------------------------------------------------- device helpers
    AmrDev view() const {
        AmrDev A{};
        A.u = u;
        A.ntot = cap * bcell;
        A.bcell = bcell;
        for (int d = 0; d < 3; d++) {
            A.ext[d] = ext[d];
            A.bd[d] = bd[d];
            A.gof[d] = gof[d];
            A.act[d] = act[d];
            A.nb0[d] = nb0[d];
            for (int s = 0; s < 2; s++) {
                A.bc[d][s] = bckind(d, s);
                for (int k = 0; k < 7; k++) A.bcs[d][s][k] = k < nv ? bc[2 * d + s].state[k] : 0.0;
            }
        }
        A.ndims = (int)dims.size();
        for (int i = 0; i < 3; i++) A.dims[i] = i < A.ndims ? dims[i] : 0;
        A.ng = ng;
        A.levels = levels;
        A.map = dmap.p;
        for (int l = 0; l < levels && l < AMR_MAX_LEVELS; l++) A.mapoff[l] = mapoff[l];
        std::memcpy(A.wp, wp, sizeof wp);
        std::memcpy(A.wr, wr, sizeof wr);
        std::memcpy(A.wrs, wrs, sizeof wrs);
        A.eos = EosD{eos.gamma, eos.p_inf, eos.b, eos.q};
        for (int k = 0; k < 2; k++) A.fsys.e[k] = EosD{five.eos[k].gamma, five.eos[k].p_inf, five.eos[k].b, five.eos[k].q};
        A.fsys.kapila = five.kapila;
        A.id_limit = id_limit;
        A.err = err;
        return A;
    }

    // Device copy of the block map: the whole map on first use, afterwards only
    // the entries changed since (a regrid edits a few entries per refinement).
    int upload_map() {
        if (!map_dirty) return EMG_OK;
        size_t total = 0;
        for (auto& m : map) total += m.size();
        if (!map_uploaded || map_changed.size() * 8 > total) {
            std::vector<int> flat;
            flat.reserve(total);
            for (auto& m : map) flat.insert(flat.end(), m.begin(), m.end());
            int rc = dmap.put(flat, stream);
            if (rc) return rc;
            map_uploaded = true;
        } else if (!map_changed.empty()) {
            std::sort(map_changed.begin(), map_changed.end());
            map_changed.erase(std::unique(map_changed.begin(), map_changed.end()), map_changed.end());
            std::vector<int64_t> pairs;
            pairs.reserve(2 * map_changed.size());
            for (int64_t f : map_changed) {
                int l = 0;
                while (l + 1 < levels && mapoff[l + 1] <= f) l++;
                pairs.push_back(f);
                pairs.push_back(map[l][f - mapoff[l]]);
            }
            int rc = dmap_edits.put(pairs, stream);
            if (rc) return rc;
            const int n = (int)map_changed.size();
            map_scatter<<<(n + 255) / 256, 256, 0, stream>>>(dmap.p, dmap_edits.p, n);
            launches++;
            AMR_CUDA(cudaGetLastError());
        }
        map_changed.clear();
        map_dirty = false;
        return EMG_OK;
    }
    DevVec<int64_t> dmap_edits;

    // grow the pool to hold at least n blocks, preserving block data
    int reserve(int64_t n) {
        if (n <= cap) return EMG_OK;
        int64_t nc = std::max<int64_t>(n, cap + cap / 2 + 16);
        double *nu = nullptr, *nu0 = nullptr, *nr = nullptr, *nf = nullptr;
        const size_t bytes = (size_t)nc * bcell * nv * sizeof(double);
        const size_t fbytes = (size_t)nc * 3 * 2 * nv * npen * sizeof(double);
        if (cudaMalloc(&nu, bytes) != cudaSuccess || cudaMalloc(&nu0, bytes) != cudaSuccess ||
            cudaMalloc(&nr, bytes) != cudaSuccess || cudaMalloc(&nf, fbytes) != cudaSuccess) {
            cudaFree(nu);
            cudaFree(nu0);
            cudaFree(nr);
            cudaFree(nf);
            cudaGetLastError();
            return set_error(EMG_ERR_CUDA, "AMR pool allocation failed");
        }
        cudaMemsetAsync(nu, 0, bytes, stream);
        cudaMemsetAsync(nr, 0, bytes, stream);
        cudaMemsetAsync(nf, 0, fbytes, stream);
        if (u) {
            // fields are strided by the capacity: copy field by field
            for (int k = 0; k < nv; k++)
                AMR_CUDA(cudaMemcpyAsync(nu + (size_t)k * nc * bcell, u + (size_t)k * cap * bcell,
                                         (size_t)cap * bcell * sizeof(double), cudaMemcpyDeviceToDevice, stream));
        }
        AMR_CUDA(cudaStreamSynchronize(stream));
        cudaFree(u);
        cudaFree(u0);
        cudaFree(rhs);
        cudaFree(face);
        u = nu;
        u0 = nu0;
        rhs = nr;
        face = nf;
        cap = nc;
        return EMG_OK;
    }

    // Growing the pool reallocates and copies it (hundreds of ms for a pool of
    // 10 GB), and every regrid that refines holds the new children before the
    // coarsened blocks are removed. The pool therefore starts with room for
    // twice the initial hierarchy, when old and new pool fit in half of the
    // free device memory.
    int reserve_headroom() {
        int rc = EMG_OK;
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            fr = 0;
        }
        const int64_t want = 2 * (int64_t)blocks.size();
        const size_t per_block = (size_t)bcell * nv * sizeof(double) * 3 + (size_t)3 * 2 * nv * npen * sizeof(double);
        if (want > cap && (size_t)(want + cap) * per_block <= fr / 2 && (rc = reserve(want))) return rc;
        // the block lists of the layout and of regrids likewise, so that a
        // regrid allocates nothing (an allocation or free in the middle of a
        // run stalls the host for milliseconds, at times for hundreds)
        if ((rc = ensure_layout())) return rc;
        const size_t nb = blocks.size();
        if ((rc = dleaves.grow(2 * nb)) || (rc = dlevel.grow(2 * nb)) || (rc = didx.grow(6 * nb)) ||
            (rc = dbcleaves.grow(2 * nb)) || (rc = dcopy.grow(2 * dcopy.n)) || (rc = dcopy_sweep.grow(2 * dcopy.n)) || (rc = dpbox.grow(2 * dpbox.n)) ||
            (rc = dreflux.grow(2 * dreflux.n)) || (rc = dtmp_pbox.grow(8 * nb)) || (rc = dtmp_rbox.grow(4 * nb)) ||
            (rc = dmap_edits.grow(2 * map_size())) || (rc = rg_grow()))
            return rc;
        for (int d = 0; d < 3; d++)
            if ((rc = dchain_off[d].grow(2 * nb + 1)) || (rc = dchain_slot[d].grow(2 * nb))) return rc;
        for (auto& r : drbox)
            if ((rc = r.grow(2 * r.n))) return rc;
        for (auto& a : drbsel)
            for (auto& v : a)
                if ((rc = v.grow(2 * v.n + 64))) return rc;
        if ((rc = grow_det(2 * (int64_t)nb))) return rc;
        layout_valid = false;  // grown lists do not keep their contents
        return EMG_OK;
    }
    size_t map_size() const {
        size_t t = 0;
        for (auto& m : map) t += m.size();
        return t;
    }

    int scratch(int64_t cells) {
        if (cells <= scr_cap) return EMG_OK;
        int64_t nc = std::max<int64_t>(cells, scr_cap * 2);
        for (int i = 0; i < 2; i++) {
            cudaFree(scr[i]);
            cudaFree(sok[i]);
            scr[i] = nullptr;
            sok[i] = nullptr;
            if (cudaMalloc(&scr[i], (size_t)nc * nv * sizeof(double)) != cudaSuccess ||
                cudaMalloc(&sok[i], (size_t)nc) != cudaSuccess) {
                cudaGetLastError();
                scr_cap = 0;
                return set_error(EMG_ERR_CUDA, "AMR scratch allocation failed");
            }
        }
        scr_cap = nc;
        return EMG_OK;
    }

    // x = box / task / leaf, y = chunks of its cells
    static dim3 box_grid(int64_t maxcells, int nbox) {
        int64_t gy = (maxcells + 255) / 256;
        if (gy < 1) gy = 1;
        if (gy > 64) gy = 64;
        return dim3((unsigned)nbox, (unsigned)gy, 1);
    }

    // ---------------------------------------------------------------- prediction boxes
    // predict_box(l, fmin, fmax) written to `slot` at ext coordinates t0 (C/amr.rs:548-586)
    PBox make_pbox(int l, const Key& fmin, const Key& fmax, int slot, const int* t0) const {
        PBox b{};
        b.l = l;
        b.slot = slot;
        for (int d = 0; d < 3; d++) {
            b.fmin[d] = fmin[d];
            b.fsz[d] = (int)(fmax[d] - fmin[d] + 1);
            b.cmin[d] = act[d] ? ediv(fmin[d], 2) - 3 : 0;
            const int64_t cmax = act[d] ? ediv(fmax[d], 2) + 3 : 0;
            b.csz[d] = (int)(cmax - b.cmin[d] + 1);
            b.t0[d] = t0[d];
        }
        b.bcmask = 0;
        for (int di = 0; di < (int)dims.size(); di++) {
            const int d = dims[di];
            const int64_t nc = n_level(l - 1, d);
            if ((b.cmin[d] < 0 && bckind(d, 0) != EMG_BC_PERIODIC) ||
                (b.cmin[d] + b.csz[d] > nc && bckind(d, 1) != EMG_BC_PERIODIC))
                b.bcmask |= 1 << di;
        }
        int64_t c = (int64_t)b.csz[0] * b.csz[1] * b.csz[2], mx = c;
        int s[3] = {b.csz[0], b.csz[1], b.csz[2]};
        for (int d : dims) {
            s[d] = b.fsz[d];
            mx = std::max<int64_t>(mx, (int64_t)s[0] * s[1] * s[2]);
        }
        b.cap = mx;
        return b;
    }

    // one CTA per box in shared memory when the largest box stage fits; the
    // multi-launch pipeline (global scratch) otherwise
    size_t pbox_smem(int64_t maxcells) const { return (size_t)maxcells * (2 * nv * sizeof(double) + 1); }
    // (227 KB per CTA, less 1 KB for the kernel's static shared memory)
    bool pbox_fused_fits(int64_t maxcells) const { return pbox_smem(maxcells) <= 226 * 1024; }

    int run_pboxes(const PBox* dboxes, int nbox, int64_t maxcells) {
        if (!nbox) return EMG_OK;
        AmrDev A = view();
        const size_t fused_smem = pbox_smem(maxcells);
        if (pbox_fused_fits(maxcells)) {
            if (!pbox_fused_ready) {
                AMR_CUDA(cudaFuncSetAttribute(pbox_fused<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, 226 * 1024));
                AMR_CUDA(cudaFuncSetAttribute(pbox_fused<7>, cudaFuncAttributeMaxDynamicSharedMemorySize, 226 * 1024));
                pbox_fused_ready = true;
            }
            NVK(pbox_fused)<<<nbox, PBOX_THREADS, fused_smem, stream>>>(A, dboxes, (int)maxcells);
            launches++;
            AMR_CUDA(cudaGetLastError());
            return EMG_OK;
        }
        const dim3 gr = box_grid(maxcells, nbox);
        NVK(pbox_gather)<<<gr, 256, 0, stream>>>(A, dboxes, scr[0], sok[0]);
        for (int di = 0; di < (int)dims.size(); di++) NVK(pbox_bc)<<<gr, 256, 0, stream>>>(A, dboxes, scr[0], sok[0], di);
        NVK(pbox_fallback)<<<gr, 256, 0, stream>>>(A, dboxes, scr[0], sok[0]);
        int cur = 0;
        for (int di = 0; di < (int)dims.size(); di++) {
            NVK(pbox_pass)<<<gr, 256, 0, stream>>>(A, dboxes, scr[cur], scr[1 - cur], di);
            cur = 1 - cur;
        }
        NVK(pbox_scatter)<<<gr, 256, 0, stream>>>(A, dboxes, scr[cur]);
        launches += 3 + 2 * dims.size();
        AMR_CUDA(cudaGetLastError());
        return EMG_OK;
    }

    // a one-off list of prediction boxes (refined children)
    int predict_now(std::vector<PBox> boxes) {
        int rc = upload_map();
        if (rc) return rc;
        int64_t off = 0, mx = 0;
        for (auto& b : boxes) {
            b.off = off;
            off += b.cap;
            mx = std::max(mx, b.cap);
        }
        if (!pbox_fused_fits(mx) && (rc = scratch(off))) return rc;
        if ((rc = dtmp_pbox.put(boxes, stream))) return rc;
        return run_pboxes(dtmp_pbox.p, (int)boxes.size(), mx);
    }

    // ---------------------------------------------------------------- restriction boxes
    // boxes of edge ancestor id (C/amr.rs:745-787)
    std::vector<std::pair<std::array<int, 3>, std::array<int, 3>>> restrict_boxes(int id) const {
        const HBlock& b = blocks[id];
        int l = b.level;
        std::vector<std::pair<std::array<int, 3>, std::array<int, 3>>> bx;
        int r[3];
        for (int d = 0; d < 3; d++) r[d] = act[d] ? 1 : 0;
        for (int o0 = -r[0]; o0 <= r[0]; o0++)
            for (int o1 = -r[1]; o1 <= r[1]; o1++)
                for (int o2 = -r[2]; o2 <= r[2]; o2++) {
                    int o[3] = {o0, o1, o2};
                    if (!o0 && !o1 && !o2) continue;
                    Key nk;
                    bool skip = false;
                    for (int d = 0; d < 3; d++) {
                        nk[d] = b.idx[d] + o[d];
                        const int64_t n = nbl(l, d);
                        if (nk[d] < 0 || nk[d] >= n) {
                            if (bckind(d, nk[d] >= n ? 1 : 0) == EMG_BC_PERIODIC)
                                nk[d] = erem(nk[d], n);
                            else
                                skip = true;
                        }
                    }
                    if (skip) continue;
                    int j = get(l, nk);
                    if (j >= 0 && !blocks[j].leaf) continue;
                    const int w = std::min(ng + 3, std::max(bd[0], std::max(bd[1], bd[2])));
                    std::array<int, 3> lo_, hi_;
                    for (int d = 0; d < 3; d++) {
                        lo_[d] = o[d] == 1 ? std::max(bd[d] - w, 0) : 0;
                        hi_[d] = o[d] == -1 ? std::min(w, bd[d]) : bd[d];
                    }
                    bx.push_back({lo_, hi_});
                }
        int64_t vol = 0;
        for (auto& p : bx) vol += (int64_t)(p.second[0] - p.first[0]) * (p.second[1] - p.first[1]) * (p.second[2] - p.first[2]);
        if (2 * vol > bcells()) {
            bx.clear();
            bx.push_back({{0, 0, 0}, {bd[0], bd[1], bd[2]}});
        }
        return bx;
    }

    RBox make_rbox(int l, int slot, const Key& idx, const std::array<int, 3>& lo_, const std::array<int, 3>& hi_) const {
        RBox b{};
        b.l = l;
        b.slot = slot;
        for (int d = 0; d < 3; d++) {
            b.lo[d] = lo_[d];
            b.hi[d] = hi_[d];
            const int64_t c0 = idx[d] * bd[d] + lo_[d];
            b.f0[d] = act[d] ? 2 * c0 - 4 : 0;
            b.sz[d] = act[d] ? 2 * (hi_[d] - lo_[d]) + 8 : 1;
        }
        b.cap = (int64_t)b.sz[0] * b.sz[1] * b.sz[2];
        b.seq = -1;
        b.fast = 1;
        for (int d = 0; d < 3; d++)
            if (act[d] && (b.f0[d] < 0 || b.f0[d] + b.sz[d] > n_level(l + 1, d) || b.sz[d] > 3 * bd[d] + 1)) b.fast = 0;
        return b;
    }

    // `bsel[di]` (optional): the boxes whose fine patch crosses a non-periodic
    // domain side along dims[di], the only ones the boundary pass of that axis
    // changes (all boxes when null)
    int run_rboxes(const RBox* dboxes, int nbox, int64_t maxcells, const int* rem = nullptr,
                   const int* const* bsel = nullptr, const int* nbsel = nullptr) {
        if (!nbox) return EMG_OK;
        AmrDev A = view();
        const dim3 gr = box_grid(maxcells, nbox);
        // boxes inside the domain: gather and first pass fused, straight into the first pass's output
        NVK(rbox_gather_pass0)<<<gr, 256, 0, stream>>>(A, dboxes, scr[1], sok[1], rem);
        NVK(rbox_gather)<<<gr, 256, 0, stream>>>(A, dboxes, scr[0], sok[0], rem, 1);
        for (int di = 0; di < (int)dims.size(); di++) {
            if (bsel && !nbsel[di]) continue;
            const dim3 gb(bsel ? (unsigned)nbsel[di] : gr.x, gr.y, 1);
            NVK(rbox_bc)<<<gb, 256, 0, stream>>>(A, dboxes, scr[0], sok[0], di, bsel ? bsel[di] : nullptr);
            launches++;
        }
        int cur = 0;
        for (int di = 0; di < (int)dims.size(); di++) {
            NVK(rbox_pass)<<<gr, 256, 0, stream>>>(A, dboxes, scr[cur], sok[cur], scr[1 - cur], sok[1 - cur], di, di == 0 ? 1 : 0);
            cur = 1 - cur;
        }
        NVK(rbox_scatter)<<<gr, 256, 0, stream>>>(A, dboxes, scr[cur]);
        launches += 3 + dims.size();
        AMR_CUDA(cudaGetLastError());
        return EMG_OK;
    }

    // restrict_all with the current hierarchy (C/amr.rs:737-816), finest first
    int restrict_all() {
        int rc = ensure_layout();
        if (rc) return rc;
        for (int l = levels - 2; l >= 0; l--) {
            if (!rbox_count[l]) continue;
            const int* sel[3] = {drbsel[l][0].p, drbsel[l][1].p, drbsel[l][2].p};
            if ((rc = run_rboxes(drbox[l].p, rbox_count[l], rbox_max[l], nullptr, sel, rbsel_count[l].data()))) return rc;
        }
        return EMG_OK;
    }
    std::vector<int64_t> rbox_max;
    std::vector<std::array<DevVec<int>, 3>> drbsel;  // per level and axis: boxes the boundary pass changes
    std::vector<std::array<int, 3>> rbsel_count;

    // Face ghost slabs of the blocks `ids` (C/amr.rs:1148-1203): same-level
    // copies, prediction boxes from the next coarser level, and the blocks that
    // touch a non-periodic domain side (boundary passes).
    void ghost_tasks(const std::vector<int>& ids, std::vector<CopyTask>& copies, std::vector<PBox>& pboxes,
                     std::vector<int>& bcl, int64_t& pmax, int64_t& poff) const {
        for (int id : ids) {
            const HBlock& b = blocks[id];
            const int l = b.level;
            int r[3];
            for (int d = 0; d < 3; d++) r[d] = act[d] ? 1 : 0;
            bool touches = false;
            for (int o0 = -r[0]; o0 <= r[0]; o0++)
                for (int o1 = -r[1]; o1 <= r[1]; o1++)
                    for (int o2 = -r[2]; o2 <= r[2]; o2++) {
                        int o[3] = {o0, o1, o2};
                        if (!o0 && !o1 && !o2) continue;
                        // only the six face slabs: the sweeps read ghost rows along
                        // their own axis within the block's interior lanes, and every
                        // gather (prediction, restriction, details) reads block
                        // interiors, so edge and corner ghost regions are never read
                        if ((o0 != 0) + (o1 != 0) + (o2 != 0) > 1) continue;
                        Key nk;
                        bool inside = true;
                        for (int d = 0; d < 3; d++) {
                            nk[d] = b.idx[d] + o[d];
                            const int64_t n = nbl(l, d);
                            if (nk[d] < 0 || nk[d] >= n) {
                                if (bckind(d, nk[d] >= n ? 1 : 0) == EMG_BC_PERIODIC)
                                    nk[d] = erem(nk[d], n);
                                else
                                    inside = false;
                            }
                        }
                        if (!inside) {
                            touches = true;
                            continue;
                        }
                        int nid = get(l, nk);
                        if (nid >= 0) {
                            copies.push_back(CopyTask{id, nid, {o[0], o[1], o[2]}});
                            continue;
                        }
                        int rs[3], re[3];
                        for (int d = 0; d < 3; d++) {
                            if (!act[d]) {
                                rs[d] = 0;
                                re[d] = 1;
                            } else if (o[d] == -1) {
                                rs[d] = 0;
                                re[d] = ng;
                            } else if (o[d] == 0) {
                                rs[d] = ng;
                                re[d] = ng + bd[d];
                            } else {
                                rs[d] = ng + bd[d];
                                re[d] = 2 * ng + bd[d];
                            }
                        }
                        Key fmin, fmax;
                        for (int d = 0; d < 3; d++) {
                            fmin[d] = b.idx[d] * bd[d] + rs[d] - gof[d];
                            fmax[d] = b.idx[d] * bd[d] + (re[d] - 1) - gof[d];
                        }
                        PBox pb = make_pbox(l, fmin, fmax, id, rs);
                        pb.off = poff;
                        poff += pb.cap;
                        pmax = std::max(pmax, pb.cap);
                        pboxes.push_back(pb);
                    }
            if (touches) bcl.push_back(id);
        }
    }

    // Chains of same-level blocks along d for the sweeps: runs of +d neighbours
    // (periodic sides included), at most AMR_CHAIN_MAX blocks each, every block
    // of `leaves` in exactly one chain. Members are the leaves (global steps)
    // or, with `any_block`, every block of the level (a subcycled level step,
    // whose list holds the level's leaves and ancestors). `off` gets one start
    // per chain plus the end, `slot` the blocks in order.
    void build_chains(int d, const std::vector<int>& leaves, std::vector<int>& off, std::vector<int>& slot,
                      bool any_block = false) const {
        off.clear();
        slot.clear();
        std::vector<char> seen(blocks.size(), 0);
        auto nbr = [&](int id, int dir) -> int {  // the same-level leaf beside id along d, or −1
            const HBlock& b = blocks[id];
            Key nk = b.idx;
            nk[d] += dir;
            const int64_t n = nbl(b.level, d);
            if (nk[d] < 0 || nk[d] >= n) {
                if (bckind(d, nk[d] >= n ? 1 : 0) != EMG_BC_PERIODIC) return -1;
                nk[d] = erem(nk[d], n);
            }
            const int j = get(b.level, nk);
            return (j >= 0 && j != id && (any_block || blocks[j].leaf)) ? j : -1;
        };
        for (int id : leaves) {
            if (seen[id]) continue;
            int h = id;  // the first unvisited block of the run (a periodic ring stops where it began)
            for (;;) {
                const int q = nbr(h, -1);
                if (q < 0 || seen[q] || q == id) break;
                h = q;
            }
            int cur = h;
            while (cur >= 0 && !seen[cur]) {
                off.push_back((int)slot.size());
                for (int k = 0; k < AMR_CHAIN_MAX && cur >= 0 && !seen[cur]; k++) {
                    seen[cur] = 1;
                    slot.push_back(cur);
                    cur = nbr(cur, +1);
                }
            }
        }
        off.push_back((int)slot.size());
    }

    // ---------------------------------------------------------------- layout
    int ensure_layout() {
        if (layout_valid) return upload_map();
        int rc = upload_map();
        if (rc) return rc;
        std::vector<int> leaves, lvl(blocks.size()), bcl;
        std::vector<int64_t> idx(3 * blocks.size());
        for (size_t i = 0; i < blocks.size(); i++) {
            lvl[i] = blocks[i].level;
            for (int d = 0; d < 3; d++) idx[3 * i + d] = blocks[i].idx[d];
            if (blocks[i].leaf) leaves.push_back((int)i);
        }
        nleaves = (int)leaves.size();
        // ghost slabs of every leaf (C/amr.rs:1148-1203)
        std::vector<CopyTask> copies;
        std::vector<PBox> pboxes;
        int64_t pmax = 0, poff = 0;
        ghost_tasks(leaves, copies, pboxes, bcl, pmax, poff);
        // restriction boxes per level
        rbox_count.assign(levels, 0);
        rbox_max.assign(levels, 0);
        if ((int)drbox.size() < levels) drbox.resize(levels);
        if ((int)drbsel.size() < levels) drbsel.resize(levels);
        rbsel_count.assign(levels, {0, 0, 0});
        int64_t rneed = 0;
        for (int l = levels - 2; l >= 0; l--) {
            std::vector<RBox> rb;
            std::vector<int> bsel[3];
            int64_t off = 0;
            for (size_t i = 0; i < blocks.size(); i++) {
                if (blocks[i].level != l || !is_edge_ancestor((int)i)) continue;
                for (auto& bx : restrict_boxes((int)i)) {
                    RBox r = make_rbox(l, (int)i, blocks[i].idx, bx.first, bx.second);
                    r.off = off;
                    off += r.cap;
                    rbox_max[l] = std::max(rbox_max[l], r.cap);
                    for (int di = 0; di < (int)dims.size(); di++) {
                        const int d = dims[di];
                        const int64_t nf = n_level(l + 1, d);
                        if ((r.f0[d] < 0 && bckind(d, 0) != EMG_BC_PERIODIC) ||
                            (r.f0[d] + r.sz[d] > nf && bckind(d, 1) != EMG_BC_PERIODIC))
                            bsel[di].push_back((int)rb.size());
                    }
                    rb.push_back(r);
                }
            }
            rneed = std::max(rneed, off);
            rbox_count[l] = (int)rb.size();
            if ((rc = drbox[l].put(rb, stream))) return rc;
            for (int di = 0; di < 3; di++) {
                rbsel_count[l][di] = (int)bsel[di].size();
                if ((rc = drbsel[l][di].put(bsel[di], stream))) return rc;
            }
        }
        // refluxing faces (C/amr.rs:1327-1406), bucketed by (d, side) in the reference's order
        std::vector<RefluxFace> rfaces;
        for (int bucket = 0; bucket < 6; bucket++) {
            rface_start[bucket] = (int)rfaces.size();
            const int d = bucket / 2, side = bucket % 2;
            if (!act[d]) continue;
            const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            for (size_t id = 0; id < blocks.size(); id++) {
                const HBlock& b = blocks[id];
                const int l = b.level;
                if (!b.leaf || l + 1 >= levels) continue;
                const int64_t nbk = nb0[d] << l;
                Key nk = b.idx;
                nk[d] += side == 1 ? 1 : -1;
                if (nk[d] < 0 || nk[d] >= nbk) {
                    if (bckind(d, side) != EMG_BC_PERIODIC) continue;
                    nk[d] = erem(nk[d], nbk);
                }
                const int nj = get(l, nk);
                if (!(nj >= 0 && !blocks[nj].leaf)) continue;
                RefluxFace rf{};
                rf.slot = (int)id;
                rf.d = d;
                rf.side = side;
                rf.dx = dxl[3 * l + d];
                for (int qa = 0; qa < 2; qa++)
                    for (int qb = 0; qb < 2; qb++) {
                        rf.fine[qa][qb] = -1;
                        if ((qa && !act[e0]) || (qb && !act[e1])) continue;
                        Key ck = nk;
                        ck[d] = 2 * nk[d] + (side == 1 ? 0 : 1);
                        ck[e0] = act[e0] ? 2 * b.idx[e0] + qa : 0;
                        ck[e1] = act[e1] ? 2 * b.idx[e1] + qb : 0;
                        const int cid = get(l + 1, ck);
                        if (cid >= 0 && blocks[cid].leaf) rf.fine[qa][qb] = cid;
                    }
                rfaces.push_back(rf);
            }
        }
        rface_start[6] = (int)rfaces.size();
        // chains of the global sweeps; the chain's sweep reads the neighbour's
        // interior at a joint, so the face slab between two blocks of a chain
        // is not filled before the sweeps (the regrid's details, whose sensor
        // stencils reach one cell into the face slabs, get the full list)
        std::vector<int> next_in_chain(3 * blocks.size(), -1);
        for (int d = 0; d < 3; d++) {
            nchain[d] = 0;
            if (!act[d]) continue;
            std::vector<int> coff, cslot;
            build_chains(d, leaves, coff, cslot);
            for (size_t c = 0; c + 1 < coff.size(); c++)
                for (int i = coff[c]; i + 1 < coff[c + 1]; i++) next_in_chain[3 * cslot[i] + d] = cslot[i + 1];
            if ((rc = dchain_off[d].put(coff, stream)) || (rc = dchain_slot[d].put(cslot, stream))) return rc;
            nchain[d] = (int)coff.size() - 1;
        }
        std::vector<CopyTask> copies_sweep;
        {
            for (const CopyTask& t : copies) {
                int d = -1, nz = 0;
                for (int e = 0; e < 3; e++)
                    if (t.o[e]) {
                        d = e;
                        nz++;
                    }
                const bool inner = nz == 1 && ((t.o[d] == 1 && next_in_chain[3 * t.slot + d] == t.src) ||
                                               (t.o[d] == -1 && next_in_chain[3 * t.src + d] == t.slot));
                if (!inner) copies_sweep.push_back(t);
            }
        }
        if ((rc = dleaves.put(leaves, stream)) || (rc = dlevel.put(lvl, stream)) || (rc = didx.put(idx, stream)) ||
            (rc = dbcleaves.put(bcl, stream)) || (rc = dcopy.put(copies, stream)) || (rc = dcopy_sweep.put(copies_sweep, stream)) || (rc = dpbox.put(pboxes, stream)) ||
            (rc = dreflux.put(rfaces, stream)))
            return rc;
        ncopy = (int)copies.size();
        ncopy_sweep = (int)copies_sweep.size();
        npbox = (int)pboxes.size();
        nbcleaves = (int)bcl.size();
        pbox_max = pmax;
        if ((rc = scratch(std::max(pbox_fused_fits(pmax) ? 0 : poff, rneed)))) return rc;
        layout_valid = true;
        layout_gen++;
        return EMG_OK;
    }
    int64_t pbox_max = 0;
    bool pbox_fused_ready = false;  // dynamic shared-memory opt-in of pbox_fused (per handle and device)

    // ghost-extended boxes of every leaf (fill_scratch, C/amr.rs:1113-1221)
    // `for_sweeps`: only the slabs the (chained) global sweeps read
    int fill_ghosts(bool for_sweeps = false) {
        AmrDev A = view();
        const int nc = for_sweeps ? ncopy_sweep : ncopy;
        if (nc) {
            NVK(ghost_copy)<<<nc, COPY_THREADS, 0, stream>>>(A, for_sweeps ? dcopy_sweep.p : dcopy.p);
            launches++;
        }
        int rc = run_pboxes(dpbox.p, npbox, pbox_max);
        if (rc) return rc;
        if (nbcleaves)
            for (int di = 0; di < (int)dims.size(); di++) {
                NVK(ghost_bc)<<<box_grid(2 * (int64_t)ng * std::max(bd[0], 1) * std::max(bd[1], 1), nbcleaves), 256, 0, stream>>>(
                    A, dbcleaves.p, dlevel.p, didx.p, di);
                launches++;
            }
        AMR_CUDA(cudaGetLastError());
        return EMG_OK;
    }

    // pencils per CTA of the sweep along d: the tuned value, else 32 (two
    // rows of a 16-wide block per CTA) unless the block face has fewer cells
    int amr_sweep_P(int d, int lane, int other) const {
        if (amrP[d]) return amrP[d];
        return bd[lane] > 16 ? 32 : (bd[lane] * bd[other] >= 32 ? 32 : 16);
    }
    // sweeps of every active axis over the leaves, or over the `nlist` blocks of `list`
    // `lv`: the subcycled level whose block chains replace `list` in the launch
    int sweeps(int stage, const int* list = nullptr, int nlist = 0, const ScLevel* lv = nullptr) {
        for (int d : dims) {
            int rc = sweep_axis(stage, d, dims[0], list, nlist, lv);
            if (rc) return rc;
        }
        return EMG_OK;
    }
    int sweep_axis(int stage, int d, int first, const int* list = nullptr, int nlist = 0, const ScLevel* lv = nullptr) {
        const int* blk = list ? list : dleaves.p;
        const int nblk = list ? nlist : nleaves;
        AmrDev A = view();
        {
            int o[2], no_ = 0;
            for (int e = 0; e < 3; e++)
                if (e != d) o[no_++] = e;
            int lane = o[1], other = o[0];
            if (!act[o[1]] && act[o[0]]) {
                lane = o[0];
                other = o[1];
            }
            SweepParams p{};
            p.uin = u;
            p.rhs = rhs;
            p.ctl = ctl;
            p.ncell = A.ntot;
            const int64_t st[3] = {(int64_t)ext[1] * ext[2], ext[2], 1};
            p.sd = st[d];
            p.sl = st[lane];
            p.so = st[other];
            p.nd = bd[d];
            p.nl = bd[lane];
            p.no = bd[other];
            p.gd = gof[d];
            p.gl = gof[lane];
            p.go = gof[other];
            p.d = d;
            p.seg = bd[d];
            p.first = d == first;
            p.last = 0;
            p.stage = stage;
            p.rows_contig = p.sd == 1;
            p.ndim = (double)dims.size();
            p.positivity = opts.positivity ? 1 : 0;
            p.tol = opts.tol;
            p.eos = A.eos;
            const int P = amr_sweep_P(d, lane, other);
            p.lw = std::min(P, bd[lane]);
            p.amr = 1;
            p.leaf_slot = blk;
            p.leaf_level = dlevel.p;
            p.bcell = bcell;
            const int rows = P / p.lw;
            p.ngroups = (bd[other] + rows - 1) / rows;
            for (int l = 0; l < levels && l < 16; l++) p.dx_level[l] = dxl[3 * l + d];
            p.dx = dxl[d];
            p.face = face;
            p.nface = cap * 3 * 2 * nv * (int64_t)npen;
            p.npen = npen;
            p.pen_lane_major = lane < other ? 1 : 0;
            int nz = nblk;
            if (!list && nchain[d] > 0) {  // global sweeps: chains of same-level leaves
                p.chain_off = dchain_off[d].p;
                p.chain_slot = dchain_slot[d].p;
                nz = nchain[d];
            } else if (lv && lv->nch[d] > 0) {  // a subcycled level: chains of its blocks
                p.chain_off = lv->choff[d].p;
                p.chain_slot = lv->chslot[d].p;
                nz = lv->nch[d];
            }
            const dim3 grid((unsigned)(nz * p.ngroups), 1, 1);
            cudaError_t e;
            if (nv == 7) {
                // the five-equation sweep with the same geometry (FP64 only)
                FiveSweepParams q{};
                q.uin = p.uin;
                q.rhs = p.rhs;
                q.ctl = p.ctl;
                q.ncell = p.ncell;
                q.sd = p.sd;
                q.sl = p.sl;
                q.so = p.so;
                q.nd = p.nd;
                q.nl = p.nl;
                q.no = p.no;
                q.gd = p.gd;
                q.gl = p.gl;
                q.go = p.go;
                q.d = d;
                q.seg = p.seg;
                q.first = p.first;
                q.last = 0;
                q.stage = stage;
                q.rows_contig = p.rows_contig;
                q.dx = p.dx;
                q.ndim = p.ndim;
                q.positivity = p.positivity;
                q.tol = p.tol;
                q.sys = A.fsys;
                q.leaf_slot = blk;
                q.leaf_level = dlevel.p;
                q.bcell = bcell;
                q.ngroups = p.ngroups;
                q.lw = p.lw;
                for (int l = 0; l < 16; l++) q.dx_level[l] = p.dx_level[l];
                q.face = face;
                q.nface = p.nface;
                q.npen = npen;
                q.pen_lane_major = p.pen_lane_major;
                q.chain_off = p.chain_off;
                q.chain_slot = p.chain_slot;
                e = opts.precision == EMG_PRECISION_F64_FAST ? five_sweep_launch_amr_fast(P, opts.mode, q, grid, stream)
                                                             : five_sweep_launch_amr(P, opts.mode, q, grid, stream);
            } else {
                e = opts.precision == EMG_PRECISION_MIXED      ? sweep_launch_amr_mixed(P, opts.mode, p, grid, stream)
                    : opts.precision == EMG_PRECISION_F64_FAST ? sweep_launch_amr_fast(P, opts.mode, p, grid, stream)
                                                               : sweep_launch_amr_f64(P, opts.mode, p, grid, stream);
            }
            launches++;
            if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("AMR sweep: ") + cudaGetErrorString(e));
        }
        return EMG_OK;
    }

    // Launch shape of the batched sweeps (EMG_OPT_AUTOTUNE): per axis, time
    // the sweep over all leaves with 16 and 32 pencils per CTA (one or two rows
    // of the block face) on the current state and keep the faster. The sweeps
    // only write the residual and the face-flux record, which the step then
    // overwrites; results do not depend on the shape.
    int autotune_sweeps() {
        int rc = restrict_all();
        if (rc) return rc;
        if ((rc = fill_ghosts(true))) return rc;
        cudaEvent_t a, b;
        AMR_CUDA(cudaEventCreate(&a));
        AMR_CUDA(cudaEventCreate(&b));
        for (int d : dims) {
            int o[2], no_ = 0;
            for (int e = 0; e < 3; e++)
                if (e != d) o[no_++] = e;
            int lane = o[1], other = o[0];
            if (!act[o[1]] && act[o[0]]) {
                lane = o[0];
                other = o[1];
            }
            std::vector<int> cands;
            if (bd[lane] <= 16) cands.push_back(16);
            if (bd[lane] > 16 || bd[lane] * bd[other] >= 32) cands.push_back(32);
            float best_ms = 1e30f;
            int best = 0;
            for (int P : cands) {
                amrP[d] = P;
                if ((rc = sweep_axis(1, d, dims[0]))) break;
                cudaEventRecord(a, stream);
                for (int r = 0; r < 3 && !rc; r++) rc = sweep_axis(1, d, dims[0]);
                cudaEventRecord(b, stream);
                if (rc) break;
                if (cudaEventSynchronize(b) != cudaSuccess) {
                    rc = set_error(EMG_ERR_CUDA, "AMR autotune timing failed");
                    break;
                }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, a, b);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = P;
                }
            }
            amrP[d] = best;
            if (rc) break;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return rc;
    }

    int compute_rhs(int stage) {
        cudaEvent_t* ev = stage_ev[stage - 1];
        record_ev(ev[0]);
        int rc = restrict_all();
        if (rc) return rc;
        record_ev(ev[1]);
        if ((rc = fill_ghosts(true))) return rc;
        record_ev(ev[2]);
        if ((rc = sweeps(stage))) return rc;
        record_ev(ev[3]);
        {
            AmrDev A = view();
            for (int bucket = 0; bucket < 6; bucket++) {
                const int nf = rface_start[bucket + 1] - rface_start[bucket];
                if (!nf) continue;
                NVK(reflux_faces)<<<nf, 256, 0, stream>>>(A, rhs, face, npen, dreflux.p + rface_start[bucket]);
                launches++;
            }
            AMR_CUDA(cudaGetLastError());
        }
        record_ev(ev[4]);
        record_ev(ev[5]);  // start of the RK update (rk follows)
        return EMG_OK;
    }
    // per stage: [restrict, ghosts, fluxes, reflux, rk start, rk end] events,
    // created once (a captured step graph records into the same events)
    cudaEvent_t stage_ev[3][7]{};
    bool stage_pending = false;
    // external records: inside a step capture they become event-record nodes
    // of the graph, so replays record the events too
    bool capturing = false;
    void record_ev(cudaEvent_t e) {
        if (capturing)
            cudaEventRecordWithFlags(e, stream, cudaEventRecordExternal);
        else
            cudaEventRecord(e, stream);
    }
    int make_events() {
        for (auto& st : stage_ev)
            for (auto& e : st)
                if (!e) AMR_CUDA(cudaEventCreate(&e));
        return EMG_OK;
    }
    void collect_times() {
        if (!stage_pending) return;
        for (auto& e : stage_ev) {
            float t[6] = {0, 0, 0, 0, 0, 0};
            for (int i = 0; i < 6; i++) cudaEventElapsedTime(&t[i], e[i], e[i + 1]);
            phase_ms[0] += t[0];
            phase_ms[1] += t[1];
            phase_ms[2] += t[2];
            phase_ms[3] += t[3] + t[5];  // reflux + RK update
        }
        cudaGetLastError();  // timing queries never leave an error behind
        stage_pending = false;
    }

    int rk(int stage) {
        AmrDev A = view();
        PHK(amr_rk)<<<dim3((unsigned)nleaves, (unsigned)std::min<int64_t>((bcells() + 255) / 256, 16)), 256, 0, stream>>>(
            A, u0, rhs, dleaves.p, dlevel.p, ddxl.p, stage, ctl, 0);
        launches++;
        AMR_CUDA(cudaGetLastError());
        record_ev(stage_ev[stage - 1][6]);
        return EMG_OK;
    }

    // the three stages of one step (the work a step graph holds)
    int step_body() {
        for (int s = 1; s <= 3; s++) {
            int rc = compute_rhs(s);
            if (rc) return rc;
            if ((rc = rk(s))) return rc;
        }
        return EMG_OK;
    }

    // ---- CUDA graph of a step: between regrids the launch sequence of a step
    // (every kernel, its grid and its arguments) is fixed, so the first step
    // after a layout change runs eagerly, the second is captured into a graph
    // and later steps replay it; dt reaches the kernels through the control
    // block, copied in before each launch.
    cudaGraphExec_t step_exec = nullptr;
    uint64_t layout_gen = 0, graph_gen = 0, eager_gen = 0;
    uint64_t graph_launches = 0;
    bool use_graph = true;
    void drop_graph() {
        if (step_exec) cudaGraphExecDestroy(step_exec);
        step_exec = nullptr;
    }
    int run_step_body() {
        if (!use_graph) return step_body();
        if (step_exec && graph_gen == layout_gen) {
            AMR_CUDA(cudaGraphLaunch(step_exec, stream));
            launches += graph_launches;
            return EMG_OK;
        }
        drop_graph();
        if (eager_gen != layout_gen) {  // first step with this layout: eager (sets up kernels)
            eager_gen = layout_gen;
            return step_body();
        }
        AMR_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const uint64_t l0 = launches;
        capturing = true;
        int rc = step_body();
        capturing = false;
        cudaGraph_t gph = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream, &gph);
        graph_launches = launches - l0;
        launches = l0;
        if (rc) {
            if (gph) cudaGraphDestroy(gph);
            return rc;
        }
        if (e != cudaSuccess) return set_error(EMG_ERR_CUDA, std::string("step capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&step_exec, gph, 0);
        cudaGraphDestroy(gph);
        if (e != cudaSuccess) {
            step_exec = nullptr;
            return set_error(EMG_ERR_CUDA, std::string("step graph: ") + cudaGetErrorString(e));
        }
        graph_gen = layout_gen;
        AMR_CUDA(cudaGraphLaunch(step_exec, stream));
        launches += graph_launches;
        return EMG_OK;
    }

    // ---------------------------------------------------------------- tree edits
    int add_block(int level, const Key& idx) {
        int id = (int)blocks.size();
        int rc = reserve(id + 1);
        if (rc) return rc;
        blocks.push_back(HBlock{level, idx, true});
        insert(level, idx, id);
        return EMG_OK;
    }

    // conserved variables of a five-equation primitive state (C/multiphase.rs:
    // 152-163, the closure of :58-75), on the host for initial data
    void five_to_cons(const double* w, double* u_) const {
        const double al[2] = {w[6], 1.0 - w[6]};
        double d = 0.0, b = 0.0;
        for (int k = 0; k < 2; k++) {
            const emg_eos& e = five.eos[k];
            const double vol = al[k] - e.b * w[k];
            d = d + vol / (e.gamma - 1.0);
            b = b + e.gamma * e.p_inf * vol / (e.gamma - 1.0) + e.q * w[k];
        }
        const double r = w[0] + w[1];
        u_[0] = w[0];
        u_[1] = w[1];
        u_[2] = r * w[2];
        u_[3] = r * w[3];
        u_[4] = r * w[4];
        u_[5] = (w[5] * d + b) + 0.5 * r * (w[2] * w[2] + w[3] * w[3] + w[4] * w[4]);
        u_[6] = w[6];
    }

    int init_block_data(int id, emg_init_fn init, void* ictx) {
        const HBlock& b = blocks[id];
        const int64_t n = bcells();
        std::vector<double> xs(3 * n), ws(nv * n), us(nv * n);
        for (int64_t i = 0; i < bd[0]; i++)
            for (int64_t j = 0; j < bd[1]; j++)
                for (int64_t k = 0; k < bd[2]; k++) {
                    const int64_t q = (i * bd[1] + j) * bd[2] + k;
                    const int64_t g[3] = {b.idx[0] * bd[0] + i, b.idx[1] * bd[1] + j, b.idx[2] * bd[2] + k};
                    for (int d = 0; d < 3; d++)
                        xs[3 * q + d] = act[d] ? lo[d] + ((double)g[d] + 0.5) * dxl[3 * b.level + d] : 0.5 * (lo[d] + hi[d]);
                }
        init(ictx, xs.data(), n, ws.data());
        for (int64_t q = 0; q < n; q++) {
            const double* w = &ws[nv * q];
            double* u_ = &us[nv * q];
            if (nv == 7) {
                five_to_cons(w, u_);
                continue;
            }
            // to_cons (C/system.rs:210-217; ρe as C/eos.rs:44-54)
            const double rho = w[0];
            const double ke = 0.5 * rho * (w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
            const double v = 1.0 / rho;
            const double e = (w[4] + eos.gamma * eos.p_inf) * (v - eos.b) / (eos.gamma - 1.0) + eos.q;
            u_[0] = rho;
            u_[1] = rho * w[1];
            u_[2] = rho * w[2];
            u_[3] = rho * w[3];
            u_[4] = rho * e + ke;
        }
        // the staging buffer is reused: wait for the previous block's copy-in
        AMR_CUDA(cudaStreamSynchronize(stream));
        int rc = dstage.put(us, stream);
        if (rc) return rc;
        AmrDev A = view();
        NVK(pool_put_interior)<<<16, 256, 0, stream>>>(A, id, dstage.p);
        launches++;
        AMR_CUDA(cudaGetLastError());
        return EMG_OK;
    }

    // Refinements are predicted in batches: the children of a parent at level l
    // read levels <= l only and write level l + 1, so refinements of parents of
    // one level are independent and run as one launch; a refinement of another
    // level first flushes the batch, which keeps the sequential order's data
    // and block map for every box.
    int queue_pboxes(int l, std::vector<PBox>& boxes) {
        if (l != pend_level) {
            int rc = flush_pboxes();
            if (rc) return rc;
        }
        pend_level = l;
        pend_pbox.insert(pend_pbox.end(), boxes.begin(), boxes.end());
        return EMG_OK;
    }
    int flush_pboxes() {
        if (pend_pbox.empty()) return EMG_OK;
        std::vector<PBox> boxes;
        boxes.swap(pend_pbox);
        pend_level = -1;
        return predict_now(std::move(boxes));
    }

    // C/amr.rs:952-1011
    int refine_block(int id, emg_init_fn init, void* ictx) {
        const int l = blocks[id].level;
        const Key idx = blocks[id].idx;
        if (!blocks[id].leaf) return EMG_OK;
        int rc;
        if (l > 0) {
            for (auto& nk : neighbours(l, idx)) {
                if (get(l, nk) < 0) {
                    for (int m = l - 1; m >= 0; m--) {
                        Key pk;
                        for (int d = 0; d < 3; d++) pk[d] = act[d] ? nk[d] >> (l - m) : 0;
                        int pid = get(m, pk);
                        if (pid >= 0) {
                            if ((rc = refine_block(pid, init, ictx))) return rc;
                            break;
                        }
                    }
                }
            }
        }
        id = get(l, idx);
        if (id < 0 || !blocks[id].leaf) return EMG_OK;
        std::vector<Key> kids = children(idx);
        const int first = (int)blocks.size();
        if ((rc = reserve(first + (int64_t)kids.size()))) return rc;
        // children data first (the parent level is unchanged while they are computed)
        std::vector<PBox> boxes;
        for (size_t n = 0; n < kids.size(); n++) {
            const Key& c = kids[n];
            blocks.push_back(HBlock{l + 1, c, true});  // not yet in the index
            if (!init) {
                Key fmin, fmax;
                for (int d = 0; d < 3; d++) {
                    fmin[d] = c[d] * bd[d];
                    fmax[d] = c[d] * bd[d] + bd[d] - 1;
                }
                boxes.push_back(make_pbox(l + 1, fmin, fmax, first + (int)n, gof));
            }
        }
        if (init) {
            for (size_t n = 0; n < kids.size(); n++)
                if ((rc = init_block_data(first + (int)n, init, ictx))) return rc;
        } else if ((rc = queue_pboxes(l, boxes))) {
            return rc;
        }
        blocks[id].leaf = false;
        for (size_t n = 0; n < kids.size(); n++) insert(l + 1, kids[n], first + (int)n);
        layout_valid = false;
        return EMG_OK;
    }

    int grow_det(int64_t n) {
        if (n <= det_cap) return EMG_OK;
        cudaFree(det);
        det_cap = std::max<int64_t>(n, 2 * det_cap);
        AMR_CUDA(cudaMalloc(&det, det_cap * sizeof(unsigned long long)));
        return EMG_OK;
    }
    // details of all leaves (C/amr.rs:823-867), ancestors 0
    int details(std::vector<double>& out) {
        int rc = ensure_layout();
        if (rc) return rc;
        if ((rc = fill_ghosts())) return rc;
        if ((rc = grow_det((int64_t)blocks.size()))) return rc;
        AMR_CUDA(cudaMemsetAsync(det, 0, blocks.size() * sizeof(unsigned long long), stream));
        AmrDev A = view();
        PHK(amr_detail)<<<dim3((unsigned)nleaves, (unsigned)std::min<int64_t>((bcells() + 255) / 256, 16)), 256, 0, stream>>>(
            A, dleaves.p, det);
        launches++;
        AMR_CUDA(cudaGetLastError());
        std::vector<unsigned long long> bits(blocks.size());
        AMR_CUDA(cudaMemcpyAsync(bits.data(), det, bits.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaStreamSynchronize(stream));
        out.resize(blocks.size());
        for (size_t i = 0; i < bits.size(); i++) std::memcpy(&out[i], &bits[i], sizeof(double));
        return EMG_OK;
    }
    // C/amr.rs:877-892
    std::vector<int8_t> flags_from(const std::vector<double>& det) const {
        std::vector<int8_t> f(blocks.size(), 0);
        for (size_t i = 0; i < blocks.size(); i++) {
            if (!blocks[i].leaf)
                f[i] = 0;
            else if (det[i] > cfg.eps && blocks[i].level + 1 < levels)
                f[i] = 1;
            else if (det[i] < cfg.eps / 128.0)
                f[i] = -1;
        }
        return f;
    }
    int flags(std::vector<int8_t>& f) {
        int rc = restrict_all();
        if (rc) return rc;
        std::vector<double> det;
        if ((rc = details(det))) return rc;
        f = flags_from(det);
        return EMG_OK;
    }

    // ---------------------------------------------------------------- regrid on the device
    // Amr::regrid (C/amr.rs:1039-1106): flags, the one-block buffer, the
    // refinements with 2:1 balance and the coarsening batches are decided and
    // applied to a device copy of the tree (amr_regrid.cuh); the host mirror
    // of the tree is then read back from the device, and the data work (the
    // prediction of new children, the restriction of coarsened parents and the
    // block moves of the compaction) runs as before, in the reference's order.
    int id_limit = 0x7fffffff;  // see AmrDev::id_limit
    DevVec<int> rg_level, rg_leaf, rg_count, rg_events, rg_rem, rg_orig, rg_moves;
    DevVec<int64_t> rg_idx, rg_ckey, rg_par;
    DevVec<signed char> rg_f, rg_wantd, rg_mark;
    bool rg_ready = false;

    RgTree rg_tree() const {
        return RgTree{rg_level.p, rg_idx.p, rg_leaf.p, dmap.p, rg_count.p, (int)map_size()};
    }
    RgGeom rg_geom() const {
        RgGeom G{};
        for (int d = 0; d < 3; d++) {
            G.act[d] = act[d];
            G.nb0[d] = nb0[d];
            G.periodic[d] = bckind(d, 0) == EMG_BC_PERIODIC;
        }
        G.levels = levels;
        for (int l = 0; l < levels && l < AMR_MAX_LEVELS; l++) G.mapoff[l] = mapoff[l];
        G.mapsize = (int64_t)map_size();
        return G;
    }
    // the device tree's arrays, sized for every map slot (at most one block per slot)
    int rg_grow() {
        const size_t cap_ = map_size();
        int rc;
        if ((rc = rg_level.grow(cap_)) || (rc = rg_leaf.grow(cap_)) || (rc = rg_idx.grow(3 * cap_)) ||
            (rc = rg_f.grow(cap_)) || (rc = rg_wantd.grow(cap_)) || (rc = rg_mark.grow(cap_)) || (rc = rg_events.grow(3 * cap_)) ||
            (rc = rg_rem.grow(cap_)) || (rc = rg_orig.grow(cap_)) || (rc = rg_moves.grow(2 * cap_)) ||
            (rc = rg_ckey.grow(4 * cap_)) || (rc = rg_par.grow(4 * cap_)) || (rc = rg_count.grow(8)))
            return rc;
        return EMG_OK;
    }
    // the host mirror to the device tree
    int rg_upload_tree() {
        int rc = rg_grow();
        if (rc) return rc;
        std::vector<int> lv(blocks.size()), lf(blocks.size());
        std::vector<int64_t> ix(3 * blocks.size());
        for (size_t i = 0; i < blocks.size(); i++) {
            lv[i] = blocks[i].level;
            lf[i] = blocks[i].leaf ? 1 : 0;
            for (int d = 0; d < 3; d++) ix[3 * i + d] = blocks[i].idx[d];
        }
        std::vector<int> cnt(8, 0);
        cnt[0] = (int)blocks.size();
        if ((rc = rg_level.put(lv, stream)) || (rc = rg_leaf.put(lf, stream)) || (rc = rg_idx.put(ix, stream)) ||
            (rc = rg_count.put(cnt, stream)))
            return rc;
        if (!rg_ready) {
            AMR_CUDA(cudaFuncSetAttribute(rg_refine, cudaFuncAttributeMaxDynamicSharedMemorySize, RG_SMEM_MAX));
            AMR_CUDA(cudaFuncSetAttribute(rg_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, RG_SMEM_MAX));
            rg_ready = true;
        }
        return EMG_OK;
    }
    static constexpr int RG_SMEM_MAX = 200 * 1024;
    int rg_counts(int* c) {
        AMR_CUDA(cudaMemcpyAsync(c, rg_count.p, 8 * sizeof(int), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaStreamSynchronize(stream));
        if (c[3]) return set_error(EMG_ERR_CUDA, "device regrid: tree capacity or recursion bound exceeded");
        return EMG_OK;
    }
    // the host mirror of the tree read back from the device (the device block map is current)
    int rg_mirror() {
        int c[8];
        int rc = rg_counts(c);
        if (rc) return rc;
        const int nb = c[0];
        std::vector<int> lv(nb), lf(nb);
        std::vector<int64_t> ix(3 * (size_t)nb);
        AMR_CUDA(cudaMemcpyAsync(lv.data(), rg_level.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaMemcpyAsync(lf.data(), rg_leaf.p, nb * sizeof(int), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaMemcpyAsync(ix.data(), rg_idx.p, 3 * (size_t)nb * sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaStreamSynchronize(stream));
        blocks.resize(nb);
        for (auto& m : map) std::fill(m.begin(), m.end(), -1);
        for (int i = 0; i < nb; i++) {
            blocks[i] = HBlock{lv[i], Key{ix[3 * i], ix[3 * i + 1], ix[3 * i + 2]}, lf[i] != 0};
            const int64_t sl = slot_of(lv[i], blocks[i].idx);
            if (sl >= 0) map[lv[i]][sl] = i;
        }
        map_changed.clear();
        map_dirty = false;  // the device map holds the same edits
        map_uploaded = true;
        layout_valid = false;
        return EMG_OK;
    }
    // wavelet details of every leaf into `det` (ancestors 0), on the device only
    int details_device() {
        int rc = ensure_layout();
        if (rc) return rc;
        if ((rc = fill_ghosts())) return rc;
        if ((rc = grow_det((int64_t)blocks.size()))) return rc;
        AMR_CUDA(cudaMemsetAsync(det, 0, blocks.size() * sizeof(unsigned long long), stream));
        AmrDev A = view();
        PHK(amr_detail)<<<dim3((unsigned)nleaves, (unsigned)std::min<int64_t>((bcells() + 255) / 256, 16)), 256, 0, stream>>>(
            A, dleaves.p, det);
        launches++;
        AMR_CUDA(cudaGetLastError());
        return EMG_OK;
    }
    int rg_flags_now(int nb) {
        RgTree T = rg_tree();
        rg_flags<<<(nb + 255) / 256, 256, 0, stream>>>(T, det, nb, levels, cfg.eps, rg_f.p);
        launches++;
        AMR_CUDA(cudaGetLastError());
        return EMG_OK;
    }

    int regrid() {
        int rc = restrict_all();  // and the layout, with the device map
        if (rc) return rc;
        if ((rc = details_device())) return rc;
        const int nb0_ = (int)blocks.size();
        if ((rc = rg_upload_tree())) return rc;
        RgTree T = rg_tree();
        const RgGeom G = rg_geom();
        if ((rc = rg_flags_now(nb0_))) return rc;
        rg_want<<<(nb0_ + 255) / 256, 256, 0, stream>>>(T, G, rg_f.p, nb0_, rg_wantd.p);
        const size_t msm = map_size() * sizeof(int);
        const int in_smem = msm <= (size_t)RG_SMEM_MAX ? 1 : 0;
        rg_refine<<<1, 256, in_smem ? msm : 0, stream>>>(T, G, rg_wantd.p, nb0_, in_smem, rg_events.p);
        launches += 2;
        AMR_CUDA(cudaGetLastError());
        int c[8];
        if ((rc = rg_counts(c))) return rc;
        if (c[0] != nb0_) {
            // the refined tree, then the children's data in the reference's order:
            // refinements of parents of one level in one launch, each such batch
            // seeing only the blocks that existed when its first refinement ran
            const int nev = c[1];
            std::vector<int> ev(3 * (size_t)nev);
            AMR_CUDA(cudaMemcpyAsync(ev.data(), rg_events.p, ev.size() * sizeof(int), cudaMemcpyDeviceToHost, stream));
            AMR_CUDA(cudaStreamSynchronize(stream));
            if ((rc = rg_mirror())) return rc;
            if ((rc = reserve((int64_t)blocks.size()))) return rc;
            for (int e0 = 0; e0 < nev;) {
                const int l = ev[3 * e0 + 2];
                int e1 = e0;
                std::vector<PBox> boxes;
                while (e1 < nev && ev[3 * e1 + 2] == l) {
                    const int first = ev[3 * e1 + 1];
                    const std::vector<Key> kids = children(blocks[ev[3 * e1]].idx);
                    for (size_t n = 0; n < kids.size(); n++) {
                        Key fmin, fmax;
                        for (int d = 0; d < 3; d++) {
                            fmin[d] = kids[n][d] * bd[d];
                            fmax[d] = kids[n][d] * bd[d] + bd[d] - 1;
                        }
                        boxes.push_back(make_pbox(l + 1, fmin, fmax, first + (int)n, gof));
                    }
                    e1++;
                }
                id_limit = ev[3 * e0 + 1];
                rc = predict_now(std::move(boxes));
                id_limit = 0x7fffffff;
                if (rc) return rc;
                e0 = e1;
            }
            // flags of the refined hierarchy
            if ((rc = restrict_all()) || (rc = details_device()) || (rc = rg_flags_now((int)blocks.size()))) return rc;
        }
        // coarsening, level by level from the finest
        const size_t msm2 = in_smem ? msm : 0;
        {
            const int nb = (int)blocks.size();
            rg_candidate_flags<<<(nb + 255) / 256, 256, 0, stream>>>(T, G, rg_f.p, rg_wantd.p, nb0_, rg_mark.p);
            rg_compact<<<1, RG_SCAN_T, 0, stream>>>(T, rg_mark.p, rg_ckey.p);
            launches += 2;
            AMR_CUDA(cudaGetLastError());
            if ((rc = rg_counts(c))) return rc;
        }
        const int ncand = c[4];
        for (int l = levels - 2; l >= 0 && ncand > 0; l--) {
            rg_decide_flags<<<(ncand + 255) / 256, 256, 0, stream>>>(T, G, rg_ckey.p, l, rg_mark.p);
            rg_decide<<<1, 256, 0, stream>>>(T, G, rg_ckey.p, rg_mark.p, l, rg_par.p, rg_rem.p);
            launches += 2;
            AMR_CUDA(cudaGetLastError());
            if ((rc = rg_counts(c))) return rc;
            const int npar = c[5];
            if (!npar) continue;
            std::vector<int64_t> par(4 * (size_t)npar);
            AMR_CUDA(cudaMemcpyAsync(par.data(), rg_par.p, par.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, stream));
            AMR_CUDA(cudaStreamSynchronize(stream));
            // restrictions on the pool and the map as before the batch, each box
            // seeing the fine blocks removed by earlier parents of the batch as absent
            if ((rc = upload_map())) return rc;
            std::vector<RBox> boxes;
            for (int q = 0; q < npar; q++) {
                const Key key = {par[4 * q + 1], par[4 * q + 2], par[4 * q + 3]};
                RBox b = make_rbox(l, (int)par[4 * q], key, {0, 0, 0}, {bd[0], bd[1], bd[2]});
                b.seq = q;
                boxes.push_back(b);
            }
            const int chunk = 64;
            for (int c0 = 0; c0 < (int)boxes.size(); c0 += chunk) {
                const int nbx = std::min<int>(chunk, (int)boxes.size() - c0);
                int64_t off = 0, mx = 0;
                std::vector<RBox> part(boxes.begin() + c0, boxes.begin() + c0 + nbx);
                for (auto& b : part) {
                    b.off = off;
                    off += b.cap;
                    mx = std::max(mx, b.cap);
                }
                if ((rc = scratch(off))) return rc;
                if ((rc = dtmp_rbox.put(part, stream))) return rc;
                if ((rc = run_rboxes(dtmp_rbox.p, nbx, mx, rg_rem.p))) return rc;
            }
            // the edits, then the block moves of the compaction
            rg_apply<<<1, 256, msm2, stream>>>(T, G, rg_par.p, l, in_smem, rg_orig.p, rg_moves.p);
            launches++;
            AMR_CUDA(cudaGetLastError());
            if ((rc = rg_counts(c))) return rc;
            const int nm = c[6];
            if (nm) {
                AmrDev A = view();
                const unsigned cy = (unsigned)std::max(1, std::min(16, 296 / nm));
                NVK(pool_move_list)<<<dim3((unsigned)nm, cy), 256, 0, stream>>>(A, rg_moves.p);
                launches++;
                AMR_CUDA(cudaGetLastError());
            }
            if ((rc = rg_mirror())) return rc;
        }
        rate_valid = false;
        return EMG_OK;
    }

    std::vector<std::tuple<int, Key, bool>> structure() const {
        std::vector<std::tuple<int, Key, bool>> s;
        for (auto& b : blocks) s.push_back({b.level, b.idx, b.leaf});
        return s;
    }

    // C/amr.rs:1470-1537
    int step(double dt) {
        int rc = ensure_layout();
        if (rc) return rc;
        ctl_host->dt = dt;
        ctl_host->done = 0;
        ctl_host->status = 0;
        ctl_host->rate_bits = 0;
        AMR_CUDA(cudaMemcpyAsync(ctl, ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, stream));
        if ((opts.flags & EMG_OPT_AUTOTUNE) && !tuned) {
            tuned = true;
            if ((rc = autotune_sweeps())) return rc;
            // the timing launches counted faces and fallbacks: restore the control block
            AMR_CUDA(cudaMemcpyAsync(ctl, ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, stream));
        }
        if ((rc = make_events())) return rc;
        if ((rc = run_step_body())) return rc;
        stage_pending = true;
        uint64_t f = 0;
        for (int d : dims) f += (uint64_t)nleaves * (bcells() / bd[d]) * (bd[d] + 1);
        faces += 3 * f;
        if (opts.mode == EMG_MODE_WENO) weno_faces += 3 * f;
        AMR_CUDA(cudaMemcpyAsync(ctl_host, ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaStreamSynchronize(stream));
        collect_times();
        rate_valid = true;
        t += dt;
        steps += 1;
        if (ctl_host->status == EMG_ERR_INADMISSIBLE) return inadmissible();
        if (steps >= next_regrid) {
            cudaEvent_t a, b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, stream);
            auto before = structure();
            if ((rc = regrid())) return rc;
            const bool changed = structure() != before;
            regrid_interval = changed ? cfg.regrid_every : std::min(2 * regrid_interval, 2 * cfg.regrid_every);
            next_regrid = steps + regrid_interval;
            cudaEventRecord(b, stream);
            cudaEventSynchronize(b);
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            phase_ms[4] += ms;
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
        unsigned int e = 0;
        AMR_CUDA(cudaMemcpy(&e, err, sizeof e, cudaMemcpyDeviceToHost));
        if ((e & 4u) || ctl_host->status == EMG_ERR_BOUNDS)
            return set_error(EMG_ERR_BOUNDS, "device index out of range (bounds-check build)");
        if (e) return set_error(EMG_ERR_UNFILLABLE, "AMR ghost cell without a source (prediction depth or box)");
        return EMG_OK;
    }

    int dt_cfl(double* dt) {
        if (!rate_valid) {
            int rc = ensure_layout();
            if (rc) return rc;
            ctl_host->rate_bits = 0;
            ctl_host->status = 0;
            AMR_CUDA(cudaMemcpyAsync(ctl, ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, stream));
            AmrDev A = view();
            PHK(amr_cfl)<<<dim3((unsigned)nleaves, (unsigned)std::min<int64_t>((bcells() + 255) / 256, 16)), 256, 0, stream>>>(
                A, dleaves.p, dlevel.p, ddxl.p, ctl);
            launches++;
            AMR_CUDA(cudaGetLastError());
        }
        unsigned long long sbits = 0;
        if (nv == 7) {
            // the dilatation limit of the multiphase system (C/amr.rs:1426-1461)
            int rc = ensure_layout();
            if (rc) return rc;
            if (!src_bits) AMR_CUDA(cudaMalloc(&src_bits, sizeof(unsigned long long)));
            AMR_CUDA(cudaMemsetAsync(src_bits, 0, sizeof(unsigned long long), stream));
            AmrDev A = view();
            int64_t ninner = 1, nface = 1;
            for (int d = 0; d < 3; d++) {
                ninner *= act[d] ? bd[d] - 2 : 1;
                nface = std::max<int64_t>(nface, bcells() / std::max(bd[d], 1));
            }
            amr_dilatation_five<<<dim3((unsigned)nleaves, (unsigned)std::min<int64_t>((ninner + 255) / 256, 16)), 256, 0,
                                  stream>>>(A, dleaves.p, dlevel.p, didx.p, ddxl.p, src_bits);
            amr_dilatation_five_faces<<<dim3((unsigned)nleaves, (unsigned)(2 * dims.size()),
                                             (unsigned)std::min<int64_t>((nface + 127) / 128, 32)),
                                        128, 0, stream>>>(A, dleaves.p, dlevel.p, didx.p, ddxl.p, src_bits);
            launches += 2;
            AMR_CUDA(cudaGetLastError());
            AMR_CUDA(cudaMemcpyAsync(&sbits, src_bits, sizeof sbits, cudaMemcpyDeviceToHost, stream));
        }
        AMR_CUDA(cudaMemcpyAsync(ctl_host, ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaStreamSynchronize(stream));
        rate_valid = true;
        if (ctl_host->status == EMG_ERR_INADMISSIBLE) return inadmissible();
        double rate;
        std::memcpy(&rate, &ctl_host->rate_bits, sizeof rate);
        *dt = opts.cfl / rate;
        if (nv == 7) {
            double src;
            std::memcpy(&src, &sbits, sizeof src);
            if (src > 0.0) *dt = std::fmin(*dt, 0.5 / src);
        }
        return EMG_OK;
    }
    unsigned long long* src_bits = nullptr;  // dilatation rate of the five-equation CFL step

    static int inadmissible() {
        return set_error(EMG_ERR_INADMISSIBLE,
                         "non-finite or inadmissible state (density, pressure or specific volume) in a leaf cell");
    }

    // ---------------------------------------------------------------- subcycling
    // Amr::step_subcycled (C/amr.rs:1654-1954) with the reference's schedule on
    // the host: level l advances every block of the level (leaves and covered
    // ancestors) with its own dt, its ghost prediction reads the coarser level
    // interpolated in time, coarse–fine faces are corrected from flux
    // registers, and ancestors are restricted from the finer level after its
    // two half steps. Launches run eagerly (no step graph): θ of the time
    // views depends on t and dt of every step.

    // per-level lists, rebuilt with the layout
    int ensure_sc_layout() {
        int rc = ensure_layout();
        if (rc) return rc;
        if (sc_gen == layout_gen) return EMG_OK;
        if ((int)sc.size() < levels) sc.resize(levels);
        std::vector<int> all(blocks.size());
        for (size_t i = 0; i < blocks.size(); i++) all[i] = (int)i;
        if ((rc = dall.put(all, stream))) return rc;
        int nreg = 0;
        int64_t scr_need = 0;
        for (int l = 0; l < levels; l++) {
            ScLevel& L = sc[l];
            std::vector<int> ids;
            for (size_t i = 0; i < blocks.size(); i++)
                if (blocks[i].level == l) ids.push_back((int)i);
            L.nblk = (int)ids.size();
            std::vector<CopyTask> copies;
            std::vector<PBox> pboxes;
            std::vector<int> bcl;
            int64_t pmax = 0, poff = 0;
            ghost_tasks(ids, copies, pboxes, bcl, pmax, poff);
            for (int d = 0; d < 3; d++) {
                L.nch[d] = 0;
                if (!act[d]) continue;
                std::vector<int> coff, cslot;
                build_chains(d, ids, coff, cslot, true);
                if ((rc = L.choff[d].put(coff, stream)) || (rc = L.chslot[d].put(cslot, stream))) return rc;
                L.nch[d] = (int)coff.size() - 1;
            }
            L.ncopy = (int)copies.size();
            L.npbox = (int)pboxes.size();
            L.nbcl = (int)bcl.size();
            L.pmax = pmax;
            if (!pbox_fused_fits(pmax)) scr_need = std::max(scr_need, poff);
            // whole-block restriction of every ancestor (restrict_level_full, C/amr.rs:1902-1910)
            std::vector<RBox> rb;
            L.rchunk.clear();
            L.rchunk_max.clear();
            int64_t off = 0, mx = 0;
            for (int id : ids) {
                if (blocks[id].leaf) continue;
                if (rb.size() % SC_RCHUNK == 0) {
                    if (!rb.empty()) L.rchunk_max.push_back(mx);
                    L.rchunk.push_back((int)rb.size());
                    off = 0;
                    mx = 0;
                }
                RBox r = make_rbox(l, id, blocks[id].idx, {0, 0, 0}, {bd[0], bd[1], bd[2]});
                r.off = off;
                off += r.cap;
                mx = std::max(mx, r.cap);
                scr_need = std::max(scr_need, off);
                rb.push_back(r);
            }
            if (!rb.empty()) L.rchunk_max.push_back(mx);
            L.rchunk.push_back((int)rb.size());
            // coarse–fine faces of the level's leaves, coarse side (C/amr.rs:1725-1760, kind 0)
            std::vector<ScFace> faces;
            L.reg0 = nreg;
            for (int bucket = 0; bucket < 6; bucket++) {
                L.face_start[bucket] = (int)faces.size();
                const int d = bucket / 2, side = bucket % 2;
                if (!act[d]) continue;
                const int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
                for (int id : ids) {
                    const HBlock& b = blocks[id];
                    if (!b.leaf || l + 1 >= levels) continue;
                    const int64_t nbk = nb0[d] << l;
                    Key nk = b.idx;
                    nk[d] += side == 1 ? 1 : -1;
                    if (nk[d] < 0 || nk[d] >= nbk) {
                        if (bckind(d, side) != EMG_BC_PERIODIC) continue;
                        nk[d] = erem(nk[d], nbk);
                    }
                    const int nj = get(l, nk);
                    if (!(nj >= 0 && !blocks[nj].leaf)) continue;
                    ScFace f{};
                    f.slot = id;
                    f.d = d;
                    f.side = side;
                    f.reg = nreg++;
                    f.dx = dxl[3 * l + d];
                    for (int qa = 0; qa < 2; qa++)
                        for (int qb = 0; qb < 2; qb++) {
                            f.fine[qa][qb] = -1;
                            if ((qa && !act[e0]) || (qb && !act[e1])) continue;
                            Key ck = nk;
                            ck[d] = 2 * nk[d] + (side == 1 ? 0 : 1);
                            ck[e0] = act[e0] ? 2 * b.idx[e0] + qa : 0;
                            ck[e1] = act[e1] ? 2 * b.idx[e1] + qb : 0;
                            const int cid = get(l + 1, ck);
                            if (cid >= 0 && blocks[cid].leaf) f.fine[qa][qb] = cid;
                        }
                    faces.push_back(f);
                }
            }
            L.face_start[6] = (int)faces.size();
            if ((rc = L.blist.put(ids, stream)) || (rc = L.copies.put(copies, stream)) ||
                (rc = L.pboxes.put(pboxes, stream)) || (rc = L.bcl.put(bcl, stream)) || (rc = L.rfull.put(rb, stream)) ||
                (rc = L.faces.put(faces, stream)))
                return rc;
        }
        if ((rc = scratch(scr_need))) return rc;
        if (nreg > reg_cap) {
            const int64_t want = std::max<int64_t>(nreg, 2 * reg_cap);
            cudaFree(creg);
            cudaFree(freg);
            creg = freg = nullptr;
            reg_cap = 0;
            if (cudaMalloc(&creg, (size_t)want * nv * npen * sizeof(double)) != cudaSuccess ||
                cudaMalloc(&freg, (size_t)want * nv * npen * sizeof(double)) != cudaSuccess) {
                cudaGetLastError();
                return set_error(EMG_ERR_CUDA, "flux register allocation failed");
            }
            reg_cap = want;
        }
        if (usave_cap != cap) {
            cudaFree(usave);
            usave = nullptr;
            usave_cap = 0;
            if (cudaMalloc(&usave, (size_t)cap * bcell * nv * sizeof(double)) != cudaSuccess) {
                cudaGetLastError();
                return set_error(EMG_ERR_CUDA, "time-view buffer allocation failed");
            }
            usave_cap = cap;
        }
        if (!level_rates) AMR_CUDA(cudaMalloc(&level_rates, AMR_MAX_LEVELS * sizeof(unsigned long long)));
        level_t0.resize(levels, 0.0);
        level_dt.resize(levels, 0.0);
        sc_gen = layout_gen;
        return EMG_OK;
    }

    int coarsest_leaf_level() const {  // C/amr.rs:1694-1700
        int m = -1;
        for (auto& b : blocks)
            if (b.leaf && (m < 0 || b.level < m)) m = b.level;
        return m < 0 ? 0 : m;
    }

    dim3 level_grid(int nblk) const { return dim3((unsigned)nblk, 1, 1); }

    int restrict_full(int l) {  // C/amr.rs:1902-1910
        if (l < 0 || l + 1 >= levels) return EMG_OK;
        ScLevel& L = sc[l];
        for (size_t c = 0; c + 1 < L.rchunk.size(); c++) {
            const int b0 = L.rchunk[c], nb = L.rchunk[c + 1] - b0;
            if (nb <= 0) continue;
            int rc = run_rboxes(L.rfull.p + b0, nb, L.rchunk_max[c]);
            if (rc) return rc;
        }
        return EMG_OK;
    }

    int fill_ghosts_level(int l) {
        ScLevel& L = sc[l];
        AmrDev A = view();
        if (L.ncopy) {
            NVK(ghost_copy)<<<L.ncopy, COPY_THREADS, 0, stream>>>(A, L.copies.p);
            launches++;
        }
        int rc = run_pboxes(L.pboxes.p, L.npbox, L.pmax);
        if (rc) return rc;
        if (L.nbcl)
            for (int di = 0; di < (int)dims.size(); di++) {
                NVK(ghost_bc)<<<box_grid(2 * (int64_t)ng * std::max(bd[0], 1) * std::max(bd[1], 1), L.nbcl), 256, 0, stream>>>(
                    A, L.bcl.p, dlevel.p, didx.p, di);
                launches++;
            }
        AMR_CUDA(cudaGetLastError());
        return EMG_OK;
    }

    // Amr::advance_level (C/amr.rs:1836-1900)
    int advance_level(int l, double dt, int lmin) {
        ScLevel& L = sc[l];
        if (!L.nblk) return EMG_OK;
        const double t0 = level_t0[l];
        level_dt[l] = dt;
        const int nf = L.face_start[6];
        if (nf) {
            AMR_CUDA(cudaMemsetAsync(creg + (size_t)L.reg0 * nv * npen, 0, (size_t)nf * nv * npen * sizeof(double), stream));
            AMR_CUDA(cudaMemsetAsync(freg + (size_t)L.reg0 * nv * npen, 0, (size_t)nf * nv * npen * sizeof(double), stream));
        }
        sc_set_dt<<<1, 1, 0, stream>>>(ctl, dt);
        launches++;
        const double stage_t[3] = {t0, t0 + dt, t0 + 0.5 * dt};
        const double weights[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
        const double nsub = (double)((size_t)1 << (dims.size() - 1));
        // the coarser level's time view: its blocks were all advanced in this
        // step; below lmin no level-l ghost reads the coarser level
        const bool view_on = l > 0 && l - 1 >= lmin && sc[l - 1].nblk > 0;
        uint64_t f = 0;
        for (int d : dims) f += (uint64_t)L.nblk * (bcells() / bd[d]) * (bd[d] + 1);
        int rc;
        AmrDev A = view();
        const unsigned gy = (unsigned)std::min<int64_t>((bcells() + 255) / 256, 16);
        for (int s = 0; s < 3; s++) {
            if (view_on) {
                const double pt0 = level_t0[l - 1], pdt = level_dt[l - 1];
                double th = 1.0;
                if (pdt > 0.0) {
                    th = (stage_t[s] - pt0) / pdt;
                    if (th < 0.0) th = 0.0;
                    if (th > 1.0) th = 1.0;
                }
                NVK(sc_time_view)<<<sc[l - 1].nblk, 256, 0, stream>>>(A, sc[l - 1].blist.p, u0, usave, th);
                launches++;
            }
            if ((rc = fill_ghosts_level(l))) return rc;
            if (view_on) {
                NVK(sc_restore)<<<sc[l - 1].nblk, 256, 0, stream>>>(A, sc[l - 1].blist.p, usave);
                launches++;
            }
            if ((rc = sweeps(s + 1, L.blist.p, L.nblk, &L))) return rc;
            const double w = weights[s] * dt;
            if (nf) {
                NVK(sc_reg_coarse)<<<nf, 256, 0, stream>>>(A, L.faces.p, face, npen, creg, w);
                launches++;
            }
            if (l > 0 && sc[l - 1].face_start[6]) {
                NVK(sc_reg_fine)<<<sc[l - 1].face_start[6], 256, 0, stream>>>(A, sc[l - 1].faces.p, face, npen, freg, w, nsub);
                launches++;
            }
            PHK(amr_rk)<<<dim3((unsigned)L.nblk, gy), 256, 0, stream>>>(A, u0, rhs, L.blist.p, dlevel.p, ddxl.p, s + 1, ctl, 1);
            launches++;
            AMR_CUDA(cudaGetLastError());
        }
        faces += 3 * f;
        if (opts.mode == EMG_MODE_WENO) weno_faces += 3 * f;
        if (l + 1 < levels && sc[l + 1].nblk) {
            level_t0[l + 1] = t0;
            if ((rc = advance_level(l + 1, 0.5 * dt, lmin))) return rc;
            level_t0[l + 1] = t0 + 0.5 * dt;
            if ((rc = advance_level(l + 1, 0.5 * dt, lmin))) return rc;
            for (int bucket = 0; bucket < 6; bucket++) {
                const int n = L.face_start[bucket + 1] - L.face_start[bucket];
                if (!n) continue;
                NVK(sc_reflux)<<<n, 256, 0, stream>>>(A, L.faces.p + L.face_start[bucket], creg, freg, npen);
                launches++;
            }
            AMR_CUDA(cudaGetLastError());
            if ((rc = restrict_full(l))) return rc;
        }
        level_t0[l] = t0 + dt;
        return EMG_OK;
    }

    int step_subcycled(double dt) {  // C/amr.rs:1912-1952
        int rc = ensure_sc_layout();
        if (rc) return rc;
        ctl_host->dt = dt;
        ctl_host->done = 0;
        ctl_host->status = 0;
        ctl_host->rate_bits = 0;
        AMR_CUDA(cudaMemcpyAsync(ctl, ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice, stream));
        for (int l = 0; l < levels; l++) level_t0[l] = t;
        for (int l = levels - 2; l >= 0; l--)
            if ((rc = restrict_full(l))) return rc;
        const int lmin = coarsest_leaf_level();
        if ((rc = advance_level(lmin, dt, lmin))) return rc;
        for (int l = lmin - 1; l >= 0; l--)
            if ((rc = restrict_full(l))) return rc;
        {  // CFL rate and admissibility of the new leaf states (amr.rs:1409-1427)
            AmrDev A = view();
            PHK(amr_cfl)<<<dim3((unsigned)nleaves, (unsigned)std::min<int64_t>((bcells() + 255) / 256, 16)), 256, 0, stream>>>(
                A, dleaves.p, dlevel.p, ddxl.p, ctl);
            launches++;
            AMR_CUDA(cudaGetLastError());
        }
        AMR_CUDA(cudaMemcpyAsync(ctl_host, ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, stream));
        AMR_CUDA(cudaStreamSynchronize(stream));
        rate_valid = true;  // the leaves' rate; a regrid below invalidates it
        t += dt;
        steps += 1;
        if (ctl_host->status == EMG_ERR_INADMISSIBLE) return inadmissible();
        if (next_regrid > steps + 2) next_regrid = steps + 1;
        if (steps >= next_regrid) {
            auto before = structure();
            if ((rc = regrid())) return rc;
            const bool changed = structure() != before;
            regrid_interval = changed ? cfg.regrid_every : std::min(2 * regrid_interval, 2 * cfg.regrid_every);
            next_regrid = steps + (changed ? 1 : 2);
        }
        unsigned int e = 0;
        AMR_CUDA(cudaMemcpy(&e, err, sizeof e, cudaMemcpyDeviceToHost));
        if ((e & 4u) || ctl_host->status == EMG_ERR_BOUNDS)
            return set_error(EMG_ERR_BOUNDS, "device index out of range (bounds-check build)");
        if (e) return set_error(EMG_ERR_UNFILLABLE, "AMR ghost cell without a source (prediction depth or box)");
        return EMG_OK;
    }

    // Amr::dt_cfl_subcycled (C/amr.rs:1681-1692)
    int dt_cfl_subcycled(double* out) {
        int rc = ensure_sc_layout();
        if (rc) return rc;
        AMR_CUDA(cudaMemsetAsync(level_rates, 0, AMR_MAX_LEVELS * sizeof(unsigned long long), stream));
        AmrDev A = view();
        if (!blocks.empty()) {
            PHK(sc_cfl_levels)<<<(unsigned)blocks.size(), 256, 0, stream>>>(A, dall.p, dlevel.p, ddxl.p, level_rates);
            launches++;
            AMR_CUDA(cudaGetLastError());
        }
        unsigned long long bits[AMR_MAX_LEVELS];
        AMR_CUDA(cudaMemcpyAsync(bits, level_rates, sizeof bits, cudaMemcpyDeviceToHost, stream));
        double g = 0.0;
        if ((rc = dt_cfl(&g))) return rc;  // synchronises the stream
        const int lmin = coarsest_leaf_level();
        double dt = INFINITY;
        for (int l = lmin; l < levels; l++) {
            double rate;
            std::memcpy(&rate, &bits[l], sizeof rate);
            const double dl = rate > 0.0 ? opts.cfl / rate : INFINITY;
            dt = std::fmin(dt, dl * (double)((uint64_t)1 << (l - lmin)));
        }
        int finest = 0;
        for (int l = levels - 1; l >= 0; l--) {
            bool any = false;
            for (auto& b : blocks) any = any || (b.level == l && b.leaf);
            if (any) {
                finest = l;
                break;
            }
        }
        *out = std::fmin(dt, g * (double)((uint64_t)1 << (finest - lmin)));
        return EMG_OK;
    }

    // Consistency of an adopted hierarchy (create_from_blocks), on the host
    // before any device work. Structure errors (a block outside the levels or
    // the domain, twice, without its parent, a leaf with children, an
    // ancestor without all 2^D children) are EMG_ERR_INVALID. A hierarchy
    // whose ghost cells would have no source — a base block missing, or a
    // block whose parent lacks a same-level neighbour, i.e. not 2:1 balanced
    // as Amr::refine_block keeps it (C/amr.rs:951-972) — is
    // EMG_ERR_UNFILLABLE: the ghost prediction reads one coarser level only.
    int check_hierarchy(const int64_t* desc, size_t nblocks) {
        std::vector<std::vector<int>> seen(levels);
        for (int l = 0; l < levels; l++) seen[l].assign(map[l].size(), -1);
        for (size_t i = 0; i < nblocks; i++) {
            const int64_t l = desc[5 * i];
            const Key k = {desc[5 * i + 1], desc[5 * i + 2], desc[5 * i + 3]};
            const int64_t sl = (l >= 0 && l < levels) ? slot_of((int)l, k) : -1;
            if (sl < 0) return set_error(EMG_ERR_INVALID, "block outside the hierarchy");
            if (seen[l][sl] >= 0) return set_error(EMG_ERR_INVALID, "block given twice");
            seen[l][sl] = (int)i;
        }
        auto has = [&](int l, Key k) -> bool {
            if (l < 0 || l >= levels) return false;
            for (int d = 0; d < 3; d++) {
                if (!act[d]) {
                    k[d] = 0;
                    continue;
                }
                const int64_t nbl_ = nb0[d] << l;
                if (k[d] < 0 || k[d] >= nbl_) {
                    if (bc[2 * d + (k[d] >= nbl_ ? 1 : 0)].kind != EMG_BC_PERIODIC) return true;  // outside: no block needed
                    k[d] = ((k[d] % nbl_) + nbl_) % nbl_;
                }
            }
            const int64_t sl = slot_of(l, k);
            return sl >= 0 && seen[l][sl] >= 0;
        };
        for (int64_t i = 0; i < nb0[0]; i++)
            for (int64_t j = 0; j < nb0[1]; j++)
                for (int64_t k = 0; k < nb0[2]; k++)
                    if (!has(0, Key{i, j, k}))
                        return set_error(EMG_ERR_UNFILLABLE, "a base block is missing: part of the domain has no source");
        int nkids = 1;
        for (int d = 0; d < 3; d++) nkids *= act[d] ? 2 : 1;
        for (size_t i = 0; i < nblocks; i++) {
            const int l = (int)desc[5 * i];
            const Key k = {desc[5 * i + 1], desc[5 * i + 2], desc[5 * i + 3]};
            const bool leaf = desc[5 * i + 4] != 0;
            int kids = 0;
            for (int c = 0; c < 8; c++) {
                Key ck = k;
                bool valid = true;
                for (int d = 0; d < 3; d++) {
                    const int bit = (c >> d) & 1;
                    if (!act[d]) {
                        if (bit) valid = false;
                        continue;
                    }
                    ck[d] = 2 * k[d] + bit;
                }
                if (valid && l + 1 < levels && has(l + 1, ck)) kids++;
            }
            if (leaf && kids > 0) return set_error(EMG_ERR_INVALID, "a leaf block has children");
            if (!leaf && kids != nkids) return set_error(EMG_ERR_INVALID, "an ancestor block lacks some of its children");
            if (l == 0) continue;
            Key pk = k;
            for (int d = 0; d < 3; d++) pk[d] = act[d] ? k[d] >> 1 : 0;
            if (!has(l - 1, pk)) return set_error(EMG_ERR_INVALID, "a block without its parent");
            for (int a = -1; a <= 1; a++)
                for (int b = -1; b <= 1; b++)
                    for (int c = -1; c <= 1; c++) {
                        const int o[3] = {a, b, c};
                        bool skip = false;
                        Key nk = pk;
                        for (int d = 0; d < 3; d++) {
                            if (!act[d] && o[d] != 0) skip = true;
                            nk[d] += o[d];
                        }
                        if (skip || (a == 0 && b == 0 && c == 0)) continue;
                        if (!has(l - 1, nk))
                            return set_error(EMG_ERR_UNFILLABLE,
                                             "ghost cells without a source: the hierarchy is not 2:1 balanced (a block's "
                                             "parent lacks a same-level neighbour)");
                    }
        }
        return EMG_OK;
    }

    // host part of the set-up (configuration checks, level geometry, block
    // map); no device work, so a bad configuration is reported on any host
    // f5: the five-equation system (nv = 7), or null for the Euler system `e`
    int setup_host(const emg_amr_config* c, const emg_eos* e, const emg_five_system* f5, const double* lo_,
                   const double* hi_, const emg_bc7* b, const emg_opts* o) {
        cfg = *c;
        if (f5) {
            nv = 7;
            five = *f5;
            eos = f5->eos[1];
        } else {
            eos = *e;
        }
        opts = *o;
        for (int d = 0; d < 3; d++) {
            lo[d] = lo_[d];
            hi[d] = hi_[d];
        }
        for (int i = 0; i < 6; i++) bc[i] = b[i];
        if (nv == 7 && opts.precision != EMG_PRECISION_F64 && opts.precision != EMG_PRECISION_F64_FAST)
            return set_error(EMG_ERR_INVALID, "the five-equation system runs in the plain or fast FP64 form only");
        if (cfg.b < 6 || cfg.levels < 1 || cfg.levels > AMR_MAX_LEVELS || cfg.regrid_every < 1)
            return set_error(EMG_ERR_INVALID, "invalid AMR configuration (b >= 6, 1 <= levels <= 12, regrid_every >= 1)");
        for (int i = 0; i < 6; i++) {
            if (bc[i].kind == EMG_BC_CHARACTERISTIC)
                return set_error(EMG_ERR_INVALID, "characteristic boundaries are not available on the AMR path");
            if (bc[i].kind < 0 || bc[i].kind > 4) return set_error(EMG_ERR_INVALID, "unknown boundary condition");
        }
        if (opts.mode != EMG_MODE_WENO && opts.mode != EMG_MODE_HYBRID && opts.mode != EMG_MODE_CENTRAL)
            return set_error(EMG_ERR_INVALID, "unknown flux mode");
        if (opts.mode == EMG_MODE_HYBRID && !(opts.tol > 0.0))
            return set_error(EMG_ERR_INVALID, "hybrid mode needs tol > 0");
        if (opts.precision != EMG_PRECISION_F64 && opts.precision != EMG_PRECISION_MIXED &&
            opts.precision != EMG_PRECISION_F64_FAST)
            return set_error(EMG_ERR_INVALID, "unknown precision");
        ng = (int)std::max<int64_t>(cfg.ghosts, 5);
        for (int d = 0; d < 3; d++) {
            bd[d] = cfg.base_blocks[d] == 0 ? 1 : (int)cfg.b;
            // C/amr.rs:251-253
            act[d] = cfg.base_blocks[d] > 0 && (hi[d] - lo[d]) > 0.0 && bd[d] > 1;
            nb0[d] = std::max<int64_t>(cfg.base_blocks[d], 1);
            ext[d] = act[d] ? bd[d] + 2 * ng : 1;
            gof[d] = act[d] ? ng : 0;
            if (act[d]) dims.push_back(d);
        }
        if (dims.empty()) return set_error(EMG_ERR_INVALID, "no active axis");
        for (int d : dims)
            if ((bc[2 * d].kind == EMG_BC_PERIODIC) != (bc[2 * d + 1].kind == EMG_BC_PERIODIC))
                return set_error(EMG_ERR_INVALID, "periodic boundaries must be paired");
        if (cfg.b > 32) return set_error(EMG_ERR_INVALID, "block side above 32");
        levels = (int)cfg.levels;
        dxl.assign(3 * levels, 0.0);
        for (int l = 0; l < levels; l++)
            for (int d = 0; d < 3; d++) dxl[3 * l + d] = (hi[d] - lo[d]) / (double)n_level(l, d);
        auto a = lagrange6(-3.0, -0.25), bb = lagrange6(-2.0, 0.25);
        for (int k = 0; k < 6; k++) {
            wp[0][k] = a[k];
            wp[1][k] = bb[k];
        }
        const double wr_[6] = {3.0 / 256.0, -25.0 / 256.0, 150.0 / 256.0, 150.0 / 256.0, -25.0 / 256.0, 3.0 / 256.0};
        std::memcpy(wr, wr_, sizeof wr);
        const int shifts[5] = {0, -1, 1, -2, 2};
        for (int m = 0; m < 5; m++) {
            auto w = m == 0 ? std::array<double, 6>{wr[0], wr[1], wr[2], wr[3], wr[4], wr[5]}
                            : lagrange6(-2.5 + (double)shifts[m], 0.0);
            for (int k = 0; k < 6; k++) wrs[m][k] = w[k];
        }
        bcell = (int64_t)ext[0] * ext[1] * ext[2];
        npen = 1;
        for (int d = 0; d < 3; d++) {
            int p = 1;
            for (int e2 = 0; e2 < 3; e2++)
                if (e2 != d) p *= bd[e2];
            npen = std::max(npen, p);
        }
        map.resize(levels);
        mapoff.assign(levels, 0);
        int64_t off = 0;
        for (int l = 0; l < levels; l++) {
            map[l].assign(nbl(l, 0) * nbl(l, 1) * nbl(l, 2), -1);
            mapoff[l] = off;
            off += (int64_t)map[l].size();
        }
        regrid_interval = cfg.regrid_every;
        next_regrid = cfg.regrid_every;
        return EMG_OK;
    }

    // device part of the set-up: stream, error word, control block, per-level dx
    int setup_device() {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            return set_error(EMG_ERR_NO_DEVICE, "no CUDA device visible");
        }
        AMR_CUDA(cudaGetDevice(&device));
        cudaDeviceProp pr;
        AMR_CUDA(cudaGetDeviceProperties(&pr, device));
        if (pr.major != 10) return set_error(EMG_ERR_NO_DEVICE, "device is not sm_100 (B200)");
        AMR_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        AMR_CUDA(cudaMalloc(&err, sizeof(unsigned int)));
        AMR_CUDA(cudaMemset(err, 0, sizeof(unsigned int)));
        AMR_CUDA(cudaMalloc(&ctl, sizeof(StepCtl)));
        AMR_CUDA(cudaMallocHost(&ctl_host, sizeof(StepCtl)));
        std::memset(ctl_host, 0, sizeof(StepCtl));
        ctl_host->t_end = INFINITY;
        AMR_CUDA(cudaMemcpy(ctl, ctl_host, sizeof(StepCtl), cudaMemcpyHostToDevice));
        int rc = ddxl.put(dxl, stream);
        if (rc) return rc;
        if (sweep_prepare_device() != cudaSuccess) return set_error(EMG_ERR_CUDA, "sweep setup failed");
        if (nv == 7 && five_sweep_prepare_device() != cudaSuccess) return set_error(EMG_ERR_CUDA, "sweep setup failed");
        return EMG_OK;
    }

    int setup(const emg_amr_config* c, const emg_eos* e, const emg_five_system* f5, const double* lo_,
              const double* hi_, const emg_bc7* b, const emg_opts* o) {
        int rc = setup_host(c, e, f5, lo_, hi_, b, o);
        return rc ? rc : setup_device();
    }

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        collect_times();
        drop_graph();
        for (auto& st : stage_ev)
            for (auto& e : st)
                if (e) cudaEventDestroy(e);
        cudaFree(u);
        cudaFree(u0);
        cudaFree(rhs);
        cudaFree(face);
        cudaFree(err);
        cudaFree(ctl);
        if (ctl_host) cudaFreeHost(ctl_host);
        for (int i = 0; i < 2; i++) {
            cudaFree(scr[i]);
            cudaFree(sok[i]);
        }
        cudaFree(det);
        cudaFree(usave);
        cudaFree(src_bits);
        cudaFree(creg);
        cudaFree(freg);
        cudaFree(level_rates);
        for (auto& L : sc) {
            L.blist.release();
            L.copies.release();
            L.pboxes.release();
            L.bcl.release();
            L.rfull.release();
            L.faces.release();
            for (int d = 0; d < 3; d++) {
                L.choff[d].release();
                L.chslot[d].release();
            }
        }
        dall.release();
        dmap.release();
        dmap_edits.release();
        dleaves.release();
        for (int d = 0; d < 3; d++) {
            dchain_off[d].release();
            dchain_slot[d].release();
        }
        dlevel.release();
        dbcleaves.release();

        didx.release();

        ddxl.release();
        dcopy.release();
        dcopy_sweep.release();
        dpbox.release();
        for (auto& r : drbox) r.release();
        for (auto& a : drbsel)
            for (auto& v : a) v.release();
        dreflux.release();
        dtmp_pbox.release();
        dtmp_rbox.release();
        for (auto* v : {&rg_level, &rg_leaf, &rg_count, &rg_events, &rg_rem, &rg_orig, &rg_moves}) v->release();
        for (auto* v : {&rg_idx, &rg_ckey, &rg_par}) v->release();
        for (auto* v : {&rg_f, &rg_wantd, &rg_mark}) v->release();
        dstage.release();
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

}  // extern "C"

namespace {
// emg_bc → emg_bc7 (5 Dirichlet values, the rest zero)
void widen_bcs(const emg_bc* bc, emg_bc7* out) {
    for (int i = 0; i < 6; i++) {
        out[i] = emg_bc7{};
        out[i].kind = bc[i].kind;
        for (int k = 0; k < 5; k++) out[i].state[k] = bc[i].state[k];
    }
}

// Amr::new (C/amr.rs:289-344) for either system
int amr_create(const emg_amr_config* cfg, const emg_eos* eos, const emg_five_system* f5, const double* lo,
               const double* hi, const emg_bc7* bc, const emg_opts* opts, emg_init_fn init, void* ctx, emg_amr** out) {
    *out = nullptr;
    emg_amr* h = new emg_amr();
    int rc = h->setup(cfg, eos, f5, lo, hi, bc, opts);
    auto bail = [&](int code) {
        h->release();
        delete h;
        return code;
    };
    if (rc) return bail(rc);
    for (int64_t i = 0; i < h->nb0[0]; i++)
        for (int64_t j = 0; j < h->nb0[1]; j++)
            for (int64_t k = 0; k < h->nb0[2]; k++) {
                const int id = (int)h->blocks.size();
                if ((rc = h->add_block(0, Key{i, j, k}))) return bail(rc);
                if ((rc = h->init_block_data(id, init, ctx))) return bail(rc);
            }
    for (int it = 0; it < h->levels; it++) {
        std::vector<int8_t> f;
        if ((rc = h->flags(f))) return bail(rc);
        std::vector<std::pair<int, Key>> keys;
        for (size_t i = 0; i < h->blocks.size(); i++)
            if (f[i] > 0 && h->blocks[i].leaf) keys.push_back({h->blocks[i].level, h->blocks[i].idx});
        if (keys.empty()) break;
        for (auto& k : keys) {
            int id = h->get(k.first, k.second);
            if (id >= 0 && (rc = h->refine_block(id, init, ctx))) return bail(rc);
        }
    }
    if ((rc = h->reserve_headroom())) return bail(rc);
    *out = h;
    return EMG_OK;
}

int amr_create_from_blocks(const emg_amr_config* cfg, const emg_eos* eos, const emg_five_system* f5, const double* lo,
                           const double* hi, const emg_bc7* bc, const emg_opts* opts, const int64_t* desc,
                           size_t nblocks, const double* u, emg_amr** out) {
    *out = nullptr;
    if (nblocks == 0) return set_error(EMG_ERR_INVALID, "a hierarchy needs at least one block");
    emg_amr* h = new emg_amr();
    auto bail = [&](int code) {
        h->release();
        delete h;
        return code;
    };
    int rc = h->setup_host(cfg, eos, f5, lo, hi, bc, opts);
    if (rc) return bail(rc);
    // the hierarchy is checked on the host before any device work
    if ((rc = h->check_hierarchy(desc, nblocks))) return bail(rc);
    if ((rc = h->setup_device())) return bail(rc);
    if ((rc = h->reserve((int64_t)nblocks))) return bail(rc);
    for (size_t i = 0; i < nblocks; i++) {
        const int l = (int)desc[5 * i];
        const Key k = {desc[5 * i + 1], desc[5 * i + 2], desc[5 * i + 3]};
        h->blocks.push_back(HBlock{l, k, desc[5 * i + 4] != 0});
        h->insert(l, k, (int)i);
    }
    const int64_t nb = h->bcells();
    const int nv = h->nv;
    double* tmp = nullptr;
    if (cudaMalloc(&tmp, (size_t)nb * nv * sizeof(double)) != cudaSuccess) return bail(set_error(EMG_ERR_CUDA, "alloc"));
    AmrDev A = h->view();
    for (size_t i = 0; i < nblocks; i++) {
        cudaMemcpyAsync(tmp, u + i * nb * nv, (size_t)nb * nv * sizeof(double), cudaMemcpyHostToDevice, h->stream);
        NVK(pool_put_interior)<<<16, 256, 0, h->stream>>>(A, (int)i, tmp);
    }
    cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    if ((rc = h->reserve_headroom())) return bail(rc);
    *out = h;
    return EMG_OK;
}
}  // namespace

extern "C" {

int emg_amr_create(const emg_amr_config* cfg, const emg_eos* eos, const double lo[3], const double hi[3],
                   const emg_bc bc[6], const emg_opts* opts, emg_init_fn init, void* ctx, emg_amr** out) {
    if (!cfg || !eos || !lo || !hi || !bc || !opts || !init || !out) return set_error(EMG_ERR_INVALID, "null argument");
    emg_bc7 b7[6];
    widen_bcs(bc, b7);
    return amr_create(cfg, eos, nullptr, lo, hi, b7, opts, init, ctx, out);
}

int emg_amr_create_five(const emg_amr_config* cfg, const emg_five_system* sys, const double lo[3], const double hi[3],
                        const emg_bc7 bc[6], const emg_opts* opts, emg_init_fn init, void* ctx, emg_amr** out) {
    if (!cfg || !sys || !lo || !hi || !bc || !opts || !init || !out) return set_error(EMG_ERR_INVALID, "null argument");
    return amr_create(cfg, nullptr, sys, lo, hi, bc, opts, init, ctx, out);
}

int emg_amr_create_from_blocks(const emg_amr_config* cfg, const emg_eos* eos, const double lo[3], const double hi[3],
                               const emg_bc bc[6], const emg_opts* opts, const int64_t* desc, size_t nblocks,
                               const double* u, emg_amr** out) {
    if (!cfg || !eos || !lo || !hi || !bc || !opts || !desc || !u || !out) return set_error(EMG_ERR_INVALID, "null argument");
    emg_bc7 b7[6];
    widen_bcs(bc, b7);
    return amr_create_from_blocks(cfg, eos, nullptr, lo, hi, b7, opts, desc, nblocks, u, out);
}

int emg_amr_create_five_from_blocks(const emg_amr_config* cfg, const emg_five_system* sys, const double lo[3],
                                    const double hi[3], const emg_bc7 bc[6], const emg_opts* opts,
                                    const int64_t* desc, size_t nblocks, const double* u, emg_amr** out) {
    if (!cfg || !sys || !lo || !hi || !bc || !opts || !desc || !u || !out)
        return set_error(EMG_ERR_INVALID, "null argument");
    return amr_create_from_blocks(cfg, nullptr, sys, lo, hi, bc, opts, desc, nblocks, u, out);
}

int emg_amr_nv(emg_amr* h, int32_t* nv) {
    if (!h || !nv) return set_error(EMG_ERR_INVALID, "null argument");
    *nv = h->nv;
    return EMG_OK;
}

int emg_amr_destroy(emg_amr* h) {
    if (!h) return EMG_OK;
    cudaSetDevice(h->device);
    h->release();
    delete h;
    return EMG_OK;
}

static int amr_check(emg_amr* h) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    if (cudaSetDevice(h->device) != cudaSuccess) return set_error(EMG_ERR_CUDA, "cudaSetDevice failed");
    return EMG_OK;
}

int emg_amr_step(emg_amr* h, double dt) {
    int rc = amr_check(h);
    return rc ? rc : h->step(dt);
}

int emg_amr_dt_cfl(emg_amr* h, double* dt) {
    int rc = amr_check(h);
    if (rc) return rc;
    if (!dt) return set_error(EMG_ERR_INVALID, "null dt");
    return h->dt_cfl(dt);
}

int emg_amr_run_to(emg_amr* h, double t_end, uint64_t* steps) {
    int rc = amr_check(h);
    if (rc) return rc;
    const bool sub = (h->opts.flags & EMG_OPT_SUBCYCLE) != 0;
    uint64_t n = 0;
    while (h->t < t_end * (1.0 - 1e-14)) {
        double dt = 0.0;
        if ((rc = sub ? h->dt_cfl_subcycled(&dt) : h->dt_cfl(&dt))) return rc;
        dt = std::fmin(dt, t_end - h->t);
        if (!(std::isfinite(dt) && dt > 0.0)) return set_error(EMG_ERR_DT_COLLAPSED, "time step collapsed");
        if ((rc = sub ? h->step_subcycled(dt) : h->step(dt))) return rc;
        n++;
    }
    if (steps) *steps = n;
    return EMG_OK;
}

int emg_amr_step_subcycled(emg_amr* h, double dt) {
    int rc = amr_check(h);
    if (rc) return rc;
    if (!(std::isfinite(dt) && dt > 0.0)) return set_error(EMG_ERR_INVALID, "dt must be finite and positive");
    return h->step_subcycled(dt);
}

int emg_amr_dt_cfl_subcycled(emg_amr* h, double* dt) {
    int rc = amr_check(h);
    if (rc) return rc;
    if (!dt) return set_error(EMG_ERR_INVALID, "null dt");
    return h->dt_cfl_subcycled(dt);
}

int emg_amr_regrid(emg_amr* h) {
    int rc = amr_check(h);
    return rc ? rc : h->regrid();
}

int emg_amr_block_count(emg_amr* h, uint64_t* blocks, uint64_t* leaves) {
    if (!h) return set_error(EMG_ERR_INVALID, "null handle");
    uint64_t n = 0;
    for (auto& b : h->blocks) n += b.leaf ? 1 : 0;
    if (blocks) *blocks = h->blocks.size();
    if (leaves) *leaves = n;
    return EMG_OK;
}

int emg_amr_structure(emg_amr* h, int64_t* desc, size_t cap) {
    if (!h || !desc) return set_error(EMG_ERR_INVALID, "null argument");
    if (cap < h->blocks.size()) return set_error(EMG_ERR_INVALID, "structure buffer too small");
    for (size_t i = 0; i < h->blocks.size(); i++) {
        desc[5 * i] = h->blocks[i].level;
        for (int d = 0; d < 3; d++) desc[5 * i + 1 + d] = h->blocks[i].idx[d];
        desc[5 * i + 4] = h->blocks[i].leaf ? 1 : 0;
    }
    return EMG_OK;
}

int emg_amr_download(emg_amr* h, double* u, size_t nblocks) {
    int rc = amr_check(h);
    if (rc) return rc;
    if (!u || nblocks < h->blocks.size()) return set_error(EMG_ERR_INVALID, "buffer too small");
    const int nv = h->nv;
    const size_t n = h->blocks.size() * (size_t)h->bcells() * nv;
    double* tmp = nullptr;
    AMR_CUDA(cudaMalloc(&tmp, n * sizeof(double)));
    AmrDev A = h->view();
    NVK(pool_get_interior)<<<256, 256, 0, h->stream>>>(A, (int)h->blocks.size(), tmp);
    cudaMemcpyAsync(u, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    cudaStreamSynchronize(h->stream);
    cudaFree(tmp);
    AMR_CUDA(cudaGetLastError());
    return EMG_OK;
}

int emg_amr_totals(emg_amr* h, double* out) {
    if (!h || !out) return set_error(EMG_ERR_INVALID, "null argument");
    // host sum in the reference order (C/amr.rs:1991-2005) over downloaded leaves
    const int nv = h->nv;
    std::vector<double> u(h->blocks.size() * (size_t)h->bcells() * nv);
    int rc = emg_amr_download(h, u.data(), h->blocks.size());
    if (rc) return rc;
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (size_t i = 0; i < h->blocks.size(); i++) {
        if (!h->blocks[i].leaf) continue;
        double vol = 1.0;
        for (int d : h->dims) vol = vol * h->dxl[3 * h->blocks[i].level + d];
        const double* b = &u[i * h->bcells() * nv];
        for (int64_t c = 0; c < h->bcells(); c++)
            for (int q = 0; q < nv; q++) s[q] = s[q] + b[nv * c + q] * vol;
    }
    for (int q = 0; q < nv; q++) out[q] = s[q];
    return EMG_OK;
}

int emg_amr_counters(emg_amr* h, uint64_t out[4]) {
    int rc = amr_check(h);
    if (rc) return rc;
    AMR_CUDA(cudaMemcpyAsync(h->ctl_host, h->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, h->stream));
    AMR_CUDA(cudaStreamSynchronize(h->stream));
    out[0] = h->faces;
    out[1] = h->weno_faces + h->ctl_host->counters[1];
    out[2] = h->ctl_host->counters[2];
    out[3] = h->ctl_host->counters[3];
    return EMG_OK;
}

int emg_amr_get_time(emg_amr* h, double* t) {
    if (!h || !t) return set_error(EMG_ERR_INVALID, "null argument");
    *t = h->t;
    return EMG_OK;
}

int emg_amr_steps(emg_amr* h, uint64_t* steps) {
    if (!h || !steps) return set_error(EMG_ERR_INVALID, "null argument");
    *steps = (uint64_t)h->steps;
    return EMG_OK;
}

int emg_amr_synchronize(emg_amr* h) {
    int rc = amr_check(h);
    if (rc) return rc;
    AMR_CUDA(cudaStreamSynchronize(h->stream));
    return EMG_OK;
}

int emg_amr_stream(emg_amr* h, void** stream) {
    if (!h || !stream) return set_error(EMG_ERR_INVALID, "null argument");
    *stream = (void*)h->stream;
    return EMG_OK;
}

int emg_amr_phase_times(emg_amr* h, double out[5]) {
    int rc = amr_check(h);
    if (rc) return rc;
    cudaStreamSynchronize(h->stream);
    h->collect_times();
    for (int i = 0; i < 5; i++) {
        out[i] = h->phase_ms[i];
        h->phase_ms[i] = 0.0;
    }
    return EMG_OK;
}

int emg_amr_launch_count(emg_amr* h, uint64_t* launches) {
    if (!h || !launches) return set_error(EMG_ERR_INVALID, "null argument");
    *launches = h->launches;
    return EMG_OK;
}

}  // extern "C"
