// CPU ORACLE — test infrastructure only (see oracle.hpp).
//
// C++ restatement of the reference block-AMR solver:
// fluid/crates/compressible/src/amr.rs:1-2005, the global time step and the
// subcycled one (:1654-1954; the reference runs that on the CPU only, its GPU
// path refuses it, compressible-cuda/src/amr.rs:140-142). Same block pool,
// dense per-level index, sampling / prediction / restriction operators,
// refluxing, flux registers, wavelet regrid with 2:1 balance, and SSP-RK3
// stepping, in the reference's operation order.
#pragma once
#include "five_oracle.hpp"
#include "oracle.hpp"
#include <functional>
#include <map>
#include <set>
#include <tuple>

namespace oracle {

inline int64_t div_euclid(int64_t a, int64_t b) {
    int64_t q = a / b;
    if (a % b < 0) q -= 1;
    return q;
}

// amr.rs:41-47
inline std::array<double, 6> lagrange6(double x0, double x) {
    std::array<double, 6> w;
    for (int k = 0; k < 6; k++) {
        double xk = x0 + k;
        double p = 1.0;
        for (int j = 0; j < 6; j++)
            if (j != k) p = p * ((x - (x0 + j)) / (xk - (x0 + j)));
        w[k] = p;
    }
    return w;
}

// amr.rs:49-63
struct AmrConfig {
    int64_t b;
    int64_t levels;
    double eps;
    int64_t regrid_every;
    int64_t base_blocks[3];
    int64_t ghosts;
};

using Key3 = std::array<int64_t, 3>;
using InitFn = std::function<void(const double* x, int64_t n, double* w)>;  // batched primitive init

// The physical system of a block hierarchy (Amr<N, S>, amr.rs:208): the
// conserved vector, the momentum index, the line flux routine (with the face
// velocities of the non-conservative term) and whether the multiphase terms
// apply — the non-conservative α term in the block residual (amr.rs:1276-1279)
// and the dilatation limit of the CFL step (amr.rs:1426-1461).
struct AmrEuler {
    static constexpr int N = 5, IU = 1;
    static constexpr bool MULTIPHASE = false;
    using Sys = Euler<double>;
    using V = V5<double>;
    using BcT = Bc<double>;
    static void fluxes(const Sys& s, const V* line, int len, int d, int ng, const SchemeOpts& o, V* fl, double*,
                       Stats& st) {
        line_fluxes(s, line, len, d, ng, o, fl, (double*)nullptr, st);
    }
    static V char_layer(const Sys& s, const V& ub, const V& ub1, const V& far, int d, int side, double m) {
        return characteristic_ghost_layer(s, ub, ub1, far, d, side, m);
    }
};
struct AmrFive {
    static constexpr int N = 7, IU = 2;
    static constexpr bool MULTIPHASE = true;
    using Sys = FiveEq<double>;
    using V = V7<double>;
    using BcT = Bc7<double>;
    static void fluxes(const Sys& s, const V* line, int len, int d, int ng, const SchemeOpts& o, V* fl, double* uf,
                       Stats& st) {
        line_fluxes7(s, line, len, d, ng, o, fl, uf, st);
    }
    static V char_layer(const Sys& s, const V& ub, const V& ub1, const V& far, int d, int side, double m) {
        return CharStencil7<double>(s, ub, ub1, far, d, side).conserved(s, m);
    }
};

template <class V> struct AmrBlockT {  // amr.rs:194-206
    int64_t level;
    Key3 idx;
    bool leaf = true;
    std::vector<V> u, u0, u_save, rhs;
    std::vector<V> face[3][2];
};

template <class S> struct AmrT {
    using V = typename S::V;
    using BcT = typename S::BcT;
    using AmrBlock = AmrBlockT<V>;
    static constexpr int N = S::N;
    typename S::Sys sys;
    AmrConfig cfg;
    double lo[3], hi[3];
    BcT bc[3][2];
    int mode = HYBRID;
    double tol = 1e-3;
    double cfl = 0.4;
    bool positivity = true;
    double t = 0.0;
    int64_t steps = 0;
    Stats stats;
    std::vector<AmrBlock> blocks;
    // dense per-level index (amr.rs:67-131)
    int64_t nb0[3];
    bool act[3];
    std::vector<std::vector<int32_t>> map;
    int64_t ng;
    std::array<std::array<double, 6>, 2> wp;
    std::array<double, 6> wr;
    double stage_dt = 0.0;
    int64_t regrid_interval, next_regrid;
    // subcycling (amr.rs:233-245): per-level start time and step of the level
    // step in flight; flux registers keyed by (coarse leaf block, direction,
    // side, face index). The reference keeps the registers in hash maps and
    // applies them in hash order; ordered maps give the fixed order of
    // reflux_level below.
    bool subcycle = false;
    std::vector<double> level_t0, level_dt;
    using RegKey = std::tuple<int64_t, int, int, int64_t>;
    std::map<RegKey, V> creg, freg;

    // ---- geometry (amr.rs:251-292)
    bool active(int d) const { return cfg.base_blocks[d] > 0 && (hi[d] - lo[d]) > 0.0 && bd(d) > 1; }
    int64_t bd(int d) const { return cfg.base_blocks[d] == 0 ? 1 : cfg.b; }
    std::vector<int> dims() const {
        std::vector<int> v;
        for (int d = 0; d < 3; d++)
            if (active(d)) v.push_back(d);
        return v;
    }
    int64_t n_level(int64_t l, int d) const { return active(d) ? cfg.base_blocks[d] * cfg.b * (int64_t(1) << l) : 1; }
    double dx(int64_t l, int d) const { return (hi[d] - lo[d]) / (double)n_level(l, d); }
    int64_t bcells() const { return bd(0) * bd(1) * bd(2); }
    int64_t cidx(int64_t c0, int64_t c1, int64_t c2) const { return (c0 * bd(1) + c1) * bd(2) + c2; }
    void x(int64_t l, const Key3& g, double* out) const {
        for (int d = 0; d < 3; d++)
            out[d] = active(d) ? lo[d] + ((double)g[d] + 0.5) * dx(l, d) : 0.5 * (lo[d] + hi[d]);
    }

    // ---- block index
    int64_t nbl(int64_t l, int d) const { return act[d] ? nb0[d] << l : 1; }
    int64_t slot(int64_t l, const Key3& k) const {
        if (l < 0 || l >= (int64_t)map.size()) return -1;
        int64_t s = 0;
        for (int d = 0; d < 3; d++) {
            int64_t n = nbl(l, d);
            if (k[d] < 0 || k[d] >= n) return -1;
            s = s * n + k[d];
        }
        return s;
    }
    int64_t get(int64_t l, const Key3& k) const {
        int64_t s = slot(l, k);
        if (s < 0) return -1;
        return map[l][s];
    }
    void insert(int64_t l, const Key3& k, int64_t id) {
        int64_t s = slot(l, k);
        if (s >= 0) map[l][s] = (int32_t)id;
    }
    void remove(int64_t l, const Key3& k) {
        int64_t s = slot(l, k);
        if (s >= 0) map[l][s] = -1;
    }

    // ---- construction (amr.rs:289-344)
    AmrT(const typename S::Sys& s, const AmrConfig& c, const double* lo_, const double* hi_, const BcT (&b)[3][2],
         const InitFn& init)
        : sys(s), cfg(c) {
        for (int d = 0; d < 3; d++) {
            lo[d] = lo_[d];
            hi[d] = hi_[d];
            bc[d][0] = b[d][0];
            bc[d][1] = b[d][1];
        }
        ng = std::max<int64_t>(cfg.ghosts, 5);
        wp[0] = lagrange6(-3.0, -0.25);
        wp[1] = lagrange6(-2.0, 0.25);
        wr = {3.0 / 256.0, -25.0 / 256.0, 150.0 / 256.0, 150.0 / 256.0, -25.0 / 256.0, 3.0 / 256.0};
        regrid_interval = cfg.regrid_every;
        next_regrid = cfg.regrid_every;
        level_t0.assign(cfg.levels, 0.0);
        level_dt.assign(cfg.levels, 0.0);
        for (int d = 0; d < 3; d++) {
            nb0[d] = std::max<int64_t>(cfg.base_blocks[d], 1);
            act[d] = active(d);
        }
        map.resize(cfg.levels);
        for (int64_t l = 0; l < cfg.levels; l++) map[l].assign(nbl(l, 0) * nbl(l, 1) * nbl(l, 2), -1);
        for (int64_t i = 0; i < nb0[0]; i++)
            for (int64_t j = 0; j < nb0[1]; j++)
                for (int64_t k = 0; k < nb0[2]; k++) add_block(0, {i, j, k}, init);
        for (int64_t it = 0; it < cfg.levels; it++) {
            restrict_all();
            std::vector<int8_t> fl = flags();
            std::vector<std::pair<int64_t, Key3>> keys;
            for (size_t i = 0; i < blocks.size(); i++)
                if (fl[i] > 0 && blocks[i].leaf) keys.push_back({blocks[i].level, blocks[i].idx});
            if (keys.empty()) break;
            for (auto& k : keys) {
                int64_t id = get(k.first, k.second);
                if (id >= 0) refine_block(id, &init);
            }
        }
    }

    AmrBlock new_block(int64_t level, const Key3& idx) const {  // amr.rs:346-360
        AmrBlock b;
        b.level = level;
        b.idx = idx;
        b.leaf = true;
        b.u.assign(bcells(), V{});
        b.rhs.assign(bcells(), V{});
        for (int d = 0; d < 3; d++) {
            int64_t fsz = 1;
            for (int e = 0; e < 3; e++)
                if (e != d) fsz *= bd(e);
            b.face[d][0].assign(fsz, V{});
            b.face[d][1].assign(fsz, V{});
        }
        return b;
    }
    void fill_from_init(AmrBlock& b, const InitFn& init) const {
        int64_t b0 = bd(0), b1 = bd(1), b2 = bd(2), n = b0 * b1 * b2;
        std::vector<double> xs(3 * n), ws(N * n);
        for (int64_t i = 0; i < b0; i++)
            for (int64_t j = 0; j < b1; j++)
                for (int64_t k = 0; k < b2; k++) {
                    Key3 g = {b.idx[0] * b0 + i, b.idx[1] * b1 + j, b.idx[2] * b2 + k};
                    x(b.level, g, &xs[3 * ((i * b1 + j) * b2 + k)]);
                }
        init(xs.data(), n, ws.data());
        for (int64_t q = 0; q < n; q++) {
            V w;
            for (int k = 0; k < N; k++) w[k] = ws[N * q + k];
            b.u[q] = sys.to_cons(w);
        }
    }
    void add_block(int64_t level, const Key3& idx, const InitFn& init) {  // amr.rs:362-375
        AmrBlock b = new_block(level, idx);
        fill_from_init(b, init);
        insert(level, idx, blocks.size());
        blocks.push_back(std::move(b));
    }

    Key3 block_key(const Key3& g) const {
        Key3 k;
        for (int d = 0; d < 3; d++) k[d] = active(d) ? div_euclid(g[d], bd(d)) : 0;
        return k;
    }

    // amr.rs:384-439
    V sample(int64_t l, Key3 g) const {
        bool flip[3] = {false, false, false};
        for (int d = 2; d >= 0; d--) {
            if (!active(d)) {
                g[d] = 0;
                continue;
            }
            int64_t n = n_level(l, d);
            if (g[d] < 0 || g[d] >= n) {
                int side = g[d] >= n ? 1 : 0;
                switch (bc[d][side].kind) {
                    case BC_PERIODIC: g[d] = rem_euclid(g[d], n); break;
                    case BC_OUTFLOW: g[d] = std::min(std::max(g[d], int64_t(0)), n - 1); break;
                    case BC_REFLECT:
                        g[d] = side == 0 ? -1 - g[d] : 2 * n - 1 - g[d];
                        flip[d] = true;
                        break;
                    case BC_DIRICHLET: return bc[d][side].state;
                    default: {
                        Key3 gi = g;
                        gi[d] = std::min(std::max(g[d], int64_t(0)), n - 1);
                        Key3 g1 = gi;
                        g1[d] += side == 1 ? -1 : 1;
                        double m = (double)std::llabs(g[d] - gi[d]);
                        V ub = sample(l, gi), ub1 = sample(l, g1);
                        V v = S::char_layer(sys, ub, ub1, bc[d][side].state, d, side, m);
                        for (int e = 0; e < 3; e++)
                            if (flip[e]) v[S::IU + e] = -v[S::IU + e];
                        return v;
                    }
                }
            }
        }
        V v;
        int64_t id = get(l, block_key(g));
        if (id >= 0) {
            int64_t c[3];
            for (int d = 0; d < 3; d++) c[d] = active(d) ? rem_euclid(g[d], bd(d)) : 0;
            v = blocks[id].u[cidx(c[0], c[1], c[2])];
        } else {
            v = predict(l, g);
        }
        for (int d = 0; d < 3; d++)
            if (flip[d]) v[S::IU + d] = -v[S::IU + d];
        return v;
    }

    // amr.rs:450-504
    void bc_box(int64_t l, const Key3& g0, const int64_t* sz, std::vector<V>& val, std::vector<char>& ok) const {
        std::vector<int> dm = dims();
        int64_t n[3];
        for (int d = 0; d < 3; d++) n[d] = n_level(l, d);
        auto at = [&](const Key3& c) -> int64_t {
            for (int d = 0; d < 3; d++)
                if (c[d] < 0 || c[d] >= sz[d]) return -1;
            return (c[0] * sz[1] + c[1]) * sz[2] + c[2];
        };
        auto outside = [&](const Key3& g, int d) {
            return (g[d] < 0 || g[d] >= n[d]) && bc[d][g[d] >= n[d] ? 1 : 0].kind != BC_PERIODIC;
        };
        for (size_t di = 0; di < dm.size(); di++) {
            int d = dm[di];
            for (int64_t i = 0; i < sz[0]; i++)
                for (int64_t j = 0; j < sz[1]; j++)
                    for (int64_t k = 0; k < sz[2]; k++) {
                        Key3 c = {i, j, k};
                        Key3 g = {g0[0] + i, g0[1] + j, g0[2] + k};
                        if (!outside(g, d)) continue;
                        bool later = false;
                        for (size_t e = di + 1; e < dm.size(); e++) later = later || outside(g, dm[e]);
                        if (later) continue;
                        int64_t q = at(c);
                        int side = g[d] >= n[d] ? 1 : 0;
                        auto local = [&](int64_t gg) -> int64_t {
                            Key3 s = c;
                            s[d] = gg - g0[d];
                            int64_t p = at(s);
                            return (p >= 0 && ok[p]) ? p : -1;
                        };
                        int64_t gi = std::min(std::max(g[d], int64_t(0)), n[d] - 1);
                        bool has = false;
                        V v;
                        switch (bc[d][side].kind) {
                            case BC_DIRICHLET:
                                v = bc[d][side].state;
                                has = true;
                                break;
                            case BC_OUTFLOW: {
                                int64_t p = local(gi);
                                if (p >= 0) {
                                    v = val[p];
                                    has = true;
                                }
                                break;
                            }
                            case BC_REFLECT: {
                                int64_t p = local(side == 0 ? -1 - g[d] : 2 * n[d] - 1 - g[d]);
                                if (p >= 0) {
                                    v = val[p];
                                    v[S::IU + d] = -v[S::IU + d];
                                    has = true;
                                }
                                break;
                            }
                            case BC_CHARACTERISTIC: {
                                int64_t g1 = gi + (side == 1 ? -1 : 1);
                                int64_t pb = local(gi), p1 = local(g1);
                                if (pb >= 0 && p1 >= 0) {
                                    v = S::char_layer(sys, val[pb], val[p1], bc[d][side].state, d, side,
                                                                   (double)std::llabs(g[d] - gi));
                                    has = true;
                                }
                                break;
                            }
                            default: break;
                        }
                        if (has) {
                            val[q] = v;
                            ok[q] = 1;
                        }
                    }
        }
    }

    // amr.rs:508-545
    std::vector<V> gather_box(int64_t l, const Key3& g0, const int64_t* sz) const {
        int64_t n[3];
        for (int d = 0; d < 3; d++) n[d] = n_level(l, d);
        std::vector<int> dm = dims();
        int64_t len = sz[0] * sz[1] * sz[2];
        std::vector<V> val(len, V{});
        std::vector<char> ok(len, 1);
        bool any = false;
        for (int64_t i = 0; i < sz[0]; i++)
            for (int64_t j = 0; j < sz[1]; j++)
                for (int64_t k = 0; k < sz[2]; k++) {
                    Key3 g = {g0[0] + i, g0[1] + j, g0[2] + k};
                    int64_t q = (i * sz[1] + j) * sz[2] + k;
                    bool out = false;
                    for (int d : dm)
                        out = out || ((g[d] < 0 || g[d] >= n[d]) && bc[d][g[d] >= n[d] ? 1 : 0].kind != BC_PERIODIC);
                    if (out) {
                        ok[q] = 0;
                        any = true;
                    } else {
                        val[q] = sample(l, g);
                    }
                }
        if (any) {
            bc_box(l, g0, sz, val, ok);
            for (int64_t i = 0; i < sz[0]; i++)
                for (int64_t j = 0; j < sz[1]; j++)
                    for (int64_t k = 0; k < sz[2]; k++) {
                        int64_t q = (i * sz[1] + j) * sz[2] + k;
                        if (!ok[q]) val[q] = sample(l, {g0[0] + i, g0[1] + j, g0[2] + k});
                    }
        }
        return val;
    }

    // amr.rs:548-586
    std::vector<V> predict_box(int64_t l, const Key3& fmin, const Key3& fmax, int64_t* szo) const {
        std::vector<int> dm = dims();
        bool a[3] = {false, false, false};
        for (int d : dm) a[d] = true;
        Key3 cmin, cmax;
        for (int d = 0; d < 3; d++) {
            cmin[d] = a[d] ? div_euclid(fmin[d], 2) - 3 : 0;
            cmax[d] = a[d] ? div_euclid(fmax[d], 2) + 3 : 0;
        }
        int64_t sz[3];
        for (int d = 0; d < 3; d++) sz[d] = cmax[d] - cmin[d] + 1;
        std::vector<V> arr = gather_box(l - 1, cmin, sz);
        for (int d : dm) {
            int64_t nf = fmax[d] - fmin[d] + 1;
            int64_t nsz[3] = {sz[0], sz[1], sz[2]};
            nsz[d] = nf;
            std::vector<V> na(nsz[0] * nsz[1] * nsz[2]);
            for (int64_t i = 0; i < nsz[0]; i++)
                for (int64_t j = 0; j < nsz[1]; j++)
                    for (int64_t k = 0; k < nsz[2]; k++) {
                        int64_t c[3] = {i, j, k};
                        int64_t f = fmin[d] + c[d];
                        int par = (int)rem_euclid(f, 2);
                        int64_t base = div_euclid(f, 2) + (par == 1 ? -2 : -3) - cmin[d];
                        V acc{0, 0, 0, 0, 0};
                        for (int kk = 0; kk < 6; kk++) {
                            int64_t s[3] = {c[0], c[1], c[2]};
                            s[d] = base + kk;
                            const V& v = arr[(s[0] * sz[1] + s[1]) * sz[2] + s[2]];
                            double wgt = wp[par][kk];
                            for (int q = 0; q < N; q++) acc[q] = acc[q] + wgt * v[q];
                        }
                        na[(i * nsz[1] + j) * nsz[2] + k] = acc;
                    }
            arr = std::move(na);
            for (int e = 0; e < 3; e++) sz[e] = nsz[e];
        }
        if (szo)
            for (int e = 0; e < 3; e++) szo[e] = sz[e];
        return arr;
    }

    // amr.rs:589-613 (direct 6^D prediction of one cell)
    V predict(int64_t l, const Key3& g) const {
        std::vector<int> dm = dims();
        V acc{0, 0, 0, 0, 0};
        int64_t total = 1;
        for (size_t i = 0; i < dm.size(); i++) total *= 6;
        for (int64_t s = 0; s < total; s++) {
            double w = 1.0;
            Key3 c = {0, 0, 0};
            int64_t rem = s;
            for (int d : dm) {
                int64_t k = rem % 6;
                rem /= 6;
                int odd = (int)rem_euclid(g[d], 2);
                int64_t base = div_euclid(g[d], 2) + (odd == 1 ? -2 : -3);
                c[d] = base + k;
                w = w * wp[odd][k];
            }
            V v = sample(l - 1, c);
            for (int q = 0; q < N; q++) acc[q] = acc[q] + w * v[q];
        }
        return acc;
    }

    // amr.rs:622-731
    std::vector<V> restrict_box(int64_t l, const Key3& idx, const int64_t* lo_, const int64_t* hi_) const {
        std::vector<int> dm = dims();
        int64_t bd0[3] = {bd(0), bd(1), bd(2)};
        int64_t bdd[3];
        bool a[3] = {false, false, false};
        for (int d : dm) a[d] = true;
        int64_t c0[3], f0[3], sz[3], nf[3];
        for (int d = 0; d < 3; d++) {
            bdd[d] = hi_[d] - lo_[d];
            c0[d] = idx[d] * bd0[d] + lo_[d];
            f0[d] = a[d] ? 2 * c0[d] - 4 : 0;
            sz[d] = a[d] ? 2 * bdd[d] + 8 : 1;
            nf[d] = n_level(l + 1, d);
        }
        std::vector<V> val;
        std::vector<char> ok;
        val.reserve(sz[0] * sz[1] * sz[2]);
        ok.reserve(sz[0] * sz[1] * sz[2]);
        bool any_out = false;
        for (int64_t i = 0; i < sz[0]; i++)
            for (int64_t j = 0; j < sz[1]; j++)
                for (int64_t k = 0; k < sz[2]; k++) {
                    Key3 g = {f0[0] + i, f0[1] + j, f0[2] + k};
                    Key3 gw = g;
                    bool out = false;
                    for (int d = 0; d < 3; d++) {
                        if (a[d] && (g[d] < 0 || g[d] >= nf[d])) {
                            if (bc[d][g[d] >= nf[d] ? 1 : 0].kind == BC_PERIODIC)
                                gw[d] = rem_euclid(g[d], nf[d]);
                            else
                                out = true;
                        }
                    }
                    if (out) {
                        val.push_back(V{});
                        ok.push_back(0);
                        any_out = true;
                    } else {
                        int64_t bid = get(l + 1, block_key(gw));
                        if (bid >= 0) {
                            int64_t c[3];
                            for (int d = 0; d < 3; d++) c[d] = a[d] ? rem_euclid(gw[d], bd0[d]) : 0;
                            val.push_back(blocks[bid].u[cidx(c[0], c[1], c[2])]);
                            ok.push_back(1);
                        } else {
                            val.push_back(V{});
                            ok.push_back(0);
                        }
                    }
                }
        if (any_out) bc_box(l + 1, Key3{f0[0], f0[1], f0[2]}, sz, val, ok);
        const int64_t shifts[5] = {0, -1, 1, -2, 2};
        std::array<std::array<double, 6>, 5> wts;
        for (int m = 0; m < 5; m++) wts[m] = m == 0 ? wr : lagrange6(-2.5 + (double)shifts[m], 0.0);
        for (int d : dm) {
            int64_t nsz[3] = {sz[0], sz[1], sz[2]};
            nsz[d] = bdd[d];
            std::vector<V> nv(nsz[0] * nsz[1] * nsz[2], V{});
            std::vector<char> nok(nsz[0] * nsz[1] * nsz[2], 0);
            for (int64_t i = 0; i < nsz[0]; i++)
                for (int64_t j = 0; j < nsz[1]; j++)
                    for (int64_t k = 0; k < nsz[2]; k++) {
                        int64_t c[3] = {i, j, k};
                        auto at_src = [&](int64_t pos) {
                            int64_t s2[3] = {c[0], c[1], c[2]};
                            s2[d] = pos;
                            return (s2[0] * sz[1] + s2[1]) * sz[2] + s2[2];
                        };
                        int64_t base = 2 * c[d] + 2;
                        bool done = false;
                        int64_t o_ = (i * nsz[1] + j) * nsz[2] + k;
                        for (int m = 0; m < 5; m++) {
                            int64_t st = base + shifts[m];
                            if (st < 0 || st + 5 >= sz[d]) continue;
                            bool all = true;
                            for (int kk = 0; kk < 6; kk++) all = all && ok[at_src(st + kk)];
                            if (all) {
                                V acc{0, 0, 0, 0, 0};
                                for (int kk = 0; kk < 6; kk++) {
                                    const V& v = val[at_src(st + kk)];
                                    for (int q = 0; q < N; q++) acc[q] = acc[q] + wts[m][kk] * v[q];
                                }
                                nv[o_] = acc;
                                nok[o_] = 1;
                                done = true;
                                break;
                            }
                        }
                        if (!done) {
                            int64_t pa = at_src(base + 2), pb = at_src(base + 3);
                            if (ok[pa] && ok[pb]) {
                                V acc;
                                for (int q = 0; q < N; q++) acc[q] = 0.5 * (val[pa][q] + val[pb][q]);
                                nv[o_] = acc;
                                nok[o_] = 1;
                            }
                        }
                    }
            val = std::move(nv);
            ok = std::move(nok);
            for (int e = 0; e < 3; e++) sz[e] = nsz[e];
        }
        return val;
    }

    // neighbour keys at level l with periodic wrap (amr.rs:918-947)
    std::vector<Key3> neighbours(int64_t l, const Key3& idx) const {
        std::vector<Key3> out;
        int64_t nb[3];
        for (int d = 0; d < 3; d++) nb[d] = active(d) ? cfg.base_blocks[d] * (int64_t(1) << l) : 1;
        int r0 = active(0) ? 1 : 0, r1 = active(1) ? 1 : 0, r2 = active(2) ? 1 : 0;
        for (int a = -r0; a <= r0; a++)
            for (int b = -r1; b <= r1; b++)
                for (int c = -r2; c <= r2; c++) {
                    if (a == 0 && b == 0 && c == 0) continue;
                    Key3 k = {idx[0] + a, idx[1] + b, idx[2] + c};
                    bool inside = true;
                    for (int d = 0; d < 3; d++) {
                        if (k[d] < 0 || k[d] >= nb[d]) {
                            if (bc[d][k[d] >= nb[d] ? 1 : 0].kind == BC_PERIODIC)
                                k[d] = rem_euclid(k[d], nb[d]);
                            else
                                inside = false;
                        }
                    }
                    if (inside) out.push_back(k);
                }
        return out;
    }

    bool is_edge_ancestor(int64_t i) const {  // amr.rs:741-744
        const AmrBlock& b = blocks[i];
        if (b.leaf) return false;
        for (auto& nk : neighbours(b.level, b.idx)) {
            int64_t j = get(b.level, nk);
            if (j < 0 || blocks[j].leaf) return true;
        }
        return false;
    }

    // restriction boxes of an edge ancestor (amr.rs:745-787)
    std::vector<std::pair<std::array<int64_t, 3>, std::array<int64_t, 3>>> restrict_boxes(int64_t id) const {
        const AmrBlock& b = blocks[id];
        int64_t l = b.level;
        std::vector<int> dm = dims();
        bool a[3] = {false, false, false};
        for (int d : dm) a[d] = true;
        int64_t bdv[3] = {bd(0), bd(1), bd(2)};
        int64_t nbk[3];
        for (int d = 0; d < 3; d++) nbk[d] = a[d] ? cfg.base_blocks[d] * (int64_t(1) << l) : 1;
        std::vector<std::pair<std::array<int64_t, 3>, std::array<int64_t, 3>>> bx;
        int r0 = a[0] ? 1 : 0, r1 = a[1] ? 1 : 0, r2 = a[2] ? 1 : 0;
        for (int o0 = -r0; o0 <= r0; o0++)
            for (int o1 = -r1; o1 <= r1; o1++)
                for (int o2 = -r2; o2 <= r2; o2++) {
                    int o[3] = {o0, o1, o2};
                    if (o0 == 0 && o1 == 0 && o2 == 0) continue;
                    Key3 nk;
                    bool skip = false;
                    for (int d = 0; d < 3; d++) {
                        nk[d] = b.idx[d] + o[d];
                        if (nk[d] < 0 || nk[d] >= nbk[d]) {
                            if (bc[d][nk[d] >= nbk[d] ? 1 : 0].kind == BC_PERIODIC)
                                nk[d] = rem_euclid(nk[d], nbk[d]);
                            else
                                skip = true;
                        }
                    }
                    if (skip) continue;
                    int64_t j = get(l, nk);
                    if (j >= 0 && !blocks[j].leaf) continue;
                    int64_t w = std::min<int64_t>(ng + 3, std::max(bdv[0], std::max(bdv[1], bdv[2])));
                    std::array<int64_t, 3> lo_, hi_;
                    for (int d = 0; d < 3; d++) {
                        lo_[d] = o[d] == 1 ? std::max<int64_t>(bdv[d] - w, 0) : 0;
                        hi_[d] = o[d] == -1 ? std::min(w, bdv[d]) : bdv[d];
                    }
                    bx.push_back({lo_, hi_});
                }
        int64_t vol = 0;
        for (auto& p : bx) vol += (p.second[0] - p.first[0]) * (p.second[1] - p.first[1]) * (p.second[2] - p.first[2]);
        if (2 * vol > bdv[0] * bdv[1] * bdv[2]) {
            bx.clear();
            bx.push_back({{0, 0, 0}, {bdv[0], bdv[1], bdv[2]}});
        }
        return bx;
    }

    // amr.rs:737-816
    void restrict_all() {
        for (int64_t l = cfg.levels - 2; l >= 0; l--) {
            std::vector<int64_t> ids;
            for (size_t i = 0; i < blocks.size(); i++)
                if (blocks[i].level == l && is_edge_ancestor(i)) ids.push_back(i);
            std::vector<std::vector<std::pair<std::pair<std::array<int64_t, 3>, std::array<int64_t, 3>>, std::vector<V>>>>
                fresh(ids.size());
#pragma omp parallel for schedule(dynamic, 1)
            for (int64_t n = 0; n < (int64_t)ids.size(); n++) {
                for (auto& bx : restrict_boxes(ids[n]))
                    fresh[n].push_back({bx, restrict_box(l, blocks[ids[n]].idx, bx.first.data(), bx.second.data())});
            }
            for (size_t n = 0; n < ids.size(); n++)
                for (auto& part : fresh[n]) {
                    auto& lo_ = part.first.first;
                    auto& hi_ = part.first.second;
                    size_t it = 0;
                    for (int64_t i = lo_[0]; i < hi_[0]; i++)
                        for (int64_t j = lo_[1]; j < hi_[1]; j++)
                            for (int64_t k = lo_[2]; k < hi_[2]; k++) blocks[ids[n]].u[cidx(i, j, k)] = part.second[it++];
                }
        }
    }

    // amr.rs:1113-1221
    std::vector<V> fill_scratch(int64_t id) const {
        const AmrBlock& b = blocks[id];
        int64_t l = b.level;
        bool a[3];
        int64_t bdv[3], ext[3], gof[3];
        for (int d = 0; d < 3; d++) {
            a[d] = active(d);
            bdv[d] = bd(d);
            ext[d] = a[d] ? bdv[d] + 2 * ng : 1;
            gof[d] = a[d] ? ng : 0;
        }
        auto at = [&](int64_t i, int64_t j, int64_t k) { return (i * ext[1] + j) * ext[2] + k; };
        std::vector<V> out(ext[0] * ext[1] * ext[2], V{});
        std::vector<char> filled(out.size(), 1);
        for (int64_t i = 0; i < bdv[0]; i++)
            for (int64_t j = 0; j < bdv[1]; j++)
                for (int64_t k = 0; k < bdv[2]; k++) out[at(i + gof[0], j + gof[1], k + gof[2])] = b.u[cidx(i, j, k)];
        int64_t nbk[3];
        for (int d = 0; d < 3; d++) nbk[d] = a[d] ? cfg.base_blocks[d] * (int64_t(1) << l) : 1;
        auto rng = [&](int o, int d, int64_t& s, int64_t& e) {
            if (!a[d]) {
                s = 0;
                e = 1;
            } else if (o == -1) {
                s = 0;
                e = ng;
            } else if (o == 0) {
                s = ng;
                e = ng + bdv[d];
            } else {
                s = ng + bdv[d];
                e = 2 * ng + bdv[d];
            }
        };
        int r0 = a[0] ? 1 : 0, r1 = a[1] ? 1 : 0, r2 = a[2] ? 1 : 0;
        for (int o0 = -r0; o0 <= r0; o0++)
            for (int o1 = -r1; o1 <= r1; o1++)
                for (int o2 = -r2; o2 <= r2; o2++) {
                    int o[3] = {o0, o1, o2};
                    if (o0 == 0 && o1 == 0 && o2 == 0) continue;
                    int64_t rs[3], re[3];
                    for (int d = 0; d < 3; d++) rng(o[d], d, rs[d], re[d]);
                    auto gl = [&](int64_t c0, int64_t c1, int64_t c2) {
                        int64_t c[3] = {c0, c1, c2};
                        Key3 g;
                        for (int d = 0; d < 3; d++) g[d] = b.idx[d] * bdv[d] + c[d] - gof[d];
                        return g;
                    };
                    Key3 nk;
                    bool inside = true;
                    for (int d = 0; d < 3; d++) {
                        nk[d] = b.idx[d] + o[d];
                        if (nk[d] < 0 || nk[d] >= nbk[d]) {
                            if (bc[d][nk[d] >= nbk[d] ? 1 : 0].kind == BC_PERIODIC)
                                nk[d] = rem_euclid(nk[d], nbk[d]);
                            else
                                inside = false;
                        }
                    }
                    if (!inside) {
                        for (int64_t i = rs[0]; i < re[0]; i++)
                            for (int64_t j = rs[1]; j < re[1]; j++)
                                for (int64_t k = rs[2]; k < re[2]; k++) filled[at(i, j, k)] = 0;
                        continue;
                    }
                    int64_t nid = get(l, nk);
                    if (nid >= 0) {
                        const AmrBlock& nb = blocks[nid];
                        for (int64_t i = rs[0]; i < re[0]; i++)
                            for (int64_t j = rs[1]; j < re[1]; j++)
                                for (int64_t k = rs[2]; k < re[2]; k++) {
                                    int64_t c[3] = {i, j, k}, lc[3];
                                    for (int d = 0; d < 3; d++) lc[d] = a[d] ? c[d] - gof[d] - o[d] * bdv[d] : 0;
                                    out[at(i, j, k)] = nb.u[cidx(lc[0], lc[1], lc[2])];
                                }
                        continue;
                    }
                    Key3 fmin = gl(rs[0], rs[1], rs[2]);
                    Key3 fmax = gl(re[0] - 1, re[1] - 1, re[2] - 1);
                    int64_t sz[3];
                    std::vector<V> arr = predict_box(l, fmin, fmax, sz);
                    for (int64_t i = rs[0]; i < re[0]; i++)
                        for (int64_t j = rs[1]; j < re[1]; j++)
                            for (int64_t k = rs[2]; k < re[2]; k++) {
                                Key3 g = gl(i, j, k);
                                int64_t li[3];
                                for (int d = 0; d < 3; d++) li[d] = a[d] ? g[d] - fmin[d] : 0;
                                out[at(i, j, k)] = arr[(li[0] * sz[1] + li[1]) * sz[2] + li[2]];
                            }
                }
        bool anyf = false;
        for (char f : filled) anyf = anyf || !f;
        if (anyf) {
            Key3 g0;
            for (int d = 0; d < 3; d++) g0[d] = b.idx[d] * bdv[d] - gof[d];
            bc_box(l, g0, ext, out, filled);
            for (int64_t i = 0; i < ext[0]; i++)
                for (int64_t j = 0; j < ext[1]; j++)
                    for (int64_t k = 0; k < ext[2]; k++)
                        if (!filled[at(i, j, k)]) out[at(i, j, k)] = sample(l, {g0[0] + i, g0[1] + j, g0[2] + k});
        }
        return out;
    }

    // amr.rs:823-867
    double block_detail(int64_t id) const {
        std::vector<int> dm = dims();
        bool a[3];
        int64_t bdv[3], ext[3], gof[3];
        for (int d = 0; d < 3; d++) {
            a[d] = active(d);
            bdv[d] = bd(d);
            ext[d] = a[d] ? bdv[d] + 2 * ng : 1;
            gof[d] = a[d] ? ng : 0;
        }
        std::vector<V> scr = fill_scratch(id);
        std::vector<std::array<double, 3>> sens(scr.size());
        int ns = 0;
        for (size_t q = 0; q < scr.size(); q++) {
            double v[8];
            ns = sys.sensor(sys.to_prim(scr[q]), v);
            sens[q] = {v[0], v[1], ns > 2 ? v[2] : 0.0};
        }
        auto at = [&](const int64_t* c) { return (c[0] * ext[1] + c[1]) * ext[2] + c[2]; };
        double mx = 0.0;
        const int64_t offs[6] = {-5, -3, -1, 1, 3, 5};
        for (int64_t i = 0; i < bdv[0]; i++)
            for (int64_t j = 0; j < bdv[1]; j++)
                for (int64_t k = 0; k < bdv[2]; k++) {
                    int64_t c[3] = {i + gof[0], j + gof[1], k + gof[2]};
                    const auto& s0 = sens[at(c)];
                    for (int d : dm) {
                        double pred[3] = {0.0, 0.0, 0.0};
                        for (int m = 0; m < 6; m++) {
                            int64_t cc[3] = {c[0], c[1], c[2]};
                            cc[d] += offs[m];
                            const auto& sv = sens[at(cc)];
                            for (int q = 0; q < ns; q++) pred[q] = pred[q] + wr[m] * sv[q];
                        }
                        for (int q = 0; q < ns; q++) {
                            double dd = std::fabs(s0[q] - pred[q]);
                            mx = std::isfinite(dd) ? std::fmax(mx, dd) : INFINITY;
                        }
                    }
                }
        return mx;
    }

    std::vector<double> details() const {
        std::vector<double> det(blocks.size(), 0.0);
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t i = 0; i < (int64_t)blocks.size(); i++)
            if (blocks[i].leaf) det[i] = block_detail(i);
        return det;
    }
    std::vector<int8_t> flags() const { return flags_from_details(details()); }

    // amr.rs:877-892
    std::vector<int8_t> flags_from_details(const std::vector<double>& det) const {
        std::vector<int8_t> f(blocks.size(), 0);
        for (size_t i = 0; i < blocks.size(); i++) {
            const AmrBlock& b = blocks[i];
            if (!b.leaf)
                f[i] = 0;
            else if (det[i] > cfg.eps && b.level + 1 < cfg.levels)
                f[i] = 1;
            else if (det[i] < cfg.eps / 128.0)
                f[i] = -1;
            else
                f[i] = 0;
        }
        return f;
    }

    // amr.rs:894-915
    std::vector<Key3> children(const Key3& idx) const {
        std::vector<Key3> out = {Key3{0, 0, 0}};
        for (int d = 0; d < 3; d++) {
            std::vector<Key3> next;
            for (auto& c : out) {
                if (active(d)) {
                    for (int o = 0; o < 2; o++) {
                        Key3 cc = c;
                        cc[d] = 2 * idx[d] + o;
                        next.push_back(cc);
                    }
                } else {
                    Key3 cc = c;
                    cc[d] = 0;
                    next.push_back(cc);
                }
            }
            out = next;
        }
        return out;
    }

    // amr.rs:952-1011
    void refine_block(int64_t id, const InitFn* init) {
        int64_t l = blocks[id].level;
        Key3 idx = blocks[id].idx;
        if (!blocks[id].leaf) return;
        if (l > 0) {
            for (auto& nk : neighbours(l, idx)) {
                if (get(l, nk) < 0) {
                    for (int64_t m = l - 1; m >= 0; m--) {
                        Key3 pk;
                        for (int d = 0; d < 3; d++) pk[d] = active(d) ? nk[d] >> (l - m) : 0;
                        int64_t pid = get(m, pk);
                        if (pid >= 0) {
                            refine_block(pid, init);
                            break;
                        }
                    }
                }
            }
        }
        id = get(l, idx);
        if (id < 0 || !blocks[id].leaf) return;
        std::vector<Key3> kids = children(idx);
        int64_t bdv[3] = {bd(0), bd(1), bd(2)};
        std::vector<AmrBlock> newb(kids.size());
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t n = 0; n < (int64_t)kids.size(); n++) {
            const Key3& c = kids[n];
            AmrBlock b = new_block(l + 1, c);
            if (init) {
                fill_from_init(b, *init);
            } else {
                Key3 fmin, fmax;
                for (int d = 0; d < 3; d++) {
                    fmin[d] = c[d] * bdv[d];
                    fmax[d] = c[d] * bdv[d] + bdv[d] - 1;
                }
                b.u = predict_box(l + 1, fmin, fmax, nullptr);
            }
            newb[n] = std::move(b);
        }
        blocks[id].leaf = false;
        for (auto& b : newb) {
            insert(b.level, b.idx, blocks.size());
            blocks.push_back(std::move(b));
        }
    }

    // amr.rs:1014-1032
    void coarsen(int64_t l, const Key3& idx) {
        std::vector<Key3> kids = children(idx);
        int64_t pid = get(l, idx);
        int64_t lo0[3] = {0, 0, 0}, hi0[3] = {bd(0), bd(1), bd(2)};
        blocks[pid].u = restrict_box(l, idx, lo0, hi0);
        blocks[pid].leaf = true;
        std::vector<int64_t> ids;
        for (auto& c : kids) ids.push_back(get(l + 1, c));
        std::sort(ids.begin(), ids.end(), [](int64_t x, int64_t y) { return x > y; });
        for (int64_t i : ids) {
            remove(blocks[i].level, blocks[i].idx);
            std::swap(blocks[i], blocks.back());
            blocks.pop_back();
            if (i < (int64_t)blocks.size()) insert(blocks[i].level, blocks[i].idx, i);
        }
    }

    void regrid() {  // amr.rs:1039-1046
        restrict_all();
        std::vector<int8_t> f = flags();
        auto prot = regrid_refine(f);
        restrict_all();
        f = flags();
        regrid_coarsen(f, prot);
    }

    // amr.rs:1051-1076
    std::set<std::pair<int64_t, Key3>> regrid_refine(const std::vector<int8_t>& f) {
        std::vector<std::pair<int64_t, Key3>> want;
        for (size_t i = 0; i < f.size(); i++) {
            if (f[i] > 0) {
                const AmrBlock& b = blocks[i];
                want.push_back({b.level, b.idx});
                for (auto& nk : neighbours(b.level, b.idx)) {
                    int64_t j = get(b.level, nk);
                    if (j >= 0 && blocks[j].leaf) want.push_back({b.level, nk});
                }
            }
        }
        std::sort(want.begin(), want.end());
        want.erase(std::unique(want.begin(), want.end()), want.end());
        std::set<std::pair<int64_t, Key3>> prot(want.begin(), want.end());
        for (auto& k : want) {
            int64_t id = get(k.first, k.second);
            if (id >= 0 && k.first + 1 < cfg.levels) refine_block(id, nullptr);
        }
        return prot;
    }

    // amr.rs:1080-1106
    void regrid_coarsen(const std::vector<int8_t>& f, const std::set<std::pair<int64_t, Key3>>& prot) {
        size_t nkids = size_t(1) << dims().size();
        std::vector<std::pair<int64_t, Key3>> cand;
        for (size_t bi = 0; bi < blocks.size(); bi++) {
            const AmrBlock& b = blocks[bi];
            if (b.leaf) continue;
            std::vector<Key3> kids = children(b.idx);
            bool ok = kids.size() == nkids;
            for (auto& c : kids) {
                if (!ok) break;
                int64_t j = get(b.level + 1, c);
                ok = j >= 0 && blocks[j].leaf && f[j] < 0 && !prot.count({b.level + 1, c});
            }
            if (ok) cand.push_back({b.level, b.idx});
        }
        std::stable_sort(cand.begin(), cand.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
        for (auto& c : cand) {
            int64_t l = c.first;
            bool ok = true;
            for (auto& nk : neighbours(l, c.second)) {
                for (auto& ch : children(nk)) {
                    int64_t j = get(l + 1, ch);
                    if (j >= 0 && !blocks[j].leaf) ok = false;
                }
            }
            if (ok && get(l, c.second) >= 0) coarsen(l, c.second);
        }
    }

    // amr.rs:1224-1299: rhs and boundary face fluxes of leaf id
    Stats block_rhs(int64_t id, std::vector<V>& rhs, std::vector<V> (&face)[3][2]) const {
        std::vector<int> dm = dims();
        bool a[3];
        int64_t bdv[3], ext[3], gof[3];
        for (int d = 0; d < 3; d++) {
            a[d] = active(d);
            bdv[d] = bd(d);
            ext[d] = a[d] ? bdv[d] + 2 * ng : 1;
            gof[d] = a[d] ? ng : 0;
        }
        double ndim = (double)dm.size();
        const AmrBlock& b = blocks[id];
        int64_t l = b.level;
        std::vector<V> scr = fill_scratch(id);
        std::vector<V> w(scr.size());
        for (size_t q = 0; q < scr.size(); q++) w[q] = sys.to_prim(scr[q]);
        rhs.assign(bcells(), V{});
        Stats st;
        for (int d : dm) {
            int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            double dxl = dx(l, d);
            SchemeOpts opts{mode, tol, positivity ? ndim * stage_dt / dxl : 0.0};
            std::vector<V> fl(bdv[d] + 1), line(ext[d]);
            std::vector<double> uf(bdv[d] + 1, 0.0);
            face[d][0].clear();
            face[d][1].clear();
            for (int64_t aa = 0; aa < bdv[e0]; aa++)
                for (int64_t bb = 0; bb < bdv[e1]; bb++) {
                    auto at = [&](int64_t cc) {
                        int64_t c[3];
                        c[d] = cc;
                        c[e0] = aa + gof[e0];
                        c[e1] = bb + gof[e1];
                        return (c[0] * ext[1] + c[1]) * ext[2] + c[2];
                    };
                    for (int64_t cc = 0; cc < ext[d]; cc++) line[cc] = w[at(cc)];
                    S::fluxes(sys, line.data(), (int)ext[d], d, (int)ng, opts, fl.data(), uf.data(), st);
                    for (int64_t cc = 0; cc < bdv[d]; cc++) {
                        int64_t c[3];
                        c[d] = cc;
                        c[e0] = aa;
                        c[e1] = bb;
                        V& o = rhs[cidx(c[0], c[1], c[2])];
                        for (int q = 0; q < N; q++) o[q] = o[q] - (fl[cc + 1][q] - fl[cc][q]) / dxl;
                        if constexpr (S::MULTIPHASE) {
                            // the α equation's non-conservative term (amr.rs:1276-1279)
                            const V& wc = line[cc + ng];
                            o[N - 1] = o[N - 1] + sys.nc_coef(wc) * (uf[cc + 1] - uf[cc]) / dxl;
                        }
                    }
                    face[d][0].push_back(fl[0]);
                    face[d][1].push_back(fl[bdv[d]]);
                }
        }
        return st;
    }

    std::vector<int64_t> leaves() const {
        std::vector<int64_t> v;
        for (size_t i = 0; i < blocks.size(); i++)
            if (blocks[i].leaf) v.push_back(i);
        return v;
    }

    // amr.rs:1302-1323
    Stats compute_rhs() {
        restrict_all();
        std::vector<int64_t> lv = leaves();
        std::vector<Stats> st(lv.size());
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t n = 0; n < (int64_t)lv.size(); n++) {
            std::vector<V> rhs;
            std::vector<V> face[3][2];
            st[n] = block_rhs(lv[n], rhs, face);
            AmrBlock& b = blocks[lv[n]];
            b.rhs = std::move(rhs);
            for (int d = 0; d < 3; d++)
                for (int s = 0; s < 2; s++)
                    if (active(d)) b.face[d][s] = std::move(face[d][s]);
        }
        Stats total;
        for (auto& s : st) total.add(s);
        reflux();
        return total;
    }

    // amr.rs:1327-1406
    void reflux() {
        std::vector<int> dm = dims();
        int64_t bdv[3] = {bd(0), bd(1), bd(2)};
        std::vector<std::tuple<int64_t, int64_t, V>> corr;
        for (size_t id = 0; id < blocks.size(); id++) {
            const AmrBlock& b = blocks[id];
            int64_t l = b.level;
            if (!b.leaf || l + 1 >= cfg.levels) continue;
            for (int d : dm) {
                int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
                double dxl = dx(l, d);
                int64_t nbk = cfg.base_blocks[d] * (int64_t(1) << l);
                bool a0 = active(e0), a1 = active(e1);
                for (int side = 0; side < 2; side++) {
                    Key3 nk = b.idx;
                    nk[d] += side == 1 ? 1 : -1;
                    if (nk[d] < 0 || nk[d] >= nbk) {
                        if (bc[d][side].kind != BC_PERIODIC) continue;
                        nk[d] = rem_euclid(nk[d], nbk);
                    }
                    int64_t nj = get(l, nk);
                    if (!(nj >= 0 && !blocks[nj].leaf)) continue;
                    for (int64_t aa = 0; aa < bdv[e0]; aa++)
                        for (int64_t bb = 0; bb < bdv[e1]; bb++) {
                            V sum{0, 0, 0, 0, 0};
                            double cnt = 0.0;
                            for (int64_t fa = 0; fa < (a0 ? 2 : 1); fa++)
                                for (int64_t fb = 0; fb < (a1 ? 2 : 1); fb++) {
                                    int64_t ga = 2 * (b.idx[e0] * bdv[e0] + aa) + fa;
                                    int64_t gb = 2 * (b.idx[e1] * bdv[e1] + bb) + fb;
                                    Key3 ck = nk;
                                    ck[d] = 2 * nk[d] + (side == 1 ? 0 : 1);
                                    ck[e0] = a0 ? div_euclid(ga, bdv[e0]) : 0;
                                    ck[e1] = a1 ? div_euclid(gb, bdv[e1]) : 0;
                                    int64_t cid = get(l + 1, ck);
                                    if (cid < 0 || !blocks[cid].leaf) continue;
                                    int64_t la = a0 ? rem_euclid(ga, bdv[e0]) : 0;
                                    int64_t lb = a1 ? rem_euclid(gb, bdv[e1]) : 0;
                                    const V& fv = blocks[cid].face[d][1 - side][la * bdv[e1] + lb];
                                    for (int q = 0; q < N; q++) sum[q] = sum[q] + fv[q];
                                    cnt = cnt + 1.0;
                                }
                            if (cnt == 0.0) continue;
                            const V& fc = b.face[d][side][aa * bdv[e1] + bb];
                            int64_t c[3];
                            c[d] = side == 1 ? bdv[d] - 1 : 0;
                            c[e0] = aa;
                            c[e1] = bb;
                            V dr;
                            for (int q = 0; q < N; q++) {
                                double df = sum[q] / cnt - fc[q];
                                dr[q] = side == 1 ? -df / dxl : df / dxl;
                            }
                            corr.push_back({(int64_t)id, cidx(c[0], c[1], c[2]), dr});
                        }
                }
            }
        }
        for (auto& c : corr) {
            V& r = blocks[std::get<0>(c)].rhs[std::get<1>(c)];
            for (int q = 0; q < N; q++) r[q] = r[q] + std::get<2>(c)[q];
        }
    }

    // amr.rs:1409-1467 (Euler: no dilatation term)
    double cfl_rate() const {
        std::vector<int> dm = dims();
        double rate = 0.0;
        for (size_t bi = 0; bi < blocks.size(); bi++) {
            const AmrBlock& b = blocks[bi];
            if (!b.leaf) continue;
            double r = 0.0;
            for (const V& u : b.u) {
                V w = sys.to_prim(u);
                double s = -0.0;
                for (int d : dm) s = s + sys.max_speed(w, d) / dx(b.level, d);
                r = std::fmax(r, s);
            }
            rate = std::fmax(rate, r);
        }
        return rate;
    }
    // amr.rs:1408-1466: the global step, and for the multiphase system the
    // dilatation limit 0.5 / max rate over the leaves, with the velocity
    // divergence from the neighbouring cells (sampled across block faces)
    double dt_cfl() const {
        double dt = cfl / cfl_rate();
        if constexpr (S::MULTIPHASE) {
            std::vector<int> dm = dims();
            int64_t bdv[3] = {bd(0), bd(1), bd(2)};
            std::vector<double> src(blocks.size(), 0.0);
#pragma omp parallel for schedule(dynamic, 1)
            for (int64_t bi = 0; bi < (int64_t)blocks.size(); bi++) {
                const AmrBlock& b = blocks[bi];
                if (!b.leaf) continue;
                double r = 0.0;
                for (int64_t i = 0; i < bdv[0]; i++)
                    for (int64_t j = 0; j < bdv[1]; j++)
                        for (int64_t k = 0; k < bdv[2]; k++) {
                            int64_t c[3] = {i, j, k};
                            V w = sys.to_prim(b.u[cidx(i, j, k)]);
                            double divu = 0.0;
                            for (int d : dm) {
                                auto get = [&](int64_t o) {
                                    int64_t cc[3] = {c[0], c[1], c[2]};
                                    cc[d] += o;
                                    if (cc[d] >= 0 && cc[d] < bdv[d]) return sys.to_prim(b.u[cidx(cc[0], cc[1], cc[2])]);
                                    Key3 g;
                                    for (int e = 0; e < 3; e++) g[e] = b.idx[e] * bdv[e] + cc[e];
                                    return sys.to_prim(sample(b.level, g));
                                };
                                int vi = S::IU + d;
                                divu = divu + std::fabs(get(1)[vi] - get(-1)[vi]) / (2.0 * dx(b.level, d));
                            }
                            r = std::fmax(r, sys.dilatation_rate(w, divu));
                        }
                src[bi] = r;
            }
            double s = 0.0;
            for (double v : src) s = std::fmax(s, v);
            if (s > 0.0) dt = std::fmin(dt, 0.5 / s);
        }
        return dt;
    }

    // amr.rs:1470-1512
    void step(double dt) {
        stage_dt = dt;
        for (auto& b : blocks)
            if (b.leaf) b.u0 = b.u;
        Stats s1 = compute_rhs();
        for (auto& b : blocks)
            if (b.leaf)
                for (size_t c = 0; c < b.u.size(); c++)
                    for (int q = 0; q < N; q++) b.u[c][q] = b.u[c][q] + dt * b.rhs[c][q];
        Stats s2 = compute_rhs();
        for (auto& b : blocks)
            if (b.leaf)
                for (size_t c = 0; c < b.u.size(); c++)
                    for (int q = 0; q < N; q++) b.u[c][q] = 0.75 * b.u0[c][q] + 0.25 * (b.u[c][q] + dt * b.rhs[c][q]);
        Stats s3 = compute_rhs();
        for (auto& b : blocks)
            if (b.leaf)
                for (size_t c = 0; c < b.u.size(); c++)
                    for (int q = 0; q < N; q++)
                        b.u[c][q] = b.u0[c][q] / 3.0 + 2.0 / 3.0 * (b.u[c][q] + dt * b.rhs[c][q]);
        stats.add(s1);
        stats.add(s2);
        stats.add(s3);
        t += dt;  // advance_clock, amr.rs:1515-1518
        steps += 1;
        regrid_if_due();
    }

    // amr.rs:1521-1550
    bool regrid_if_due() {
        if (steps < next_regrid) return false;
        auto before = structure();
        regrid();
        bool changed = structure() != before;
        schedule_regrid(changed);
        return changed;
    }
    std::vector<std::tuple<int64_t, Key3, bool>> structure() const {
        std::vector<std::tuple<int64_t, Key3, bool>> s;
        for (auto& b : blocks) s.push_back({b.level, b.idx, b.leaf});
        return s;
    }
    void schedule_regrid(bool changed) {
        regrid_interval = changed ? cfg.regrid_every : std::min(2 * regrid_interval, 2 * cfg.regrid_every);
        next_regrid = steps + regrid_interval;
    }

    // amr.rs:1639-1652
    int64_t run_to(double t_end) {
        int64_t n = 0;
        while (t < t_end * (1.0 - 1e-14)) {
            double dt = std::fmin(subcycle ? dt_cfl_subcycled() : dt_cfl(), t_end - t);
            if (!(std::isfinite(dt) && dt > 0.0)) return -1;
            if (subcycle)
                step_subcycled(dt);
            else
                step(dt);
            n += 1;
        }
        return n;
    }

    // ---------------------------------------------------------------- subcycling

    // amr.rs:1657-1679: CFL step of the level-l blocks, leaves and ancestors
    double dt_cfl_level(int64_t l) const {
        std::vector<int> dm = dims();
        double rate = 0.0;
        for (const AmrBlock& b : blocks) {
            if (b.level != l) continue;
            double r = 0.0;
            for (const V& u : b.u) {
                V w = sys.to_prim(u);
                double sp = -0.0;
                for (int d : dm) sp = sp + sys.max_speed(w, d) / dx(l, d);
                r = std::fmax(r, sp);
            }
            rate = std::fmax(rate, r);
        }
        return rate > 0.0 ? cfl / rate : INFINITY;
    }

    // amr.rs:1681-1692: level-lmin step such that level l takes dt/2^(l-lmin)
    double dt_cfl_subcycled() const {
        int64_t lmin = coarsest_leaf_level();
        double dt = INFINITY;
        for (int64_t l = lmin; l < cfg.levels; l++) dt = std::fmin(dt, dt_cfl_level(l) * (double)(uint64_t(1) << (l - lmin)));
        double g = dt_cfl();
        int64_t finest = 0;
        for (int64_t l = cfg.levels - 1; l >= 0; l--) {
            bool any = false;
            for (const AmrBlock& b : blocks) any = any || (b.level == l && b.leaf);
            if (any) {
                finest = l;
                break;
            }
        }
        return std::fmin(dt, g * (double)(uint64_t(1) << (finest - lmin)));
    }

    // amr.rs:1694-1700
    int64_t coarsest_leaf_level() const {
        int64_t m = -1;
        for (const AmrBlock& b : blocks)
            if (b.leaf && (m < 0 || b.level < m)) m = b.level;
        return m < 0 ? 0 : m;
    }

    // amr.rs:1702-1723: level-l data linearly interpolated in time (saved, then restored)
    void set_time_view(int64_t l, double tv) {
        double t0 = level_t0[l], dt = level_dt[l];
        double th = 1.0;
        if (dt > 0.0) {
            th = (tv - t0) / dt;
            if (th < 0.0) th = 0.0;
            if (th > 1.0) th = 1.0;
        }
        for (AmrBlock& b : blocks) {
            if (b.level != l || b.u0.empty()) continue;
            b.u_save = b.u;
            for (size_t c = 0; c < b.u.size(); c++)
                for (int q = 0; q < N; q++) b.u[c][q] = (1.0 - th) * b.u0[c][q] + th * b.u[c][q];
        }
    }
    void restore_time_view(int64_t l) {
        for (AmrBlock& b : blocks)
            if (b.level == l && !b.u_save.empty()) std::swap(b.u, b.u_save);
    }

    // amr.rs:1725-1760: coarse–fine faces of block id: (d, side, kind, coarse
    // block) with kind 0 = the neighbour is refined, 1 = the neighbour is coarser
    struct CfFace {
        int d, side, kind;
        int64_t coarse;
    };
    std::vector<CfFace> cf_faces(int64_t id) const {
        const AmrBlock& b = blocks[id];
        int64_t l = b.level;
        std::vector<int> dm = dims();
        std::vector<CfFace> out;
        for (int d : dm) {
            int64_t nbk = cfg.base_blocks[d] * (int64_t(1) << l);
            for (int side = 0; side < 2; side++) {
                Key3 nk = b.idx;
                nk[d] += side == 1 ? 1 : -1;
                if (nk[d] < 0 || nk[d] >= nbk) {
                    if (bc[d][side].kind != BC_PERIODIC) continue;
                    nk[d] = rem_euclid(nk[d], nbk);
                }
                int64_t j = get(l, nk);
                if (j >= 0) {
                    if (!blocks[j].leaf) out.push_back({d, side, 0, -1});
                } else if (l > 0) {
                    Key3 pk;
                    for (int e = 0; e < 3; e++) pk[e] = active(e) ? (nk[e] >> 1) : 0;
                    int64_t cj = get(l - 1, pk);
                    if (cj >= 0) out.push_back({d, side, 1, cj});
                }
            }
        }
        return out;
    }

    // amr.rs:1762-1807: add the stage's boundary fluxes (weight wdt) to the registers
    void accumulate_registers(const std::vector<int64_t>& ids, double wdt) {
        std::vector<int> dm = dims();
        int64_t bdv[3] = {bd(0), bd(1), bd(2)};
        double nsub = (double)(size_t(1) << (dm.size() - 1));
        for (int64_t id : ids) {
            if (!blocks[id].leaf) continue;
            for (const CfFace& cf : cf_faces(id)) {
                int d = cf.d;
                int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
                const std::vector<V>& face = blocks[id].face[d][cf.side];
                if (cf.kind == 0) {
                    for (size_t fi = 0; fi < face.size(); fi++) {
                        V& e = creg.try_emplace(RegKey{id, d, cf.side, (int64_t)fi}, V{}).first->second;
                        for (int q = 0; q < N; q++) e[q] = e[q] + wdt * face[fi][q];
                    }
                } else {
                    const AmrBlock& b = blocks[id];
                    const AmrBlock& cb = blocks[cf.coarse];
                    for (int64_t a = 0; a < bdv[e0]; a++)
                        for (int64_t bb = 0; bb < bdv[e1]; bb++) {
                            int64_t ga = b.idx[e0] * bdv[e0] + a;
                            int64_t gb = b.idx[e1] * bdv[e1] + bb;
                            int64_t ca = active(e0) ? div_euclid(ga, 2) - cb.idx[e0] * bdv[e0] : 0;
                            int64_t cbb = active(e1) ? div_euclid(gb, 2) - cb.idx[e1] * bdv[e1] : 0;
                            if (ca >= bdv[e0] || cbb >= bdv[e1]) continue;
                            const V& f = face[a * bdv[e1] + bb];
                            V& e = freg.try_emplace(RegKey{cf.coarse, d, 1 - cf.side, ca * bdv[e1] + cbb}, V{})
                                       .first->second;
                            for (int q = 0; q < N; q++) e[q] = e[q] + wdt * f[q] / nsub;
                        }
                }
            }
        }
    }

    // amr.rs:1809-1834: correct the coarse leaves of level l with the registers.
    // Order: by direction, then side, then block and face index (a cell on two
    // coarse–fine faces takes the correction of the lower direction first).
    void reflux_level(int64_t l) {
        int64_t bdv[3] = {bd(0), bd(1), bd(2)};
        std::vector<RegKey> keys;
        for (auto& kv : creg)
            if (blocks[std::get<0>(kv.first)].level == l) keys.push_back(kv.first);
        std::sort(keys.begin(), keys.end(), [](const RegKey& x, const RegKey& y) {
            return std::make_tuple(std::get<1>(x), std::get<2>(x), std::get<0>(x), std::get<3>(x)) <
                   std::make_tuple(std::get<1>(y), std::get<2>(y), std::get<0>(y), std::get<3>(y));
        });
        for (const RegKey& key : keys) {
            auto fr = freg.find(key);
            if (fr == freg.end()) continue;
            const V& cr = creg[key];
            int64_t id = std::get<0>(key), fi = std::get<3>(key);
            int d = std::get<1>(key), side = std::get<2>(key);
            int e0 = d == 0 ? 1 : 0, e1 = d == 2 ? 1 : 2;
            int64_t c[3];
            c[d] = side == 1 ? bdv[d] - 1 : 0;
            c[e0] = fi / bdv[e1];
            c[e1] = fi % bdv[e1];
            double dxl = dx(l, d);
            V& u = blocks[id].u[cidx(c[0], c[1], c[2])];
            for (int q = 0; q < N; q++) {
                double df = fr->second[q] - cr[q];
                u[q] = u[q] + (side == 1 ? -df / dxl : df / dxl);
            }
        }
    }

    // amr.rs:1836-1900: advance every level-l block (leaves and ancestors) by
    // dt, then level l+1 twice by dt/2, then reflux and restrict
    void advance_level(int64_t l, double dt) {
        std::vector<int64_t> ids;
        for (size_t i = 0; i < blocks.size(); i++)
            if (blocks[i].level == l) ids.push_back(i);
        if (ids.empty()) return;
        double t0 = level_t0[l];
        level_dt[l] = dt;
        for (int64_t id : ids) blocks[id].u0 = blocks[id].u;
        for (auto it = creg.begin(); it != creg.end();)
            it = blocks[std::get<0>(it->first)].level == l ? creg.erase(it) : std::next(it);
        for (auto it = freg.begin(); it != freg.end();)
            it = blocks[std::get<0>(it->first)].level == l ? freg.erase(it) : std::next(it);
        stage_dt = dt;
        double stage_t[3] = {t0, t0 + dt, t0 + 0.5 * dt};
        double weights[3] = {1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0};
        double a0s[3] = {0.0, 0.75, 1.0 / 3.0}, a1s[3] = {1.0, 0.25, 2.0 / 3.0};
        for (int s = 0; s < 3; s++) {
            if (l > 0) set_time_view(l - 1, stage_t[s]);
            std::vector<std::vector<V>> rhs(ids.size());
            std::vector<std::array<std::array<std::vector<V>, 2>, 3>> faces(ids.size());
            std::vector<Stats> st(ids.size());
#pragma omp parallel for schedule(dynamic, 1)
            for (int64_t n = 0; n < (int64_t)ids.size(); n++) {
                std::vector<V> face[3][2];
                st[n] = block_rhs(ids[n], rhs[n], face);
                for (int d = 0; d < 3; d++)
                    for (int sd = 0; sd < 2; sd++) faces[n][d][sd] = std::move(face[d][sd]);
            }
            if (l > 0) restore_time_view(l - 1);
            for (size_t n = 0; n < ids.size(); n++) {
                AmrBlock& b = blocks[ids[n]];
                b.rhs = std::move(rhs[n]);
                for (int d = 0; d < 3; d++)
                    for (int sd = 0; sd < 2; sd++) b.face[d][sd] = std::move(faces[n][d][sd]);
                stats.add(st[n]);
            }
            accumulate_registers(ids, weights[s] * dt);
            double a0 = a0s[s], a1 = a1s[s];
            for (int64_t id : ids) {
                AmrBlock& b = blocks[id];
                for (size_t c = 0; c < b.u.size(); c++)
                    for (int q = 0; q < N; q++) b.u[c][q] = a0 * b.u0[c][q] + a1 * (b.u[c][q] + dt * b.rhs[c][q]);
            }
        }
        bool finer = false;
        if (l + 1 < cfg.levels)
            for (const AmrBlock& b : blocks) finer = finer || b.level == l + 1;
        if (finer) {
            level_t0[l + 1] = t0;
            advance_level(l + 1, 0.5 * dt);
            level_t0[l + 1] = t0 + 0.5 * dt;
            advance_level(l + 1, 0.5 * dt);
            reflux_level(l);
            restrict_level_full(l);
        }
        level_t0[l] = t0 + dt;
    }

    // amr.rs:1902-1910: every ancestor of level l from level l+1
    void restrict_level_full(int64_t l) {
        int64_t lo0[3] = {0, 0, 0}, hi0[3] = {bd(0), bd(1), bd(2)};
        std::vector<int64_t> ids;
        for (size_t i = 0; i < blocks.size(); i++)
            if (!blocks[i].leaf && blocks[i].level == l) ids.push_back(i);
        std::vector<std::vector<V>> fresh(ids.size());
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t n = 0; n < (int64_t)ids.size(); n++) fresh[n] = restrict_box(l, blocks[ids[n]].idx, lo0, hi0);
        for (size_t n = 0; n < ids.size(); n++) blocks[ids[n]].u = std::move(fresh[n]);
    }

    // amr.rs:1912-1952: one subcycled step, level lmin by dt
    void step_subcycled(double dt) {
        creg.clear();
        freg.clear();
        for (int64_t l = 0; l < cfg.levels; l++) level_t0[l] = t;
        for (int64_t l = cfg.levels - 2; l >= 0; l--) restrict_level_full(l);
        int64_t lmin = coarsest_leaf_level();
        advance_level(lmin, dt);
        for (int64_t l = lmin - 1; l >= 0; l--) restrict_level_full(l);
        t += dt;
        steps += 1;
        if (next_regrid > steps + 2) next_regrid = steps + 1;
        if (steps >= next_regrid) {
            auto before = structure();
            regrid();
            bool changed = structure() != before;
            regrid_interval = changed ? cfg.regrid_every : std::min(2 * regrid_interval, 2 * cfg.regrid_every);
            next_regrid = steps + (changed ? 1 : 2);
        }
    }

    // amr.rs:1991-2005
    V totals() const {
        std::vector<int> dm = dims();
        V s{0, 0, 0, 0, 0};
        for (auto& b : blocks) {
            if (!b.leaf) continue;
            double vol = 1.0;
            for (int d : dm) vol = vol * dx(b.level, d);
            for (const V& u : b.u)
                for (int q = 0; q < N; q++) s[q] = s[q] + u[q] * vol;
        }
        return s;
    }
    int64_t leaf_count() const {
        int64_t n = 0;
        for (auto& b : blocks) n += b.leaf ? 1 : 0;
        return n;
    }
};

using Amr = AmrT<AmrEuler>;
using AmrFiveEq = AmrT<AmrFive>;

}  // namespace oracle
