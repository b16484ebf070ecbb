// Device solver: layout, memory and the per-iteration launch sequence.
//
// Layout (sized for one GPU):
//  * interior cells renumbered along a 3D/2D Hilbert curve of their centroids
//    (B200 gathers hit L2 far more often when neighbours are close in memory),
//    then ghost cells ordered by their interior neighbour, so each interior
//    cell owns a contiguous ghost range;
//  * faces: interior faces sorted by their lower cell id, then boundary faces;
//    gathered data (cell state, gradients + limiter, face geometry) are
//    16-byte-aligned records (devgrid.hpp);
//  * per cell a CSR of (face, side) sorted by the reference's face-loop order,
//    so every per-cell sum is formed in the reference's order whatever the
//    device numbering, plus a 4-bit permutation that replays the cell's own
//    face order (used by LocalAccTime1/2 and least squares).
// One RK stage is face pass -> cell pass (the cell pass also updates the
// cell's ghosts and the norms) in the parallel modes, or face pass -> cell
// update -> ghost pass -> norms for the sequential LocalAccTime1 mode and the
// stage-by-stage API. Gradients run once per iteration before stage 0
// (psstFiniteVolumeGrid.cpp:307-308).
// Merged grids (psst_grid_merge) keep each case contiguous in device order and
// carry a per-cell case id, per-case run flags and per-case residual columns.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include <cuda_runtime_api.h>

#include "host.hpp"
#include "ops.hpp"

using namespace psst;

namespace {

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) raise(PSST_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707 (2004):
// axes -> transposed Hilbert index, then bit interleave into one key.
uint64_t hilbert_key(uint32_t *X, int b, int n) {
    uint32_t M = 1u << (b - 1), P, Q, t;
    for (Q = M; Q > 1; Q >>= 1) {
        P = Q - 1;
        for (int i = 0; i < n; i++) {
            if (X[i] & Q) {
                X[0] ^= P;
            } else {
                t = (X[0] ^ X[i]) & P;
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    for (int i = 1; i < n; i++) X[i] ^= X[i - 1];
    t = 0;
    for (Q = M; Q > 1; Q >>= 1)
        if (X[n - 1] & Q) t ^= Q - 1;
    for (int i = 0; i < n; i++) X[i] ^= t;
    uint64_t key = 0;
    for (int bit = b - 1; bit >= 0; --bit)
        for (int i = 0; i < n; ++i) key = (key << 1) | ((X[i] >> bit) & 1u);
    return key;
}

struct Layout {
    int32_t nint = 0, nghost = 0, nall = 0, nface = 0, nfi = 0, nlevels = 0, ncase = 1;
    std::vector<int32_t> cell_case;   // merged grids: case of each device cell
    std::vector<int32_t> dev_of_vol;  // reference volume -> device cell (-1: inactive)
    std::vector<int64_t> vol_of_dev;  // device cell -> reference volume
    std::vector<int32_t> c0, c1, csr_ptr, csr_ent, csr_nb, rank, gptr, g_nb, g_face, g_zone, z_dyn, z_therm, lvl_cells, lvl_ptr;
    // wavefront schedule of the sequential LocalAccTime1 (WfSched)
    int32_t wf_period = 1, wf_max_class_items = 0;
    std::vector<int32_t> wf_cells32, wf_item_level, wf_lvl_items;
    std::vector<uint32_t> wf_lowmask;
    std::vector<uint64_t> wperm;
    std::vector<double> S, n, xf, beta, V, xc, lsq_r, vk_eps2, z_u, z_p, z_T;
};

void build_layout(const psst_grid &G, const psst_scheme &sc, Layout &L) {
    const int dim = G.dim;
    // Adapted meshes: parent cells (bc 32) are never updated and parent faces
    // (bc 31) are in no cell's face list and in no face loop
    // (psstAnsysGridReader.cpp:825-883), so neither has a device slot.
    if (G.max_faces > 16) raise(PSST_ERR_UNSUPPORTED, "cells with more than 16 faces are not supported");
    // interior cells in the reference's update order (psstFiniteVolumeGrid.cpp:312-318)
    std::vector<int64_t> ref_int;
    for (auto &z : G.vz)
        if (z.bc == 1)
            for (int64_t i = 0; i < z.count; ++i) ref_int.push_back(z.first + i);
    L.nint = (int32_t)ref_int.size();
    L.nghost = (int32_t)G.nghost;
    L.nall = L.nint + L.nghost;
    L.dev_of_vol.assign(G.nvol, -1);
    std::vector<int64_t> order(L.nint);
    std::iota(order.begin(), order.end(), 0);
    if (sc.renumber && L.nint > 1) {
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int64_t v : ref_int)
            for (int k = 0; k < dim; ++k) {
                lo[k] = std::min(lo[k], G.xc[v * dim + k]);
                hi[k] = std::max(hi[k], G.xc[v * dim + k]);
            }
        const int bits = dim == 3 ? 21 : 31;
        const double scale = (double)((1u << bits) - 1);
        // (case, Hilbert key, reference position): sorting these orders each
        // case contiguously (merged grids), Hilbert order inside it, ties in
        // reference order
        struct Key {
            int64_t cs;
            uint64_t key;
            int64_t i;
            bool operator<(const Key &o) const {
                return cs != o.cs ? cs < o.cs : key != o.key ? key < o.key : i < o.i;
            }
        };
        std::vector<Key> keys(L.nint);
        parallel_for(L.nint, [&](int64_t i0, int64_t i1) {
            for (int64_t i = i0; i < i1; ++i) {
                uint32_t X[3] = {0, 0, 0};
                for (int k = 0; k < dim; ++k) {
                    const double span = hi[k] - lo[k];
                    const double t = span > 0 ? (G.xc[ref_int[i] * dim + k] - lo[k]) / span : 0.0;
                    X[k] = (uint32_t)std::min(scale, std::max(0.0, t * scale));
                }
                const int64_t cs = G.case_vol_ptr.empty()
                                       ? 0
                                       : std::upper_bound(G.case_vol_ptr.begin(), G.case_vol_ptr.end(), ref_int[i]) -
                                             G.case_vol_ptr.begin();
                keys[i] = Key{cs, hilbert_key(X, bits, dim), i};
            }
        });
        parallel_sort(keys, [](const Key &a, const Key &b) { return a < b; });
        for (int32_t i = 0; i < L.nint; ++i) order[i] = keys[i].i;
    }
    L.vol_of_dev.assign(L.nall, -1);
    L.rank.assign(L.nint, 0);
    for (int32_t d = 0; d < L.nint; ++d) {
        const int64_t v = ref_int[order[d]];
        L.dev_of_vol[v] = d;
        L.vol_of_dev[d] = v;
        L.rank[d] = (int32_t)order[d];
    }
    // ghosts, ordered by their interior neighbour
    std::vector<std::pair<int32_t, int64_t>> gh;
    for (int64_t v = 0; v < G.nvol; ++v) {
        if (!G.vol_boundary[v]) continue;
        const int64_t f = G.vf_idx[G.vf_ptr[v]];
        const int64_t nb = G.f_c0[f] == v ? G.f_c1[f] : G.f_c0[f];
        if (nb < 0 || L.dev_of_vol[nb] < 0) raise(PSST_ERR_FORMAT, "ghost cell without an interior neighbour");
        gh.emplace_back(L.dev_of_vol[nb], v);
    }
    std::stable_sort(gh.begin(), gh.end(), [](auto &a, auto &b) { return a.first < b.first; });
    std::vector<int32_t> zslot(G.vz.size(), -1);
    for (size_t i = 0; i < gh.size(); ++i) {
        const int64_t v = gh[i].second;
        const int32_t d = L.nint + (int32_t)i;
        L.dev_of_vol[v] = d;
        L.vol_of_dev[d] = v;
    }
    if (!G.case_vol_ptr.empty()) {
        L.ncase = (int32_t)G.case_vol_ptr.size() - 1;
        L.cell_case.resize(L.nall);
        for (int32_t d = 0; d < L.nall; ++d)
            L.cell_case[d] = (int32_t)(std::upper_bound(G.case_vol_ptr.begin(), G.case_vol_ptr.end(),
                                                        L.vol_of_dev[d]) - G.case_vol_ptr.begin()) - 1;
    }
    // faces: interior (both sides interior cells) first, then boundary
    std::vector<int64_t> fint, fbnd;
    for (int64_t f = 0; f < G.nface; ++f) {
        if (G.fz[G.f_fz[f]].bc == 31) continue;
        const int64_t a = G.f_c0[f], b = G.f_c1[f];
        if (a < 0 || b < 0) raise(PSST_ERR_FORMAT, "face without two neighbours");
        if (L.dev_of_vol[a] < 0 || L.dev_of_vol[b] < 0) raise(PSST_ERR_FORMAT, "face next to a parent cell");
        const bool zone_interior = G.fz[G.f_fz[f]].bc == 2;
        const bool ga = G.vol_boundary[a], gb = G.vol_boundary[b];
        if (zone_interior && (ga || gb)) raise(PSST_ERR_FORMAT, "interior face next to a ghost cell");
        if (!zone_interior && ga == gb) raise(PSST_ERR_FORMAT, "boundary face without exactly one ghost side");
        (zone_interior ? fint : fbnd).push_back(f);
    }
    // stable counting sort of each list by its lower device cell
    auto by_lowcell = [&](std::vector<int64_t> &fs) {
        std::vector<int64_t> start((size_t)L.nall + 1, 0);
        std::vector<int32_t> low(fs.size());
        for (size_t i = 0; i < fs.size(); ++i) {
            low[i] = std::min(L.dev_of_vol[G.f_c0[fs[i]]], L.dev_of_vol[G.f_c1[fs[i]]]);
            ++start[(size_t)low[i] + 1];
        }
        for (int32_t c = 0; c < L.nall; ++c) start[(size_t)c + 1] += start[(size_t)c];
        std::vector<int64_t> out(fs.size());
        for (size_t i = 0; i < fs.size(); ++i) out[(size_t)start[(size_t)low[i]]++] = fs[i];
        fs.swap(out);
    };
    by_lowcell(fint);
    by_lowcell(fbnd);
    L.nfi = (int32_t)fint.size();
    L.nface = (int32_t)(fint.size() + fbnd.size());
    std::vector<int32_t> dev_face(G.nface, -1);
    std::vector<int64_t> ref_face(L.nface);
    for (size_t i = 0; i < fint.size(); ++i) ref_face[i] = fint[i];
    for (size_t i = 0; i < fbnd.size(); ++i) ref_face[fint.size() + i] = fbnd[i];
    for (int32_t d = 0; d < L.nface; ++d) dev_face[ref_face[d]] = d;
    L.c0.resize(L.nface);
    L.c1.resize(L.nface);
    L.S.resize(L.nface);
    L.beta.resize(L.nface);
    L.n.resize((size_t)dim * L.nface);
    L.xf.resize((size_t)dim * L.nface);
    parallel_for(L.nface, [&](int64_t d0, int64_t d1) {
        for (int64_t d = d0; d < d1; ++d) {
            const int64_t f = ref_face[d];
            L.c0[d] = L.dev_of_vol[G.f_c0[f]];
            L.c1[d] = L.dev_of_vol[G.f_c1[f]];
            L.S[d] = G.S[f];
            L.beta[d] = G.beta[f];
            for (int k = 0; k < dim; ++k) {
                L.n[(size_t)k * L.nface + d] = G.n[f * dim + k];
                L.xf[(size_t)k * L.nface + d] = G.xf[f * dim + k];
            }
        }
    });
    // cells: volume, centroid, CSR sorted by reference face index (= loop order)
    L.V.resize(L.nint);
    L.xc.resize((size_t)dim * L.nall);
    parallel_for(L.nall, [&](int64_t d0, int64_t d1) {
        for (int64_t d = d0; d < d1; ++d) {
            const int64_t v = L.vol_of_dev[d];
            if (d < L.nint) L.V[d] = G.V[v];
            for (int k = 0; k < dim; ++k) L.xc[(size_t)k * L.nall + d] = G.xc[v * dim + k];
        }
    });
    L.csr_ptr.assign(L.nint + 1, 0);
    L.wperm.assign(L.nint, 0);
    for (int32_t d = 0; d < L.nint; ++d) {
        const int64_t v = L.vol_of_dev[d];
        L.csr_ptr[d + 1] = L.csr_ptr[d] + (int32_t)(G.vf_ptr[v + 1] - G.vf_ptr[v]);
    }
    L.csr_ent.resize(L.csr_ptr[L.nint]);
    L.csr_nb.resize(L.csr_ptr[L.nint]);
    parallel_for(L.nint, [&](int64_t d0, int64_t d1) {
        for (int64_t d = d0; d < d1; ++d) {
            const int64_t v = L.vol_of_dev[d];
            const int64_t b = G.vf_ptr[v], k = G.vf_ptr[v + 1] - b;  // k <= 16 (checked above)
            int idx[16], pos[16];
            std::iota(idx, idx + k, 0);
            std::stable_sort(idx, idx + k, [&](int x, int y) { return G.vf_idx[b + x] < G.vf_idx[b + y]; });
            for (int q = 0; q < k; ++q) {
                const int64_t f = G.vf_idx[b + idx[q]];
                const int side = G.f_c0[f] == v ? 0 : 1;
                L.csr_ent[L.csr_ptr[d] + q] = (dev_face[f] << 1) | side;
                L.csr_nb[L.csr_ptr[d] + q] = side ? L.c0[dev_face[f]] : L.c1[dev_face[f]];
                pos[idx[q]] = q;
            }
            uint64_t perm = 0;
            for (int j = 0; j < k; ++j) perm |= (uint64_t)pos[j] << (4 * j);
            L.wperm[d] = perm;
        }
    });
    // ghost tables and boundary zones; ghosts are sorted by interior neighbour,
    // so each interior cell owns a contiguous ghost range [gptr[d], gptr[d+1])
    L.g_nb.resize(L.nghost);
    L.g_face.resize(L.nghost);
    L.g_zone.resize(L.nghost);
    L.gptr.assign(L.nint + 1, 0);
    for (int32_t i = 0; i < L.nghost; ++i) L.gptr[gh[i].first + 1]++;
    for (int32_t d = 0; d < L.nint; ++d) L.gptr[d + 1] += L.gptr[d];
    for (int32_t i = 0; i < L.nghost; ++i) {
        const int64_t v = L.vol_of_dev[L.nint + i];
        const int64_t f = G.vf_idx[G.vf_ptr[v]];
        const int64_t nb = G.f_c0[f] == v ? G.f_c1[f] : G.f_c0[f];
        L.g_nb[i] = L.dev_of_vol[nb];
        L.g_face[i] = dev_face[f];
        const int32_t zs = G.vol_vz[v];
        if (zslot[zs] < 0) {
            const VZone &z = G.vz[zs];
            zslot[zs] = (int32_t)L.z_dyn.size();
            L.z_dyn.push_back(z.dyn);
            L.z_therm.push_back(z.therm);
            for (int k = 0; k < 3; ++k) L.z_u.push_back(z.u[k]);
            L.z_p.push_back(z.p);
            L.z_T.push_back(z.T);
        }
        L.g_zone[i] = zslot[zs];
    }
    if (L.z_dyn.empty()) {  // keep device arrays non-empty
        L.z_dyn.push_back(0);
        L.z_therm.push_back(0);
        L.z_u.assign(3, 0.0);
        L.z_p.push_back(0);
        L.z_T.push_back(0);
    }
    // least squares: r_ table indexed by the zone-local position
    // (psstGradCalculation.cpp:404-412), one device array per coefficient
    const int nr = dim == 2 ? 3 : kLsqNR;
    if (sc.order == 2 && sc.grad == 2) {
        const std::vector<double> tab = lsq_table(G);
        L.lsq_r.assign((size_t)nr * L.nint, 0.0);
        for (int32_t d = 0; d < L.nint; ++d) {
            const int64_t v = L.vol_of_dev[d];
            const int64_t i = v - G.vz[G.vol_vz[v]].first;
            for (int q = 0; q < nr; ++q) L.lsq_r[(size_t)q * L.nint + d] = tab[kLsqNR * i + q];
        }
    } else {
        L.lsq_r.assign(1, 0.0);
    }
    L.vk_eps2.assign(L.nint, 0.0);
    for (int32_t d = 0; d < L.nint; ++d) {
        const double h = dim == 2 ? std::sqrt(L.V[d]) : std::cbrt(L.V[d]);
        const double kh = sc.venkat_k * h;
        L.vk_eps2[d] = kh * kh * kh;
    }
    // level schedule for the sequential LocalAccTime1: a cell's level exceeds
    // that of every interior neighbour updated before it in the reference.
    std::vector<int32_t> level(L.nint, 0);
    std::vector<int32_t> dev_by_rank(L.nint);
    for (int32_t d = 0; d < L.nint; ++d) dev_by_rank[L.rank[d]] = d;
    int32_t maxlvl = -1;
    for (int32_t r = 0; r < L.nint; ++r) {
        const int32_t d = dev_by_rank[r];
        int32_t lv = 0;
        for (int32_t q = L.csr_ptr[d]; q < L.csr_ptr[d + 1]; ++q) {
            const int32_t f = L.csr_ent[q] >> 1;
            const int32_t nb = (L.csr_ent[q] & 1) ? L.c0[f] : L.c1[f];
            if (nb < L.nint && L.rank[nb] < r) lv = std::max(lv, level[nb] + 1);
        }
        level[d] = lv;
        maxlvl = std::max(maxlvl, lv);
    }
    L.nlevels = maxlvl + 1;
    L.lvl_ptr.assign(L.nlevels + 1, 0);
    for (int32_t d = 0; d < L.nint; ++d) L.lvl_ptr[level[d] + 1]++;
    for (int32_t l = 0; l < L.nlevels; ++l) L.lvl_ptr[l + 1] += L.lvl_ptr[l];
    L.lvl_cells.resize(L.nint);
    std::vector<int32_t> fillp(L.lvl_ptr.begin(), L.lvl_ptr.end() - 1);
    for (int32_t r = 0; r < L.nint; ++r) {
        const int32_t d = dev_by_rank[r];
        L.lvl_cells[fillp[level[d]]++] = d;
    }
    // wavefront schedule: period P = 1 + the largest level difference across
    // an interior face; items of at most kWfBlock / kWfLanes cells of one level (device
    // order inside a level), ordered by level mod P, then level
    if (sc.lc == 1 && sc.lc1_mode == PSST_LC1_SEQUENTIAL && L.nint > 0) {
        int32_t D = 0;
        for (int32_t d = 0; d < L.nint; ++d)
            for (int32_t q = L.csr_ptr[d]; q < L.csr_ptr[d + 1]; ++q) {
                const int32_t nb = L.csr_nb[q];
                if (nb < L.nint) D = std::max(D, std::abs(level[d] - level[nb]));
            }
        L.wf_period = D + 1;
        std::vector<int32_t> by_level(L.nint), fill(L.lvl_ptr.begin(), L.lvl_ptr.end() - 1);
        for (int32_t d = 0; d < L.nint; ++d) by_level[fill[level[d]]++] = d;
        L.wf_lvl_items.assign((size_t)2 * L.nlevels, 0);
        L.wf_cells32.clear();
        L.wf_item_level.clear();
        const int32_t per_item = kWfBlock / kWfLanes;
        for (int32_t r = 0; r < L.wf_period; ++r) {
            const int32_t first = (int32_t)L.wf_item_level.size();
            for (int32_t l = r; l < L.nlevels; l += L.wf_period) {
                L.wf_lvl_items[2 * (size_t)l] = (int32_t)L.wf_item_level.size();
                for (int32_t b = L.lvl_ptr[l]; b < L.lvl_ptr[l + 1]; b += per_item) {
                    L.wf_item_level.push_back(l);
                    for (int32_t i = b; i < b + per_item; ++i)
                        L.wf_cells32.push_back(i < L.lvl_ptr[l + 1] ? by_level[i] : -1);
                }
                L.wf_lvl_items[2 * (size_t)l + 1] = (int32_t)L.wf_item_level.size();
            }
            L.wf_max_class_items = std::max(L.wf_max_class_items, (int32_t)L.wf_item_level.size() - first);
        }
        // neighbours updated before each cell in the reference's order, per CSR entry
        L.wf_lowmask.assign(L.nint, 0u);
        for (int32_t d = 0; d < L.nint; ++d)
            for (int32_t q = L.csr_ptr[d]; q < L.csr_ptr[d + 1]; ++q) {
                const int32_t nb = L.csr_nb[q];
                if (nb < L.nint && L.rank[nb] < L.rank[d]) L.wf_lowmask[d] |= 1u << (q - L.csr_ptr[d]);
            }
    }
}


// Face records: neighbours, area, normal and the reconstruction offsets of the
// scheme in use (formed in FP64, rounded once to R).
template <typename R, int DIM>
std::vector<FaceRec<R, DIM>> build_face_records(const psst_grid &G, const Layout &L, int rec) {
    std::vector<FaceRec<R, DIM>> out(L.nface);
    parallel_for(L.nface, [&](int64_t d0, int64_t d1) {
        for (int64_t d = d0; d < d1; ++d) {
            FaceRec<R, DIM> r;
            std::memset(&r, 0, sizeof r);
            r.c0 = L.c0[d];
            r.c1 = L.c1[d];
            r.S = L.S[d];
            for (int k = 0; k < DIM; ++k) {
                r.n[k] = L.n[(size_t)k * L.nface + d];
                const double xf = L.xf[(size_t)k * L.nface + d];
                const double x0 = L.xc[(size_t)k * L.nall + r.c0], x1 = L.xc[(size_t)k * L.nall + r.c1];
                if (rec == 1) {  // Darwish-Moukalled: R = x_c0 - x_c1 (psstValueReconstructor.cpp:105-107)
                    r.o0[k] = (R)(x0 - x1);
                } else if (rec == 2) {  // MUSCL: x_f - x_c per side
                    r.o0[k] = (R)(xf - x0);
                    r.o1[k] = (R)(xf - x1);
                }
            }
            out[d] = r;
        }
    });
    (void)G;
    return out;
}

// The Green-Gauss table of DevGrid::gcoef (meshes with 4 faces per cell):
// per CSR entry q = 4c + j, component-major so that a cell's 4 values of one
// component are one 16-byte (FP32) or 32-byte (FP64) load. FP32: products and
// quotients in FP64, each value rounded to FP32 once. FP64: the face record's
// own values (S / V as the general path divides it, n, beta), so the kernel's
// arithmetic and its order are the general path's. Offsets: the face
// records' o0 / o1 (side 0 / side 1), rounded to R as there.
template <typename R>
std::vector<R> build_gradient_coefficients(const Layout &L, int dim, int rec) {
    constexpr bool F64 = sizeof(R) == 8;
    const int64_t ne = (int64_t)4 * L.nint;
    const int ncomp = 2 * dim + (F64 ? 2 : 1), off0 = F64 ? dim + 2 : dim + 1;
    std::vector<R> out((size_t)ncomp * ne);
    parallel_for(ne, [&](int64_t q0, int64_t q1) {
        for (int64_t q = q0; q < q1; ++q) {
            const int32_t c = (int32_t)(q / 4), ent = L.csr_ent[q], f = ent >> 1, side = ent & 1;
            const int32_t c0 = L.c0[f], c1 = L.c1[f];
            const double sv = (side ? 1.0 : -1.0) * (L.S[f] / L.V[c]);
            for (int k = 0; k < dim; ++k) {
                const double n = L.n[(size_t)k * L.nface + f];
                if (F64)
                    out[(size_t)(1 + k) * ne + q] = (R)n;
                else
                    out[(size_t)k * ne + q] = (R)(sv * n);
                const double xf = L.xf[(size_t)k * L.nface + f];
                const double x0 = L.xc[(size_t)k * L.nall + c0], x1 = L.xc[(size_t)k * L.nall + c1];
                R o = (R)0;  // as build_face_records stores o0 (side 0) / o1 (side 1)
                if (rec == 1 && !side) o = (R)(x0 - x1);
                if (rec == 2) o = (R)(xf - (side ? x1 : x0));
                out[(size_t)(off0 + k) * ne + q] = o;
            }
            if (F64) {
                out[q] = (R)sv;  // negation is exact: |sv| is the general path's S / V
                out[(size_t)(dim + 1) * ne + q] = (R)L.beta[f];
            } else {
                out[(size_t)dim * ne + q] = (R)(side ? L.beta[f] : 1.0 - L.beta[f]);
            }
        }
    });
    return out;
}

}  // namespace

struct psst_solver {
    int dim = 0, nv = 0, device = 0;
    psst_scheme sc{};
    Gas gas{};
    Layout L;
    int64_t nvol_ref = 0;
    DevGrid g{};
    DevState<double> s64[2]{};
    DevState<float> s32[2]{};
    DevWork<double> w64{};
    DevWork<float> w32{};
    int cur = 0;
    std::vector<void *> allocs;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t iter = 1;
    bool has_state = false;
    int64_t last_launches = 0;
    double last_ms = 0.0;
    int rec = 0, celllim = 0;
    bool seq = false;
    double dt_uniform = 0.0;
    int nblk = 1;  // blocks of the thread-per-cell kernels
    int norm_cap = 0;
    int last_n = 0;                    // iterations of the last psst_explicit_solve
    int32_t *d_vol = nullptr;          // reference volume of each device cell
    double *d_prim = nullptr, *d_w = nullptr, *d_rho = nullptr;  // reference-ordered state staging
    std::vector<int32_t> active_h;     // merged grids: per-case run flags (host copy)
    // pinned host staging of a call's residual columns and error word: one
    // stream synchronisation per call, no pageable-memory copies
    double *hnorm = nullptr;
    size_t hnorm_cap = 0;
    // CUDA graphs of whole psst_explicit_solve calls, keyed by (n_iter, buffer
    // parity), and of run-to-stop launches, keyed by (-chunk, buffer parity)
    bool use_graphs = false;
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
    std::map<std::pair<int, int>, int64_t> graph_launches;
    // merged grids: the per-case stop rule evaluated on the device (CaseStop)
    bool stop_on = false;
    CaseStop stop{};
    // run-to-stop launches: the loop's control block and residual history
    LoopCtl *loopctl = nullptr;
    double *hist_linf = nullptr, *hist_l2 = nullptr;
    int64_t hist_rows = 0;
    // sequential LocalAccTime1 as one persistent launch per call (FP64, single
    // grids): schedule uploaded (wf_ready), switched on (wf_on), CTAs, and the
    // bound of every grid-barrier wait
    bool wf_ready = false, wf_on = true;
    WfSched wf{};
    int wf_blocks = 0;
    uint64_t wait_ns = kDefaultWaitNs;
    static constexpr uint64_t kDefaultWaitNs = 10000000000ull;  // 10 s; a step takes microseconds

    void drop_graphs() {
        for (auto &kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
        graph_launches.clear();
    }
    void *dalloc_bytes(size_t n) {
        void *p = nullptr;
        ck(cudaMalloc(&p, std::max<size_t>(n, 16)), "cudaMalloc");
        allocs.push_back(p);
        return p;
    }
    // frees a buffer from dalloc (null: nothing)
    void dfree(void *p) {
        if (!p) return;
        auto it = std::find(allocs.begin(), allocs.end(), p);
        if (it != allocs.end()) {
            allocs.erase(it);
            cudaFree(p);
        }
    }
    template <class T>
    T *dalloc(size_t n) {
        return (T *)dalloc_bytes(std::max<size_t>(n, 1) * sizeof(T));
    }
    template <class T>
    T *upload(const std::vector<T> &v) {
        T *p = dalloc<T>(v.size());
        if (!v.empty()) ck(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
        return p;
    }
    ~psst_solver() {
        if (device >= 0) cudaSetDevice(device);
        drop_graphs();
        for (void *p : allocs) cudaFree(p);
        if (hnorm) cudaFreeHost(hnorm);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

namespace {

template <typename R>
DevState<R> *states(psst_solver *s);
template <>
DevState<double> *states<double>(psst_solver *s) {
    return s->s64;
}
template <>
DevState<float> *states<float>(psst_solver *s) {
    return s->s32;
}
template <typename R>
DevWork<R> &work(psst_solver *s);
template <>
DevWork<double> &work<double>(psst_solver *s) {
    return s->w64;
}
template <>
DevWork<float> &work<float>(psst_solver *s) {
    return s->w32;
}

template <typename R>
void alloc_state(psst_solver *s, const psst_grid &G) {
    const int dim = s->dim;
    const int32_t nall = s->L.nall, nint = s->L.nint, nface = s->L.nface;
    if (dim == 2)
        s->g.frec = s->upload(build_face_records<R, 2>(G, s->L, s->rec));
    else
        s->g.frec = s->upload(build_face_records<R, 3>(G, s->L, s->rec));
    {  // face area per CSR entry, rounded to R as the face pass rounds it
        std::vector<R> cs(s->L.csr_ent.size());
        for (size_t q = 0; q < cs.size(); ++q) cs[q] = (R)s->L.S[s->L.csr_ent[q] >> 1];
        s->g.csr_s = s->upload(cs);
    }
    if (s->g.kuni == 4 && s->sc.order == 2 && s->sc.grad == 1)
        s->g.gcoef = s->upload(build_gradient_coefficients<R>(s->L, dim, s->rec));
    DevState<R> *st = states<R>(s);
    for (int b = 0; b < 2; ++b) {
        st[b].rec = s->dalloc<CellRec<R>>(nall);
        ck(cudaMemset(st[b].rec, 0, (size_t)std::max(nall, 1) * sizeof(CellRec<R>)), "memset");
    }
    DevWork<R> &w = work<R>(s);
    const int nv = s->nv;
    const size_t gbytes = Ops<R>::grad_rec_bytes(dim);
    w.w = s->dalloc<double>((size_t)nv * nint);
    w.pw = s->dalloc<double>((size_t)nv * nint);
    w.grec = s->dalloc_bytes(gbytes * std::max(nint, 1));
    w.fout = s->dalloc_bytes(Ops<R>::face_out_bytes(dim) * std::max(nface, 1));
    w.res = s->dalloc<R>((size_t)nv * nint);
    w.dt = s->dalloc<double>(nint);
    // sized for the smallest cell-pass block (64 threads): one partial per block and RK stage
    w.l2part = s->dalloc<double>((size_t)2 * nv * std::max(nblocks(nint, kMinBlock), 1) * s->sc.rk_level);
    w.l2mid = s->dalloc<double>((size_t)2 * nv * kNormReduceBlocks * s->sc.rk_level);
    w.ticket = s->dalloc<unsigned int>(1);
    w.err = s->dalloc<int32_t>(4);
    ck(cudaMemset(w.grec, 0, gbytes * std::max(nint, 1)), "memset");
    ck(cudaMemset(w.res, 0, (size_t)std::max(nv * nint, 1) * sizeof(R)), "memset");
    ck(cudaMemset(w.dt, 0, (size_t)std::max(nint, 1) * sizeof(double)), "memset");
    ck(cudaMemset(w.ticket, 0, sizeof(unsigned int)), "memset");
    ck(cudaMemset(w.err, 0, 4 * sizeof(int32_t)), "memset");
}

// Residual-norm buffers for n_iter iterations (allocated once, grown on
// demand; growing invalidates captured graphs, which hold the old pointers).
template <typename R>
void reserve_norms(psst_solver *s, int n_iter) {
    DevWork<R> &w = work<R>(s);
    if (n_iter > s->norm_cap) {
        s->drop_graphs();
        ck(cudaStreamSynchronize(s->stream), "stream sync");  // no launch still reads the old buffers
        s->dfree(w.linf);
        s->dfree(w.l2);
        s->dfree(w.case_linf);
        s->norm_cap = std::max(n_iter, 2 * s->norm_cap);
        w.linf = s->dalloc<double>((size_t)s->norm_cap * s->nv);
        w.l2 = s->dalloc<double>((size_t)s->norm_cap * s->nv);
        if (!s->L.cell_case.empty())
            w.case_linf = s->dalloc<unsigned long long>((size_t)s->norm_cap * s->L.ncase * s->nv);
    }
}

template <typename R>
void zero_norms(psst_solver *s, int n_iter) {
    DevWork<R> &w = work<R>(s);
    ck(cudaMemsetAsync(w.linf, 0, (size_t)n_iter * s->nv * sizeof(double), s->stream), "memset");
    ck(cudaMemsetAsync(w.l2, 0, (size_t)n_iter * s->nv * sizeof(double), s->stream), "memset");
    if (w.case_linf)
        ck(cudaMemsetAsync(w.case_linf, 0, (size_t)n_iter * s->L.ncase * s->nv * sizeof(unsigned long long),
                           s->stream),
           "memset");
}

template <typename R>
void ensure_norms(psst_solver *s, int n_iter) {
    reserve_norms<R>(s, n_iter);
    zero_norms<R>(s, n_iter);
}

// e: the error word as copied to the host after the stream synchronised;
// a set word is cleared on the device and raised.
void raise_err(psst_solver *s, const int32_t e[4], const int32_t *err_dev) {
    if (e[0] == 0) return;
    ck(cudaMemsetAsync((void *)err_dev, 0, 4 * sizeof(int32_t), s->stream), "memset");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    switch (e[0]) {
    case 1:
        raise(PSST_ERR_FLUX, "Error: Could not calculate convective HLL flow!");
    case 2:
        raise(PSST_ERR_FLUX, "Error: Could not calculate convective HLLC flow!");
    case 3:
        raise(PSST_ERR_NONFINITE, "non-finite residual in cell " + std::to_string(s->L.vol_of_dev[e[1]]));
    case 5:
        raise(PSST_ERR_TIMEOUT, "a grid-barrier wait of the wavefront launch ran out (step " + std::to_string(e[1]) +
                                    "); the state is undefined until the next psst_solver_set_state");
    default:
        raise(PSST_ERR_NONFINITE, "non-positive density or temperature in cell " + std::to_string(s->L.vol_of_dev[e[1]]));
    }
}

void check_err(psst_solver *s, const int32_t *err_dev) {
    int32_t e[4] = {0, 0, 0, 0};
    ck(cudaMemcpyAsync(e, err_dev, sizeof e, cudaMemcpyDeviceToHost, s->stream), "err copy");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    raise_err(s, e, err_dev);
}

enum Kind { K_GRADIENT = 0, K_FACE = 1, K_CELL = 2, K_GHOST = 3, K_NORM = 4 };

// One RK stage. The parallel modes run face pass -> cell pass (the cell pass
// also updates ghosts and finishes the norms); the sequential LocalAccTime1
// mode and the stage-by-stage API (gather == false: residual already in
// wk.res) run face pass -> cell update -> ghost pass -> norms.
// mark(kind) is called after each launch (profiling hook).
template <typename R, typename Mark>
void one_stage(psst_solver *s, int k, int it_slot, bool gather, Mark &&mark) {
    DevState<R> *st = states<R>(s);
    DevWork<R> &w = work<R>(s);
    const DevState<R> &cur = st[s->cur], &nxt = st[s->cur ^ 1];
    if (gather) {
        Ops<R>::face(s->dim, s->sc.flux, s->rec, s->sc.limiter, s->seq ? 0 : s->sc.lc, s->g, cur, w, s->gas,
                     s->stream);
        mark(K_FACE);
    }
    if (gather && !s->seq) {
        const int stage = (k == 0 ? 1 : 0) | (k == s->sc.rk_level - 1 ? 2 : 0);
        Ops<R>::cell(s->dim, s->sc.lc, s->g, cur, nxt, w, s->gas, s->sc.cfl, s->dt_uniform, s->sc.rk[k], stage, k,
                     it_slot, s->stream);
        mark(K_CELL);
        if (k == s->sc.rk_level - 1) {  // the iteration's residual columns
            Ops<R>::norm_reduce(s->dim, s->g, w, s->sc.rk_level, it_slot, s->stream);
            mark(K_NORM);
        }
    } else {
        Ops<R>::cell_update(s->dim, s->sc.lc, s->seq, gather, s->g, cur, nxt, w, s->gas, s->sc.cfl, s->dt_uniform,
                            s->sc.rk[k], k == 0, s->stream);
        mark(K_CELL);
        Ops<R>::ghost_update(s->dim, s->g, cur, nxt, s->gas, s->stream);
        mark(K_GHOST);
        Ops<R>::norm_finish(s->dim, w, s->seq ? 1 : s->nblk, s->L.nint, it_slot, s->stream);
        mark(K_NORM);
    }
    s->cur ^= 1;
}

bool wavefront_active(const psst_solver *s) { return s->seq && s->wf_ready && s->wf_on; }

// The whole call as one cooperative launch (the wavefront schedule, WfSched);
// the norm buffers are reserved and zeroed by the caller.
template <typename R>
void wavefront_run(psst_solver *s, int n_iter) {
    DevState<R> *st = states<R>(s);
    DevWork<R> &w = work<R>(s);
    ck(cudaMemsetAsync(s->wf.sync, 0, kWfSyncWords * sizeof(unsigned), s->stream), "memset");
    WfArgs<R> a{};
    a.g = s->g;
    a.buf[0] = st[0].rec;
    a.buf[1] = st[1].rec;
    a.wk = w;
    a.gbuf[0] = w.grec;
    a.gbuf[1] = s->wf.grec2;
    a.sc = s->wf;
    a.gas = s->gas;
    a.cfl = s->sc.cfl;
    for (int k = 0; k < 16; ++k) a.alpha[k] = s->sc.rk[k];
    a.nst = s->sc.rk_level;
    a.nopi = a.nst + (s->sc.order == 2 ? 1 : 0);
    a.nops = (int64_t)n_iter * a.nopi;
    a.n_iter = n_iter;
    a.flux = s->sc.flux;
    a.grad = s->sc.grad;
    a.celllim = s->celllim;
    a.in_buf = s->cur;
    a.wait_ns = s->wait_ns;
    ck(Ops<R>::wavefront(s->dim, s->rec, s->sc.limiter, a, s->wf_blocks, s->stream), "wavefront launch");
    s->cur = (int)((s->cur + (int64_t)n_iter * a.nst) & 1);
}

template <typename R, typename Mark>
void iterations(psst_solver *s, int n_iter, Mark &&mark) {
    DevWork<R> &w = work<R>(s);
    if (wavefront_active(s)) {
        wavefront_run<R>(s, n_iter);
        mark(K_CELL);
        return;
    }
    for (int it = 0; it < n_iter; ++it) {
        if (s->sc.order == 2) {
            Ops<R>::gradient(s->dim, s->sc.grad, s->celllim, s->g, states<R>(s)[s->cur], w, s->stream);
            mark(K_GRADIENT);
        }
        for (int k = 0; k < s->sc.rk_level; ++k) one_stage<R>(s, k, it, true, mark);
        if (s->stop_on) {
            Ops<R>::case_stop(s->dim, s->g, w, s->stop, it, s->stream);
            mark(K_NORM);
        }
    }
}

// n_iter iterations. With graphs on, the whole call (norm reset + every
// launch) is captured once per (n_iter, buffer parity) and replayed.
template <typename R>
void run(psst_solver *s, int n_iter, double *res_linf, double *res_l2) {
    DevWork<R> &w = work<R>(s);
    reserve_norms<R>(s, n_iter);
    int64_t launches = 0;
    ck(cudaEventRecord(s->ev0, s->stream), "event");
    if (s->use_graphs && !wavefront_active(s)) {  // a wavefront call is one launch already
        const std::pair<int, int> key(n_iter, s->cur);
        auto it = s->graphs.find(key);
        if (it == s->graphs.end()) {
            ck(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "graph capture");
            cudaGraph_t gr = nullptr;
            try {
                zero_norms<R>(s, n_iter);
                iterations<R>(s, n_iter, [&](int) { ++launches; });
            } catch (...) {
                cudaStreamEndCapture(s->stream, &gr);
                if (gr) cudaGraphDestroy(gr);
                throw;
            }
            ck(cudaStreamEndCapture(s->stream, &gr), "graph capture");
            cudaGraphExec_t ex = nullptr;
            const cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
            cudaGraphDestroy(gr);
            ck(e, "graph instantiate");
            it = s->graphs.emplace(key, ex).first;
            s->graph_launches[key] = launches;
        } else {
            launches = s->graph_launches[key];
            if ((int64_t)n_iter * s->sc.rk_level % 2) s->cur ^= 1;
        }
        ck(cudaGraphLaunch(it->second, s->stream), "graph launch");
    } else {
        zero_norms<R>(s, n_iter);
        iterations<R>(s, n_iter, [&](int) { ++launches; });
    }
    ck(cudaEventRecord(s->ev1, s->stream), "event");
    ck(cudaGetLastError(), "kernel launch");
    // residual columns and the error word into pinned staging, one sync
    const size_t nn = (size_t)n_iter * s->nv, need = 2 * nn + 2;
    if (s->hnorm_cap < need) {
        if (s->hnorm) cudaFreeHost(s->hnorm);
        s->hnorm = nullptr;
        s->hnorm_cap = 0;
        ck(cudaMallocHost(reinterpret_cast<void **>(&s->hnorm), need * sizeof(double)), "cudaMallocHost");
        s->hnorm_cap = need;
    }
    double *li = s->hnorm, *l2 = s->hnorm + nn;
    int32_t *he = reinterpret_cast<int32_t *>(s->hnorm + 2 * nn);
    ck(cudaMemcpyAsync(li, w.linf, nn * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "norm copy");
    ck(cudaMemcpyAsync(l2, w.l2, nn * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "norm copy");
    ck(cudaMemcpyAsync(he, w.err, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream), "err copy");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    {
        const int32_t e[4] = {he[0], he[1], he[2], he[3]};
        raise_err(s, e, w.err);
    }
    float ms = 0.0f;
    ck(cudaEventElapsedTime(&ms, s->ev0, s->ev1), "event time");
    s->last_ms = ms;
    s->last_launches = launches;
    s->last_n = n_iter;
    s->iter += n_iter;
    if (res_linf) std::memcpy(res_linf, li, nn * sizeof(double));
    if (res_l2) std::memcpy(res_l2, l2, nn * sizeof(double));
}

// Iterations under the case stop rule until every case has stopped, an error
// is raised or max_iter iterations have run, as ONE launch of a CUDA graph: a
// while-loop node repeats a captured block of `chunk` iterations whose last
// kernel (k_loop_control) sets the loop's condition on the device. The host
// waits once, at the end. chunk * RK stages must be even, so every block
// starts on the same state buffer (one captured body serves every pass).
// Returns the iterations run (whole blocks); the residual columns of the
// first min(that, max_iter) iterations go to res_linf / res_l2.
template <typename R>
int64_t run_to_stop(psst_solver *s, int64_t max_iter, int chunk, double *res_linf, double *res_l2) {
    DevWork<R> &w = work<R>(s);
    if (!s->stop_on) raise(PSST_ERR_STATE, "psst_solver_run_to_stop: no stop rule set (psst_solver_set_stop_rule)");
    if (wavefront_active(s)) raise(PSST_ERR_UNSUPPORTED, "psst_solver_run_to_stop: not with the sequential mode");
    if ((int64_t)chunk * s->sc.rk_level % 2)
        raise(PSST_ERR_ARG, "psst_solver_run_to_stop: chunk * RK stages must be even");
    reserve_norms<R>(s, chunk);
    // a history only when the caller wants the residual columns (the loop skips
    // the copy once the count reaches cap_rows)
    const int64_t rows = (res_linf || res_l2) ? (max_iter + chunk - 1) / chunk * chunk : 0;
    if (!s->loopctl) s->loopctl = s->dalloc<LoopCtl>(1);
    if (rows > s->hist_rows) {  // the graph reads the history's address from the control block
        ck(cudaStreamSynchronize(s->stream), "stream sync");
        s->dfree(s->hist_linf);
        s->dfree(s->hist_l2);
        s->hist_linf = s->dalloc<double>((size_t)rows * s->nv);
        s->hist_l2 = s->dalloc<double>((size_t)rows * s->nv);
        s->hist_rows = rows;
    }
    const LoopCtl ctl{0, max_iter, rows, s->hist_linf, s->hist_l2};
    ck(cudaMemcpyAsync(s->loopctl, &ctl, sizeof ctl, cudaMemcpyHostToDevice, s->stream), "loop control");
    const std::pair<int, int> key(-chunk, s->cur);
    auto it = s->graphs.find(key);
    if (it == s->graphs.end()) {
        cudaGraph_t gr = nullptr;
        ck(cudaGraphCreate(&gr, 0), "graph");
        int64_t launches = 0;
        try {
            cudaGraphConditionalHandle h;
            ck(cudaGraphConditionalHandleCreate(&h, gr, 1, cudaGraphCondAssignDefault), "graph condition");
            cudaGraphNodeParams p{};
            p.type = cudaGraphNodeTypeConditional;
            p.conditional.handle = h;
            p.conditional.type = cudaGraphCondTypeWhile;
            p.conditional.size = 1;
            cudaGraphNode_t node;
            ck(cudaGraphAddNode(&node, gr, nullptr, 0, &p), "graph loop node");
            cudaGraph_t body = p.conditional.phGraph_out[0];
            ck(cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
               "graph capture");
            try {
                zero_norms<R>(s, chunk);
                iterations<R>(s, chunk, [&](int) { ++launches; });
                Ops<R>::loop_control(s->dim, s->g, w, s->stop, s->loopctl, chunk, h, s->stream);
                ++launches;
            } catch (...) {
                cudaGraph_t dummy = nullptr;
                cudaStreamEndCapture(s->stream, &dummy);
                throw;
            }
            ck(cudaStreamEndCapture(s->stream, &body), "graph capture");
            cudaGraphExec_t ex = nullptr;
            ck(cudaGraphInstantiate(&ex, gr, 0), "graph instantiate");
            it = s->graphs.emplace(key, ex).first;
            s->graph_launches[key] = launches;
        } catch (...) {
            cudaGraphDestroy(gr);
            throw;
        }
        cudaGraphDestroy(gr);
    }
    ck(cudaEventRecord(s->ev0, s->stream), "event");
    ck(cudaGraphLaunch(it->second, s->stream), "graph launch");
    ck(cudaEventRecord(s->ev1, s->stream), "event");
    LoopCtl out{};
    int32_t e[4] = {0, 0, 0, 0};
    ck(cudaMemcpyAsync(&out, s->loopctl, sizeof out, cudaMemcpyDeviceToHost, s->stream), "loop control");
    ck(cudaMemcpyAsync(e, w.err, sizeof e, cudaMemcpyDeviceToHost, s->stream), "err copy");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    raise_err(s, e, w.err);
    const size_t n = (size_t)std::min(out.done, max_iter) * s->nv;
    if (res_linf) ck(cudaMemcpy(res_linf, s->hist_linf, n * sizeof(double), cudaMemcpyDeviceToHost), "history");
    if (res_l2) ck(cudaMemcpy(res_l2, s->hist_l2, n * sizeof(double), cudaMemcpyDeviceToHost), "history");
    float ms = 0.0f;
    ck(cudaEventElapsedTime(&ms, s->ev0, s->ev1), "event time");
    s->last_ms = ms;
    s->last_launches = s->graph_launches[key] * (out.done / chunk);
    s->last_n = 0;  // the per-case residual buffers hold only the last block
    s->iter += out.done;
    return out.done;
}

template <typename R>
void run_profile(psst_solver *s, int n_iter, double *ms, int64_t *cnt) {
    DevWork<R> &w = work<R>(s);
    ensure_norms<R>(s, n_iter);
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    auto mark = [&](int k) {
        cudaEvent_t e;
        ck(cudaEventCreate(&e), "event");
        ck(cudaEventRecord(e, s->stream), "event");
        ev.push_back(e);
        kind.push_back(k);
    };
    mark(-1);
    iterations<R>(s, n_iter, mark);
    ck(cudaGetLastError(), "kernel launch");
    check_err(s, w.err);
    for (int k = 0; k < PSST_KERNEL_KINDS; ++k) {
        ms[k] = 0.0;
        cnt[k] = 0;
    }
    for (size_t i = 1; i < ev.size(); ++i) {
        float t = 0.0f;
        ck(cudaEventElapsedTime(&t, ev[i - 1], ev[i]), "event time");
        ms[kind[i]] += t;
        cnt[kind[i]] += 1;
    }
    for (auto e : ev) cudaEventDestroy(e);
    s->iter += n_iter;
}

// Launch-shape tuner: runs n_iter iterations per candidate block size (two
// sweeps) on the solver's own mesh and state, times each pass with events,
// keeps the fastest shape per pass, and puts the state back (device-to-device snapshot of the
// primitive records and the conservative state; everything else a stage reads
// is recomputed from those), so the solution and the iteration count are
// unchanged. Results do not depend on the shapes except for the rounding of
// the RMS column, whose block partials follow the cell-pass shape.
template <typename R>
void autotune(psst_solver *s, int n_iter, int *blocks) {
    DevState<R> *st = states<R>(s);
    DevWork<R> &w = work<R>(s);
    const size_t rb = (size_t)std::max(s->L.nall, 1) * sizeof(CellRec<R>);
    const size_t wb = (size_t)s->nv * std::max(s->L.nint, 1) * sizeof(double);
    void *snap = nullptr;
    ck(cudaMalloc(&snap, rb + wb), "cudaMalloc");
    const int cur0 = s->cur;
    const int64_t iter0 = s->iter;
    auto copy = [&](bool save) {
        void *r = st[cur0].rec, *ww = w.w, *sr = snap, *sw = (char *)snap + rb;
        ck(cudaMemcpyAsync(save ? sr : r, save ? r : sr, rb, cudaMemcpyDeviceToDevice, s->stream), "snapshot");
        ck(cudaMemcpyAsync(save ? sw : ww, save ? ww : sw, wb, cudaMemcpyDeviceToDevice, s->stream), "snapshot");
    };
    const int cand[3] = {64, 128, 256};
    const int kinds[3] = {K_GRADIENT, K_FACE, K_CELL};
    double best[3] = {1e300, 1e300, 1e300};
    int pick[3] = {s->g.blk_grad, s->g.blk_face, s->g.blk_cell};
    try {
        copy(true);
        // two sweeps in opposite orders; each shape keeps its best time, so a
        // transient (clock ramp, a neighbour's traffic) does not decide
        for (int j = 0; j < 6; ++j) {
            const int b = j < 3 ? cand[j] : cand[5 - j];
            s->g.blk_grad = s->g.blk_face = s->g.blk_cell = b;
            double ms[PSST_KERNEL_KINDS];
            int64_t cnt[PSST_KERNEL_KINDS];
            run_profile<R>(s, 1, ms, cnt);  // warm-up at this shape
            copy(false);
            s->cur = cur0;
            run_profile<R>(s, n_iter, ms, cnt);
            copy(false);
            s->cur = cur0;
            for (int i = 0; i < 3; ++i)
                if (cnt[kinds[i]] > 0 && ms[kinds[i]] / cnt[kinds[i]] < best[i]) {
                    best[i] = ms[kinds[i]] / cnt[kinds[i]];
                    pick[i] = b;
                }
        }
        ck(cudaStreamSynchronize(s->stream), "stream sync");
    } catch (...) {
        cudaMemcpyAsync(st[cur0].rec, snap, rb, cudaMemcpyDeviceToDevice, s->stream);
        cudaMemcpyAsync(w.w, (char *)snap + rb, wb, cudaMemcpyDeviceToDevice, s->stream);
        cudaStreamSynchronize(s->stream);
        cudaFree(snap);
        s->cur = cur0;
        s->iter = iter0;
        throw;
    }
    cudaFree(snap);
    s->iter = iter0;
    s->drop_graphs();
    s->g.blk_grad = pick[0];
    s->g.blk_face = pick[1];
    s->g.blk_cell = pick[2];
    if (blocks)
        for (int i = 0; i < 3; ++i) blocks[i] = pick[i];
}

// Device staging of the reference-ordered state: the host buffers move in one
// contiguous copy each way (DMA straight from pinned memory when the caller's
// buffer is pinned) and the permutation to and from the device layout runs on
// the GPU.
void ensure_staging(psst_solver *s) {
    if (s->d_vol) return;
    std::vector<int32_t> vol(s->L.nall);
    for (int32_t d = 0; d < s->L.nall; ++d) vol[d] = (int32_t)s->L.vol_of_dev[d];
    s->d_vol = s->upload(vol);
    s->d_prim = s->dalloc<double>((size_t)(2 + s->dim) * s->nvol_ref);
    s->d_w = s->dalloc<double>((size_t)s->nv * s->nvol_ref);
    s->d_rho = s->dalloc<double>((size_t)s->nvol_ref);
}

template <typename R>
void set_state(psst_solver *s, const double *prim) {
    ensure_staging(s);
    const size_t bytes = (size_t)(2 + s->dim) * s->nvol_ref * sizeof(double);
    ck(cudaMemcpyAsync(s->d_prim, prim, bytes, cudaMemcpyHostToDevice, s->stream), "state upload");
    DevState<R> &st = states<R>(s)[s->cur];
    Ops<R>::gather_prim(s->dim, s->g, st, s->d_prim, s->d_vol, s->nvol_ref, s->stream);
    Ops<R>::prologue(s->dim, s->g, st, work<R>(s), s->gas, s->stream);
    ck(cudaGetLastError(), "prologue");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
}

template <typename R>
void get_state(psst_solver *s, double *prim, double *wout) {
    ensure_staging(s);
    const int64_t nv = s->nvol_ref;
    if (prim) {
        const size_t bytes = (size_t)(2 + s->dim) * nv * sizeof(double);
        ck(cudaMemsetAsync(s->d_prim, 0, bytes, s->stream), "memset");
        Ops<R>::scatter_prim(s->dim, s->g, states<R>(s)[s->cur], s->d_prim, s->d_vol, nv, s->stream);
        ck(cudaMemcpyAsync(prim, s->d_prim, bytes, cudaMemcpyDeviceToHost, s->stream), "state copy");
    }
    if (wout) {
        const size_t bytes = (size_t)s->nv * nv * sizeof(double);
        ck(cudaMemsetAsync(s->d_w, 0, bytes, s->stream), "memset");
        Ops<R>::scatter_w(s->dim, s->g, work<R>(s), s->d_w, s->d_vol, s->stream);
        ck(cudaMemcpyAsync(wout, s->d_w, bytes, cudaMemcpyDeviceToHost, s->stream), "state copy");
    }
    ck(cudaGetLastError(), "state scatter");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
}

// Binary checkpoint: everything an iteration boundary carries, at full
// precision -- the primitive records (p, T, rho, u..) of every volume as the
// solver holds them and the FP64 conservative state w -- plus the iteration
// counter. (The reference's .sav keeps 11 decimals of p, T, u and recomputes
// rho and w on load, psstFiniteVolumeGrid.cpp:559-639, 279-300, so a restart
// from it does not continue the run exactly.)
struct CkptHeader {
    char magic[8];
    int32_t dim, precision;
    int64_t nvol, nint, iter;
};
constexpr char kCkptMagic[8] = {'P', 'S', 'S', 'T', 'C', 'K', 'P', '1'};

template <typename R>
void save_checkpoint(psst_solver *s, const char *path) {
    const int64_t nv = s->nvol_ref;
    std::vector<double> prim((size_t)(2 + s->dim) * nv), w((size_t)s->nv * nv), rho(nv);
    get_state<R>(s, prim.data(), w.data());
    {
        std::vector<CellRec<R>> h(s->L.nall);
        ck(cudaMemcpyAsync(h.data(), states<R>(s)[s->cur].rec, h.size() * sizeof(CellRec<R>),
                           cudaMemcpyDeviceToHost, s->stream),
           "copy");
        ck(cudaStreamSynchronize(s->stream), "stream sync");
        for (int32_t d = 0; d < s->L.nall; ++d) rho[s->L.vol_of_dev[d]] = (double)h[d].v[RRHO];
    }
    CkptHeader h{};
    std::memcpy(h.magic, kCkptMagic, 8);
    h.dim = s->dim;
    h.precision = s->sc.precision;
    h.nvol = nv;
    h.nint = s->L.nint;
    h.iter = s->iter;
    FILE *f = std::fopen(path, "wb");
    if (!f) raise(PSST_ERR_IO, std::string("cannot write ") + path);
    bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 &&
              std::fwrite(prim.data(), sizeof(double), prim.size(), f) == prim.size() &&
              std::fwrite(rho.data(), sizeof(double), rho.size(), f) == rho.size() &&
              std::fwrite(w.data(), sizeof(double), w.size(), f) == w.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) raise(PSST_ERR_IO, std::string("cannot write ") + path);
}

template <typename R>
void load_checkpoint(psst_solver *s, const char *path) {
    FILE *f = std::fopen(path, "rb");
    if (!f) raise(PSST_ERR_IO, std::string("cannot read ") + path);
    CkptHeader h{};
    const int64_t nv = s->nvol_ref;
    std::vector<double> prim((size_t)(2 + s->dim) * nv), w((size_t)s->nv * nv), rho(nv);
    bool ok = std::fread(&h, sizeof h, 1, f) == 1 && std::memcmp(h.magic, kCkptMagic, 8) == 0;
    const bool match = ok && h.dim == s->dim && h.nvol == nv && h.nint == s->L.nint;
    ok = match && h.precision == s->sc.precision &&
         std::fread(prim.data(), sizeof(double), prim.size(), f) == prim.size() &&
         std::fread(rho.data(), sizeof(double), rho.size(), f) == rho.size() &&
         std::fread(w.data(), sizeof(double), w.size(), f) == w.size();
    std::fclose(f);
    if (!match) raise(PSST_ERR_FORMAT, std::string(path) + ": not a checkpoint of this grid");
    if (!ok) raise(PSST_ERR_FORMAT, std::string(path) + ": truncated, or written at another precision");
    ensure_staging(s);
    ck(cudaMemcpyAsync(s->d_prim, prim.data(), prim.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream),
       "state upload");
    ck(cudaMemcpyAsync(s->d_rho, rho.data(), rho.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream),
       "state upload");
    ck(cudaMemcpyAsync(s->d_w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream),
       "state upload");
    Ops<R>::set_exact(s->dim, s->g, states<R>(s)[s->cur], work<R>(s), s->d_prim, s->d_rho, s->d_w, s->d_vol, nv,
                      s->stream);
    ck(cudaGetLastError(), "checkpoint state");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    s->iter = h.iter;
}

template <typename R, int DIM>
void grad_array(psst_solver *s, const std::string &nm, double *out) {
    const int32_t nint = s->L.nint;
    std::vector<GradRec<R, DIM>> h(nint);
    ck(cudaMemcpyAsync(h.data(), work<R>(s).grec, (size_t)nint * sizeof(GradRec<R, DIM>), cudaMemcpyDeviceToHost,
                       s->stream),
       "array copy");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    for (int32_t d = 0; d < nint; ++d) {
        const int64_t v = s->L.vol_of_dev[d];
        if (nm == "grad_u") {
            for (int j = 0; j < DIM * DIM; ++j) out[v * DIM * DIM + j] = (double)h[d].g[j];
        } else {
            const int var = nm == "grad_p" ? DIM : DIM + 1;
            for (int k = 0; k < DIM; ++k) out[v * DIM + k] = (double)h[d].g[var * DIM + k];
        }
    }
}

template <typename R>
void get_array(psst_solver *s, const std::string &nm, double *out, int64_t count) {
    const int dim = s->dim, nvv = s->nv;
    const int64_t nv = s->nvol_ref;
    const int32_t nint = s->L.nint;
    DevWork<R> &w = work<R>(s);
    auto need = [&](int64_t n) {
        if (n != count) raise(PSST_ERR_ARG, nm + ": expected " + std::to_string(n) + " elements");
        std::fill(out, out + n, 0.0);
    };
    if (nm == "rho") {  // density of every volume (ghosts included), as the state records hold it
        need(nv);
        std::vector<CellRec<R>> h(s->L.nall);
        ck(cudaMemcpyAsync(h.data(), states<R>(s)[s->cur].rec, h.size() * sizeof(CellRec<R>), cudaMemcpyDeviceToHost,
                           s->stream),
           "copy");
        ck(cudaStreamSynchronize(s->stream), "stream sync");
        for (int32_t d = 0; d < s->L.nall; ++d) out[s->L.vol_of_dev[d]] = (double)h[d].v[RRHO];
        return;
    }
    if (nm == "dt") {
        need(nv);
        std::vector<double> h(nint);
        ck(cudaMemcpyAsync(h.data(), w.dt, (size_t)nint * sizeof(double), cudaMemcpyDeviceToHost, s->stream), "copy");
        ck(cudaStreamSynchronize(s->stream), "stream sync");
        for (int32_t d = 0; d < nint; ++d) out[s->L.vol_of_dev[d]] = h[d];
        return;
    }
    if (nm == "residual") {
        need((int64_t)nvv * nv);
        std::vector<R> h((size_t)nvv * nint);
        ck(cudaMemcpyAsync(h.data(), w.res, h.size() * sizeof(R), cudaMemcpyDeviceToHost, s->stream), "copy");
        ck(cudaStreamSynchronize(s->stream), "stream sync");
        for (int32_t d = 0; d < nint; ++d)
            for (int q = 0; q < nvv; ++q) out[s->L.vol_of_dev[d] * nvv + q] = (double)h[(size_t)q * nint + d];
        return;
    }
    int64_t width;
    if (nm == "grad_u")
        width = (int64_t)dim * dim;
    else if (nm == "grad_p" || nm == "grad_T")
        width = dim;
    else
        raise(PSST_ERR_ARG, "unknown solver array " + nm);
    need(width * nv);
    if (dim == 2)
        grad_array<R, 2>(s, nm, out);
    else
        grad_array<R, 3>(s, nm, out);
}

template <typename R>
void stage_api(psst_solver *s, int k, double *res_linf) {
    ensure_norms<R>(s, 1);
    one_stage<R>(s, k, 0, false, [](int) {});
    std::vector<double> li(s->nv);
    ck(cudaMemcpyAsync(li.data(), work<R>(s).linf, li.size() * sizeof(double), cudaMemcpyDeviceToHost, s->stream),
       "norm copy");
    check_err(s, work<R>(s).err);
    if (res_linf) std::memcpy(res_linf, li.data(), li.size() * sizeof(double));
}

}  // namespace

#define PSST_API_BEGIN try {
#define PSST_API_END                          \
    return PSST_OK;                           \
    }                                         \
    catch (const Error &e) {                  \
        set_last_error(e.msg);                \
        return e.status;                      \
    }                                         \
    catch (const std::bad_alloc &) {          \
        set_last_error("out of host memory"); \
        return PSST_ERR_ARG;                  \
    }                                         \
    catch (const std::exception &e) {         \
        set_last_error(e.what());             \
        return PSST_ERR_ARG;                  \
    }

#define DISPATCH(s, call) ((s)->sc.precision == 32 ? call<float> : call<double>)

extern "C" psst_status psst_solver_create(const psst_grid *G, const psst_scheme *sc, int device, psst_solver **out) {
    PSST_API_BEGIN
    if (!G || !sc || !out) raise(PSST_ERR_ARG, "psst_solver_create: null argument");
    *out = nullptr;
    if (sc->precision != 64 && sc->precision != 32) raise(PSST_ERR_ARG, "precision must be 64 or 32");
    if (sc->flux < 1 || sc->flux > 3) raise(PSST_ERR_ARG, "Error: Unknow convective flow scheme!");
    if (sc->order != 1 && sc->order != 2) raise(PSST_ERR_ARG, "Error! Unknown scheme order!");
    if (sc->order == 2 && (sc->limiter < 1 || sc->limiter > 5))
        raise(PSST_ERR_ARG, "second order needs a limiter (1 VanAlbada, 2 MinMod, 3 VanLeer, 4 BJ, 5 Venkatakrishnan)");
    if (sc->lc < 0 || sc->lc > 2) raise(PSST_ERR_ARG, "unknown local time step mode");
    if (sc->rk_level < 1 || sc->rk_level > 16) raise(PSST_ERR_ARG, "Error: Unknow RK order!");
    if (sc->order == 2 && sc->grad != 1 && G->case_vol_ptr.size() > 2)
        raise(PSST_ERR_UNSUPPORTED, "merged grids need Green-Gauss gradients (the least-squares table is "
                                    "indexed across zones, psstGradCalculation.cpp:404-412)");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        raise(PSST_ERR_CUDA, "no CUDA device available (libpsst_b200 has no CPU fallback)");
    if (device < 0 || device >= ndev) raise(PSST_ERR_ARG, "invalid device index");
    std::unique_ptr<psst_solver> s(new psst_solver);
    s->device = device;
    ck(cudaSetDevice(device), "cudaSetDevice");
    s->dim = G->dim;
    s->nv = G->dim + 2;
    s->sc = *sc;
    s->gas = Gas{sc->rm, sc->cp, sc->cv, sc->gamma};
    s->nvol_ref = G->nvol;
    s->iter = sc->iter > 0 ? sc->iter : 1;
    s->rec = sc->order == 1 ? 0 : (sc->limiter >= 4 ? 2 : 1);
    s->celllim = (sc->order == 2 && sc->limiter >= 4) ? sc->limiter : 0;
    s->seq = sc->lc == 1 && sc->lc1_mode == PSST_LC1_SEQUENTIAL;
    if (sc->lc == 0)
        s->dt_uniform = G->dim == 2 ? sc->cfl * std::sqrt(G->min_vol) / sc->ref_vel
                                    : sc->cfl * std::pow(G->min_vol, 1.0 / 3.0) / sc->ref_vel;
    build_layout(*G, *sc, s->L);
    Layout &L = s->L;
    s->nblk = nblocks(L.nint);
    ck(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking), "stream");
    s->stream = s->own_stream;
    ck(cudaEventCreate(&s->ev0), "event");
    ck(cudaEventCreate(&s->ev1), "event");
    DevGrid &g = s->g;
    g.nint = L.nint;
    g.nghost = L.nghost;
    g.nall = L.nall;
    g.nface = L.nface;
    g.nfi = L.nfi;
    g.kuni = 0;
    if (L.nint > 0) {
        const int32_t k0 = L.csr_ptr[1] - L.csr_ptr[0];
        bool uni = true;
        for (int32_t d = 0; d < L.nint && uni; ++d) uni = L.csr_ptr[d + 1] - L.csr_ptr[d] == k0;
        g.kuni = uni ? k0 : 0;
    }
    g.beta = s->upload(L.beta);
    g.V = s->upload(L.V);
    g.xc = s->upload(L.xc);
    g.csr_ptr = s->upload(L.csr_ptr);
    g.csr_ent = s->upload(L.csr_ent);
    g.csr_nb = s->upload(L.csr_nb);
    g.wperm = s->upload(L.wperm);
    g.lsq_r = s->upload(L.lsq_r);
    g.vk_eps2 = s->upload(L.vk_eps2);
    g.rank = s->upload(L.rank);
    g.gptr = s->upload(L.gptr);
    g.g_nb = s->upload(L.g_nb);
    g.g_face = s->upload(L.g_face);
    g.g_zone = s->upload(L.g_zone);
    g.z_dyn = s->upload(L.z_dyn);
    g.z_therm = s->upload(L.z_therm);
    g.z_u = s->upload(L.z_u);
    g.z_p = s->upload(L.z_p);
    g.z_T = s->upload(L.z_T);
    g.lvl_cells = s->upload(L.lvl_cells);
    g.lvl_ptr = s->upload(L.lvl_ptr);
    g.nlevels = L.nlevels;
    g.blk_grad = g.blk_face = g.blk_cell = kBlock;
    g.ncase = L.ncase;
    if (!L.cell_case.empty()) {
        if (s->seq)
            raise(PSST_ERR_UNSUPPORTED, "merged grids run LocalAccTime1 from stage-start values only (lc1_mode 1)");
        g.cell_case = s->upload(L.cell_case);
        std::vector<int32_t> fc(L.nface);
        for (int32_t f = 0; f < L.nface; ++f) fc[f] = L.cell_case[L.c0[f]];
        g.face_case = s->upload(fc);
        s->active_h.assign(L.ncase, 1);
        g.case_active = s->upload(s->active_h);
    }
    if (sc->precision == 32)
        alloc_state<float>(s.get(), *G);
    else
        alloc_state<double>(s.get(), *G);
    if (s->seq && sc->precision == 64 && L.cell_case.empty() && !L.wf_item_level.empty()) {
        const int maxb = Ops<double>::wavefront_max_blocks(s->dim, s->rec, sc->limiter);
        // CTA 0 folds the norms; the others take the work items of a step
        s->wf_blocks = std::min(L.wf_max_class_items + 1, maxb);
        if (s->wf_blocks >= 2) {  // the items need a CTA besides CTA 0
            WfSched &w = s->wf;
            w.period = L.wf_period;
            w.nlevels = L.nlevels;
            w.nitems = (int32_t)L.wf_item_level.size();
            w.cells32 = s->upload(L.wf_cells32);
            w.lowmask = s->upload(L.wf_lowmask);
            w.item_level = s->upload(L.wf_item_level);
            w.lvl_items = s->upload(L.wf_lvl_items);
            w.ipart = s->dalloc<double>((size_t)2 * w.nitems * 2 * s->nv);
            w.nacc = L.nlevels / L.wf_period + 3;
            w.acc = s->dalloc<double>((size_t)w.nacc * 2 * s->nv);
            w.grec2 = s->dalloc_bytes(Ops<double>::grad_rec_bytes(s->dim) * std::max(L.nint, 1));
            ck(cudaMemset(w.grec2, 0, Ops<double>::grad_rec_bytes(s->dim) * std::max(L.nint, 1)), "memset");
            w.sync = s->dalloc<unsigned>(kWfSyncWords);
            s->wf_ready = true;
        }
    }
    ck(cudaDeviceSynchronize(), "setup");
    *out = s.release();
    PSST_API_END
}

extern "C" psst_status psst_solver_set_state(psst_solver *s, const double *prim) {
    PSST_API_BEGIN
    if (!s || !prim) raise(PSST_ERR_ARG, "psst_solver_set_state: null argument");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, set_state)(s, prim);
    s->has_state = true;
    PSST_API_END
}

extern "C" psst_status psst_solver_get_state(psst_solver *s, double *prim, double *w) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "psst_solver_get_state: null argument");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, get_state)(s, prim, w);
    PSST_API_END
}

extern "C" psst_status psst_solver_save_checkpoint(psst_solver *s, const char *path) {
    PSST_API_BEGIN
    if (!s || !path) raise(PSST_ERR_ARG, "psst_solver_save_checkpoint: null argument");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, save_checkpoint)(s, path);
    PSST_API_END
}

extern "C" psst_status psst_solver_load_checkpoint(psst_solver *s, const char *path) {
    PSST_API_BEGIN
    if (!s || !path) raise(PSST_ERR_ARG, "psst_solver_load_checkpoint: null argument");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, load_checkpoint)(s, path);
    s->has_state = true;
    PSST_API_END
}

extern "C" psst_status psst_gradient_calculate(psst_solver *s) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    if (s->sc.precision == 32)
        Ops<float>::gradient(s->dim, s->sc.grad, s->celllim, s->g, s->s32[s->cur], s->w32, s->stream);
    else
        Ops<double>::gradient(s->dim, s->sc.grad, s->celllim, s->g, s->s64[s->cur], s->w64, s->stream);
    ck(cudaGetLastError(), "gradient");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    PSST_API_END
}

extern "C" psst_status psst_convective_calculate(psst_solver *s) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    if (s->sc.precision == 32) {
        Ops<float>::face(s->dim, s->sc.flux, s->rec, s->sc.limiter, 0, s->g, s->s32[s->cur], s->w32, s->gas,
                         s->stream);
        Ops<float>::residual(s->dim, s->g, s->w32, s->stream);
        ck(cudaGetLastError(), "convective");
        check_err(s, s->w32.err);
    } else {
        Ops<double>::face(s->dim, s->sc.flux, s->rec, s->sc.limiter, 0, s->g, s->s64[s->cur], s->w64, s->gas,
                          s->stream);
        Ops<double>::residual(s->dim, s->g, s->w64, s->stream);
        ck(cudaGetLastError(), "convective");
        check_err(s, s->w64.err);
    }
    PSST_API_END
}

extern "C" psst_status psst_stage_update(psst_solver *s, int k, double *res_linf) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    if (k < 0 || k >= s->sc.rk_level) raise(PSST_ERR_ARG, "RK stage out of range");
    if (!s->L.cell_case.empty()) raise(PSST_ERR_UNSUPPORTED, "merged grids advance through psst_explicit_solve only");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, stage_api)(s, k, res_linf);
    PSST_API_END
}

extern "C" psst_status psst_explicit_solve(psst_solver *s, int n_iter, double *res_linf, double *res_l2) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    if (n_iter < 0) raise(PSST_ERR_ARG, "n_iter must be non-negative");
    if (n_iter == 0) return PSST_OK;
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, run)(s, n_iter, res_linf, res_l2);
    PSST_API_END
}

extern "C" psst_status psst_solver_run_to_stop(psst_solver *s, int64_t max_iter, int chunk, int64_t *iterations,
                                               double *res_linf, double *res_l2) {
    PSST_API_BEGIN
    if (!s || !iterations) raise(PSST_ERR_ARG, "psst_solver_run_to_stop: null argument");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    if (max_iter < 1 || chunk < 1) raise(PSST_ERR_ARG, "psst_solver_run_to_stop: max_iter and chunk must be >= 1");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    *iterations = DISPATCH(s, run_to_stop)(s, max_iter, chunk, res_linf, res_l2);
    PSST_API_END
}

extern "C" psst_status psst_solver_get_array(psst_solver *s, const char *name, double *out, int64_t count) {
    PSST_API_BEGIN
    if (!s || !name || !out) raise(PSST_ERR_ARG, "psst_solver_get_array: null argument");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, get_array)(s, std::string(name), out, count);
    PSST_API_END
}

extern "C" psst_status psst_solver_set_stream(psst_solver *s, void *stream) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    s->stream = stream ? (cudaStream_t)stream : s->own_stream;
    PSST_API_END
}

extern "C" psst_status psst_solver_last_stats(const psst_solver *s, int64_t *launches, double *device_ms) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (launches) *launches = s->last_launches;
    if (device_ms) *device_ms = s->last_ms;
    PSST_API_END
}

extern "C" psst_status psst_solver_profile(psst_solver *s, int n_iter, double *ms_per_kind, int64_t *launches_per_kind) {
    PSST_API_BEGIN
    if (!s || !ms_per_kind || !launches_per_kind) raise(PSST_ERR_ARG, "psst_solver_profile: null argument");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    if (n_iter <= 0) raise(PSST_ERR_ARG, "n_iter must be positive");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, run_profile)(s, n_iter, ms_per_kind, launches_per_kind);
    PSST_API_END
}

extern "C" psst_status psst_solver_autotune(psst_solver *s, int n_iter, int *blocks) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (!s->has_state) raise(PSST_ERR_STATE, "no state set");
    if (n_iter <= 0) raise(PSST_ERR_ARG, "n_iter must be positive");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    DISPATCH(s, autotune)(s, n_iter, blocks);
    PSST_API_END
}

extern "C" psst_status psst_solver_launch_shape(psst_solver *s, const int *set, int *get) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (set) {
        for (int i = 0; i < 3; ++i)
            if (set[i] != 0 && set[i] != 64 && set[i] != 128 && set[i] != 256)
                raise(PSST_ERR_ARG, "launch shape must be 0 (keep), 64, 128 or 256 threads per block");
        s->drop_graphs();
        if (set[0]) s->g.blk_grad = set[0];
        if (set[1]) s->g.blk_face = set[1];
        if (set[2]) s->g.blk_cell = set[2];
    }
    if (get) {
        get[0] = s->g.blk_grad;
        get[1] = s->g.blk_face;
        get[2] = s->g.blk_cell;
    }
    PSST_API_END
}

extern "C" psst_status psst_solver_use_graphs(psst_solver *s, int on) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    if (!on) s->drop_graphs();
    s->use_graphs = on != 0;
    PSST_API_END
}

extern "C" psst_status psst_solver_set_active(psst_solver *s, const int32_t *active) {
    PSST_API_BEGIN
    if (!s || !active) raise(PSST_ERR_ARG, "psst_solver_set_active: null argument");
    if (s->L.cell_case.empty()) raise(PSST_ERR_ARG, "psst_solver_set_active: the grid is not a merged grid");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    for (int32_t i = 0; i < s->L.ncase; ++i) s->active_h[i] = active[i] ? 1 : 0;
    ck(cudaMemcpyAsync((void *)s->g.case_active, s->active_h.data(), s->active_h.size() * sizeof(int32_t),
                       cudaMemcpyHostToDevice, s->stream),
       "flags upload");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    PSST_API_END
}

extern "C" psst_status psst_solver_set_stop_rule(psst_solver *s, double drop, int32_t scale_iters,
                                                 const double *scales, const int32_t *caps) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (s->L.cell_case.empty()) raise(PSST_ERR_ARG, "psst_solver_set_stop_rule: the grid is not a merged grid");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    s->drop_graphs();  // the launch sequence changes
    const int32_t nc = s->L.ncase;
    if (!(drop > 0.0)) {
        s->stop_on = false;
        return PSST_OK;
    }
    if (!scales && scale_iters < 1) raise(PSST_ERR_ARG, "scale_iters must be >= 1 without given scales");
    if (!s->stop.rows) {
        s->stop.rows = s->dalloc<int32_t>(nc);
        s->stop.conv_at = s->dalloc<int32_t>(nc);
        s->stop.cap = s->dalloc<int32_t>(nc);
        s->stop.scale = s->dalloc<double>((size_t)nc * s->nv);
    }
    s->stop.drop = drop;
    s->stop.scale_iters = scales ? 0 : scale_iters;
    s->stop.active = const_cast<int32_t *>(s->g.case_active);
    std::vector<int32_t> cap(nc, INT32_MAX), zero(nc, 0);
    if (caps)
        for (int32_t i = 0; i < nc; ++i) cap[i] = caps[i];
    std::vector<double> sc((size_t)nc * s->nv, 0.0);
    if (scales) std::copy(scales, scales + (size_t)nc * s->nv, sc.begin());
    for (int32_t i = 0; i < nc; ++i) s->active_h[i] = cap[i] > 0 ? 1 : 0;
    ck(cudaMemcpyAsync(const_cast<int32_t *>(s->stop.cap), cap.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice,
                       s->stream),
       "copy");
    ck(cudaMemcpyAsync(s->stop.rows, zero.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream), "copy");
    ck(cudaMemcpyAsync(s->stop.conv_at, zero.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice, s->stream),
       "copy");
    ck(cudaMemcpyAsync(s->stop.scale, sc.data(), sc.size() * sizeof(double), cudaMemcpyHostToDevice, s->stream),
       "copy");
    ck(cudaMemcpyAsync((void *)s->g.case_active, s->active_h.data(), nc * sizeof(int32_t), cudaMemcpyHostToDevice,
                       s->stream),
       "copy");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    s->stop_on = true;
    PSST_API_END
}

extern "C" psst_status psst_solver_case_status(psst_solver *s, int32_t *active, int32_t *iterations,
                                               int32_t *converged_at, double *scales) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    if (s->L.cell_case.empty()) raise(PSST_ERR_ARG, "psst_solver_case_status: the grid is not a merged grid");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    const int32_t nc = s->L.ncase;
    auto get = [&](void *dst, const void *src, size_t bytes) {
        if (dst && src) ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream), "copy");
    };
    get(active, s->g.case_active, nc * sizeof(int32_t));
    get(iterations, s->stop.rows, nc * sizeof(int32_t));
    get(converged_at, s->stop.conv_at, nc * sizeof(int32_t));
    get(scales, s->stop.scale, (size_t)nc * s->nv * sizeof(double));
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    if (!s->stop.rows) {  // no rule set yet: nothing run under it
        if (iterations) std::fill(iterations, iterations + nc, 0);
        if (converged_at) std::fill(converged_at, converged_at + nc, 0);
        if (scales) std::fill(scales, scales + (size_t)nc * s->nv, 0.0);
    }
    if (active)
        for (int32_t i = 0; i < nc; ++i) s->active_h[i] = active[i];
    PSST_API_END
}

extern "C" psst_status psst_solver_case_residuals(psst_solver *s, int n_iter, double *out) {
    PSST_API_BEGIN
    if (!s || !out) raise(PSST_ERR_ARG, "psst_solver_case_residuals: null argument");
    if (s->L.cell_case.empty()) raise(PSST_ERR_ARG, "psst_solver_case_residuals: the grid is not a merged grid");
    if (n_iter <= 0 || n_iter > s->last_n)
        raise(PSST_ERR_ARG, "psst_solver_case_residuals: n_iter exceeds the last psst_explicit_solve call");
    ck(cudaSetDevice(s->device), "cudaSetDevice");
    const size_t cnt = (size_t)n_iter * s->L.ncase * s->nv;
    std::vector<unsigned long long> h(cnt);
    const unsigned long long *src = s->sc.precision == 32 ? s->w32.case_linf : s->w64.case_linf;
    ck(cudaMemcpyAsync(h.data(), src, cnt * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s->stream),
       "norm copy");
    ck(cudaStreamSynchronize(s->stream), "stream sync");
    for (size_t i = 0; i < cnt; ++i) std::memcpy(out + i, &h[i], sizeof(double));
    PSST_API_END
}

extern "C" psst_status psst_solver_use_wavefront(psst_solver *s, int on) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    s->wf_on = on != 0;
    PSST_API_END
}

extern "C" psst_status psst_solver_set_wait_limit(psst_solver *s, int64_t ns) {
    PSST_API_BEGIN
    if (!s) raise(PSST_ERR_ARG, "null solver");
    s->wait_ns = ns < 0 ? psst_solver::kDefaultWaitNs : (uint64_t)ns;
    PSST_API_END
}

extern "C" psst_status psst_solver_schedule_info(const psst_solver *s, int64_t *info) {
    PSST_API_BEGIN
    if (!s || !info) raise(PSST_ERR_ARG, "psst_solver_schedule_info: null argument");
    info[0] = wavefront_active(s) ? 1 : 0;
    info[1] = s->L.wf_period;
    info[2] = s->L.nlevels;
    info[3] = (int64_t)s->L.wf_item_level.size();
    info[4] = s->wf_blocks;
    PSST_API_END
}

extern "C" int64_t psst_solver_iter(const psst_solver *s) { return s ? s->iter : -1; }

extern "C" void psst_solver_destroy(psst_solver *s) { delete s; }
