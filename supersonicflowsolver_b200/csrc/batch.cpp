// Batched cases: one grid that is the disjoint union of several case grids,
// so that every kernel launch advances all cases at once.
//
// Volumes, faces and zones are the cases' own, case after case, each case in
// its reference storage order; zone id z of case i becomes i * kZoneStride + z
// (so ascending zone ids keep case-major order) and its name gets "#i". Every
// per-case table the solver reads (geometry, the Green-Gauss beta table with
// its zone-index quirk, boundary values, the initial state) is the case's own,
// so each case evolves exactly as it would alone; only tables that the
// reference indexes across zones (2D least squares) cannot be merged.
#include <algorithm>
#include <memory>
#include <string>

#include "host.hpp"

using namespace psst;

namespace {

constexpr int64_t kZoneStride = 1000000;

psst_grid *merge(const psst_grid *const *gs, int32_t n) {
    std::unique_ptr<psst_grid> m(new psst_grid);
    const int dim = gs[0]->dim;
    m->dim = dim;
    m->case_vol_ptr.push_back(0);
    bool have_prim = true;
    for (int32_t i = 0; i < n; ++i) have_prim = have_prim && (int64_t)gs[i]->prim0.size() == (2 + dim) * gs[i]->nvol;
    for (int32_t i = 0; i < n; ++i) {
        const psst_grid &g = *gs[i];
        if (g.dim != dim) raise(PSST_ERR_ARG, "psst_grid_merge: cases of different dimension");
        if (!g.case_vol_ptr.empty()) raise(PSST_ERR_ARG, "psst_grid_merge: a case is itself a merged grid");
        for (auto &z : g.vz)
            if (z.id >= kZoneStride) raise(PSST_ERR_ARG, "psst_grid_merge: zone id too large");
        const int64_t v0 = m->nvol, f0 = m->nface, e0 = (int64_t)m->vf_idx.size();
        const int32_t vzs = (int32_t)m->vz.size(), fzs = (int32_t)m->fz.size();
        for (auto z : g.vz) {
            z.id += i * kZoneStride;
            z.first += v0;
            z.name += "#" + std::to_string(i);
            m->vz.push_back(z);
        }
        for (auto z : g.fz) {
            z.id += i * kZoneStride;
            z.first += f0;
            z.name += "#" + std::to_string(i);
            m->fz.push_back(z);
        }
        m->vol_boundary.insert(m->vol_boundary.end(), g.vol_boundary.begin(), g.vol_boundary.end());
        for (int32_t s : g.vol_vz) m->vol_vz.push_back(s + vzs);
        if (m->vf_ptr.empty()) m->vf_ptr.push_back(0);
        for (int64_t v = 0; v < g.nvol; ++v) m->vf_ptr.push_back(e0 + g.vf_ptr[v + 1]);
        for (int64_t f : g.vf_idx) m->vf_idx.push_back(f + f0);
        m->V.insert(m->V.end(), g.V.begin(), g.V.end());
        m->xc.insert(m->xc.end(), g.xc.begin(), g.xc.end());
        for (int64_t c : g.f_c0) m->f_c0.push_back(c < 0 ? -1 : c + v0);
        for (int64_t c : g.f_c1) m->f_c1.push_back(c < 0 ? -1 : c + v0);
        for (int32_t s : g.f_fz) m->f_fz.push_back(s + fzs);
        m->S.insert(m->S.end(), g.S.begin(), g.S.end());
        m->n.insert(m->n.end(), g.n.begin(), g.n.end());
        m->xf.insert(m->xf.end(), g.xf.begin(), g.xf.end());
        m->beta.insert(m->beta.end(), g.beta.begin(), g.beta.end());
        m->nvol += g.nvol;
        m->nface += g.nface;
        m->ninterior += g.ninterior;
        m->nghost += g.nghost;
        m->max_faces = std::max(m->max_faces, g.max_faces);
        if (g.min_vol >= 0.0 && (m->min_vol < 0.0 || g.min_vol < m->min_vol)) m->min_vol = g.min_vol;
        m->ref_vel = std::max(m->ref_vel, g.ref_vel);
        m->case_vol_ptr.push_back(m->nvol);
    }
    if (have_prim) {
        m->prim0.assign((size_t)(2 + dim) * m->nvol, 0.0);
        for (int32_t i = 0; i < n; ++i) {
            const psst_grid &g = *gs[i];
            const int64_t v0 = m->case_vol_ptr[i];
            for (int q = 0; q < 2 + dim; ++q)
                std::copy(g.prim0.begin() + q * g.nvol, g.prim0.begin() + (q + 1) * g.nvol,
                          m->prim0.begin() + q * m->nvol + v0);
        }
    }
    return m.release();
}

}  // namespace

extern "C" psst_status psst_grid_merge(const psst_grid *const *grids, int32_t n, psst_grid **out) {
    try {
        if (!grids || !out || n <= 0) raise(PSST_ERR_ARG, "psst_grid_merge: null argument or no case");
        for (int32_t i = 0; i < n; ++i)
            if (!grids[i]) raise(PSST_ERR_ARG, "psst_grid_merge: null grid");
        *out = merge(grids, n);
        return PSST_OK;
    } catch (const Error &e) {
        set_last_error(e.msg);
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("out of host memory");
        return PSST_ERR_ARG;
    }
}

extern "C" psst_status psst_grid_initial_state(const psst_grid *g, double *prim, int64_t count) {
    if (!g || !prim) {
        set_last_error("psst_grid_initial_state: null argument");
        return PSST_ERR_ARG;
    }
    if ((int64_t)g->prim0.size() != count || count != (2 + g->dim) * g->nvol) {
        set_last_error("psst_grid_initial_state: no initial state of " + std::to_string(count) + " values");
        return PSST_ERR_STATE;
    }
    std::copy(g->prim0.begin(), g->prim0.end(), prim);
    return PSST_OK;
}

extern "C" psst_status psst_grid_case_count(const psst_grid *g, int32_t *ncase, int64_t *case_vol_ptr) {
    if (!g || !ncase) {
        set_last_error("psst_grid_case_count: null argument");
        return PSST_ERR_ARG;
    }
    *ncase = g->case_vol_ptr.empty() ? 1 : (int32_t)g->case_vol_ptr.size() - 1;
    if (case_vol_ptr) {
        if (g->case_vol_ptr.empty()) {
            case_vol_ptr[0] = 0;
            case_vol_ptr[1] = g->nvol;
        } else {
            std::copy(g->case_vol_ptr.begin(), g->case_vol_ptr.end(), case_vol_ptr);
        }
    }
    return PSST_OK;
}
