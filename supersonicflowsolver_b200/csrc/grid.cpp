// Finite-volume grid construction and FP64 geometry (host, once per mesh).
//
// Follows psstAnsysInputGrid::create_finite_volume_grid
// (psstAnsysGridReader.cpp:688-907): one ghost volume per boundary face, faces
// wired to volumes zone by zone in file order (which fixes each volume's face
// order), then psstFace::initialize and psstVolume::initialize
// (psstFiniteVolumeGridTools.cpp:397-505, 709-827). The geometry formulas keep
// the reference's operand order so that areas, normals, centroids and volumes
// are bit-identical; every later parity claim rests on that.
#include <algorithm>
#include <cmath>
#include <map>
#include <memory>

#include "host.hpp"

namespace psst {

namespace {

void face_geometry(psst_grid &g, const RawMesh &m, int64_t f, int64_t loc) {
    const int dim = g.dim;
    const int64_t nv = m.face_ptr[loc + 1] - m.face_ptr[loc];
    const int64_t *nodes = &m.face_nodes[m.face_ptr[loc]];
    auto V = [&](int64_t k) { return &m.verts[(nodes[k] - 1) * dim]; };
    double sq = 0.0, nn[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    if (dim == 2) {
        if (nv != 2) raise(PSST_ERR_FORMAT, "Error: Expected to vertices but extra data found!");
        const double *v0 = V(0), *v1 = V(1);
        for (int i = 0; i < 2; ++i) {
            c[i] = 0.5 * (v1[i] + v0[i]);
            double comp = v1[i] - v0[i];
            sq += comp * comp;
        }
        sq = std::sqrt(sq);
        nn[0] = v0[1] - v1[1];
        nn[1] = v1[0] - v0[0];
    } else {
        if (nv < 3) raise(PSST_ERR_FORMAT, "Error: Expected at least 3 vertices!");
        double avg[3] = {0, 0, 0}, avg3[3];
        for (int i = 0; i < 3; ++i) {
            for (int64_t j = 0; j < nv; ++j) avg[i] += V(j)[i];
            avg[i] /= (double)nv;
            avg3[i] = avg[i] * 3;
        }
        double a[3], b[3], cc[3], ts;
        const int64_t last = nv - 1;
        auto fan = [&](const double *p, const double *q) {
            for (int j = 0; j < 3; ++j) {
                a[j] = p[j] - avg[j];
                b[j] = q[j] - avg[j];
            }
            cc[0] = a[1] * b[2] - a[2] * b[1];
            cc[1] = a[2] * b[0] - a[0] * b[2];
            cc[2] = a[0] * b[1] - a[1] * b[0];
            ts = 0.0;
            for (int j = 0; j < 3; ++j) ts += cc[j] * cc[j];
            ts = std::sqrt(ts);
            sq += ts;
        };
        for (int64_t i = 0; i < last; ++i) {
            fan(V(i), V(i + 1));
            for (int j = 0; j < 3; ++j) c[j] += ts * (a[j] + b[j] + avg3[j]);
        }
        fan(V(last), V(0));
        const double sq3 = sq * 3;
        for (int j = 0; j < 3; ++j) {
            c[j] += ts * (a[j] + b[j] + avg3[j]);
            c[j] /= sq3;
            nn[j] = cc[j];
        }
        sq *= 0.5;
    }
    double len = 0.0;  // psstGeometryVector::initialize + normalize
    for (int i = 0; i < dim; ++i) len += nn[i] * nn[i];
    len = std::sqrt(len);
    if (std::fabs(len) < 1.0e-10) raise(PSST_ERR_FORMAT, "Error: Division by zero detected!");
    for (int i = 0; i < dim; ++i) nn[i] /= len;
    g.S[f] = sq;
    for (int i = 0; i < dim; ++i) {
        g.n[f * dim + i] = nn[i];
        g.xf[f * dim + i] = c[i];
    }
}

void volume_geometry(psst_grid &g, const RawMesh &m, const std::vector<int64_t> &f_loc, int64_t v) {
    const int dim = g.dim;
    const int64_t b = g.vf_ptr[v], nf = g.vf_ptr[v + 1] - b;
    const int64_t *fl = &g.vf_idx[b];
    double *x = &g.xc[v * dim];
    for (int i = 0; i < dim; ++i) x[i] = 0.0;
    g.V[v] = 0.0;
    if (g.vol_boundary[v]) {  // ghost: centre of its face, volume 0
        for (int i = 0; i < dim; ++i) x[i] = g.xf[fl[0] * dim + i];
        return;
    }
    auto vert = [&](int64_t id1) { return &m.verts[(id1 - 1) * dim]; };
    double vol = 0.0;
    if (dim == 2) {
        double avg[2] = {0, 0}, avg3[2];
        for (int j = 0; j < 2; ++j) {
            for (int64_t i = 0; i < nf; ++i) avg[j] += g.xf[fl[i] * 2 + j];
            avg[j] /= (double)nf;
            avg3[j] = avg[j] * 3;
        }
        for (int64_t i = 0; i < nf; ++i) {
            const int64_t *nodes = &m.face_nodes[m.face_ptr[f_loc[fl[i]]]];
            double a[2], bb[2];
            for (int k = 0; k < 2; ++k) {
                a[k] = vert(nodes[0])[k] - avg[k];
                bb[k] = vert(nodes[1])[k] - avg[k];
            }
            double tv = std::fabs(a[0] * bb[1] - a[1] * bb[0]);
            vol += tv;
            for (int k = 0; k < 2; ++k) x[k] += tv * (a[k] + bb[k] + avg3[k]);
        }
        const double v3 = vol * 3;
        for (int k = 0; k < 2; ++k) x[k] /= v3;
        vol /= 2;
    } else {
        double avg[3] = {0, 0, 0}, avg4[3];
        for (int j = 0; j < 3; ++j) {
            for (int64_t i = 0; i < nf; ++i) avg[j] += g.xf[fl[i] * 3 + j];
            avg[j] /= (double)nf;
            avg4[j] = avg[j] * 4;
        }
        for (int64_t i = 0; i < nf; ++i) {
            const int64_t loc = f_loc[fl[i]];
            const int64_t nvx = m.face_ptr[loc + 1] - m.face_ptr[loc];
            const int64_t *nodes = &m.face_nodes[m.face_ptr[loc]];
            const double *cen = &g.xf[fl[i] * 3];
            for (int64_t j = 0; j < nvx; ++j) {
                int64_t nx = j + 1;
                if (nx == nvx) nx = 0;
                double a[3], bb[3], cc[3];
                for (int k = 0; k < 3; ++k) {
                    a[k] = vert(nodes[j])[k] - avg[k];
                    bb[k] = vert(nodes[nx])[k] - avg[k];
                    cc[k] = cen[k] - avg[k];
                }
                double tv = std::fabs(a[0] * (bb[1] * cc[2] - bb[2] * cc[1]) - a[1] * (bb[0] * cc[2] - bb[2] * cc[0]) +
                                      a[2] * (bb[0] * cc[1] - bb[1] * cc[0]));
                vol += tv;
                for (int k = 0; k < 3; ++k) x[k] += tv * (a[k] + bb[k] + cc[k] + avg4[k]);
            }
        }
        const double v4 = vol * 4.0;
        for (int k = 0; k < 3; ++k) x[k] /= v4;
        vol /= 6.0;
    }
    g.V[v] = vol;
}

// psstGreenGauss::initialize (psstGradCalculation.cpp:17-72). beta_ is sized by
// the total face count but indexed by the face's position inside its zone, so
// after the loop beta_[i] holds the value of the last zone (ascending id, zone
// 31 skipped) with more than i faces, and calculate() reads it back the same
// way (:139-142). The per-face array below is that final table.
void green_gauss_beta(psst_grid &g) {
    const int dim = g.dim;
    int64_t maxc = 0;
    for (auto &z : g.fz) maxc = std::max(maxc, z.count);
    std::vector<double> bz((size_t)maxc + 1, 0.0);
    for (auto &z : g.fz) {
        if (z.bc == 31) continue;
        parallel_for(z.count, [&](int64_t i0, int64_t i1) {
            for (int64_t i = i0; i < i1; ++i) {
                const int64_t f = z.first + i;
                double d[2];
                for (int j = 0; j < 2; ++j) {
                    d[j] = 0.0;
                    const int64_t v = j == 0 ? g.f_c0[f] : g.f_c1[f];
                    if (v >= 0 && !g.vol_boundary[v]) {
                        double dist = 0.0;
                        for (int k = 0; k < dim; ++k) {
                            double add = (g.xf[f * dim + k] - g.xc[v * dim + k]);
                            add = add * add;
                            dist += add;
                        }
                        d[j] = std::sqrt(dist);
                    }
                }
                bz[i] = d[1] / (d[0] + d[1]);
            }
        });
    }
    for (auto &z : g.fz)
        for (int64_t i = 0; i < z.count; ++i) g.beta[z.first + i] = bz[i];
}

}  // namespace

psst_grid *build_grid(const RawMesh &m) {
    std::unique_ptr<psst_grid> gp(new psst_grid);
    psst_grid &g = *gp;
    g.dim = m.dim;
    const int dim = m.dim;
    std::map<int64_t, int64_t> vzs, fzs;  // zone id -> slot in m.zones, ascending id
    for (size_t i = 0; i < m.zones.size(); ++i) {
        const int64_t bc = m.zones[i].bc;
        if (bc == 1 || bc == 32)
            vzs[m.zones[i].id] = (int64_t)i;
        else if (bc == 2 || bc == 31)
            fzs[m.zones[i].id] = (int64_t)i;
        else {
            vzs[m.zones[i].id] = (int64_t)i;
            fzs[m.zones[i].id] = (int64_t)i;
        }
    }
    std::map<int64_t, int32_t> vslot, fslot;
    for (auto &kv : vzs) {
        const Zone &z = m.zones[kv.second];
        vslot[z.id] = (int32_t)g.vz.size();
        VZone v;
        v.id = z.id;
        v.bc = z.bc;
        v.first = g.nvol;
        v.count = z.size;
        v.name = z.name;
        g.vz.push_back(v);
        g.nvol += z.size;
        if (z.bc == 1) g.ninterior += z.size;
        if (z.bc != 1 && z.bc != 32) g.nghost += z.size;
    }
    for (auto &kv : fzs) {
        const Zone &z = m.zones[kv.second];
        fslot[z.id] = (int32_t)g.fz.size();
        FZone f;
        f.id = z.id;
        f.bc = z.bc;
        f.first = g.nface;
        f.count = z.size;
        f.name = z.name;
        g.fz.push_back(f);
        g.nface += z.size;
    }
    g.vol_boundary.assign(g.nvol, 0);
    g.vol_vz.assign(g.nvol, 0);
    for (size_t s = 0; s < g.vz.size(); ++s) {
        const bool bnd = !(g.vz[s].bc == 1 || g.vz[s].bc == 32);
        for (int64_t j = 0; j < g.vz[s].count; ++j) {
            g.vol_boundary[g.vz[s].first + j] = bnd;
            g.vol_vz[g.vz[s].first + j] = (int32_t)s;
        }
    }
    const int64_t nfile_faces = (int64_t)m.face_c0.size();
    g.f_c0.assign(g.nface, -1);
    g.f_c1.assign(g.nface, -1);
    g.f_fz.assign(g.nface, 0);
    std::vector<int64_t> f_loc(g.nface);
    for (size_t s = 0; s < g.fz.size(); ++s) {
        const Zone &z = m.zones[fzs[g.fz[s].id]];
        for (int64_t j = 0; j < g.fz[s].count; ++j) {
            const int64_t f = g.fz[s].first + j;
            g.f_fz[f] = (int32_t)s;
            f_loc[f] = z.first + j - 1;
            if (f_loc[f] < 0 || f_loc[f] >= nfile_faces) raise(PSST_ERR_FORMAT, "mesh: face index out of range");
        }
    }
    g.S.assign(g.nface, 0.0);
    g.n.assign(g.nface * dim, 0.0);
    g.xf.assign(g.nface * dim, 0.0);
    g.beta.assign(g.nface, 0.0);

    // Wiring in file zone order (psstAnsysGridReader.cpp:825-883): the order in
    // which faces are appended to a volume is its face order everywhere after.
    // volume of every file cell (-1: its zone is no volume zone)
    std::vector<int64_t> cell_vol(m.cell_zone.size(), -1);
    for (auto &kv : vzs) {
        const Zone &z = m.zones[kv.second];
        const int64_t base = g.vz[vslot[z.id]].first;
        for (int64_t c = 0; c < z.size; ++c)
            if (z.first - 1 + c >= 0 && z.first - 1 + c < (int64_t)cell_vol.size() && m.cell_zone[z.first - 1 + c] == z.id)
                cell_vol[z.first - 1 + c] = base + c;
    }
    std::vector<int64_t> cnt(g.nvol, 0);
    std::vector<int64_t> worder;  // faces in wiring order
    worder.reserve(g.nface);
    for (size_t zi = 0; zi < m.zones.size(); ++zi) {
        const Zone &z = m.zones[zi];
        if (z.bc == 1 || z.bc == 32) continue;
        const int32_t fs = fslot[z.id];
        const int64_t ghost0 = z.bc == 2 || z.bc == 31 ? -1 : g.vz[vslot[z.id]].first;
        for (int64_t j = 0; j < g.fz[fs].count; ++j) {
            const int64_t f = g.fz[fs].first + j;
            const int64_t loc = f_loc[f];
            for (int k = 0; k < 2; ++k) {
                const int64_t cell = k == 0 ? m.face_c0[loc] : m.face_c1[loc];
                int64_t vol;
                if (cell == 0) {
                    if (z.bc == 31) continue;
                    if (ghost0 < 0) raise(PSST_ERR_FORMAT, "mesh: interior face without two neighbours");
                    vol = ghost0 + j;
                } else {
                    if (cell - 1 >= (int64_t)m.cell_zone.size()) raise(PSST_ERR_FORMAT, "mesh: cell index out of range");
                    vol = cell_vol[cell - 1];
                    if (vol < 0) raise(PSST_ERR_FORMAT, "mesh: face refers to a cell outside any cell zone");
                }
                (k == 0 ? g.f_c0[f] : g.f_c1[f]) = vol;
                if (z.bc != 31) ++cnt[vol];
            }
            worder.push_back(f);
        }
    }
    // face lists in wiring order: faces of zone 31 are in none
    g.vf_ptr.assign(g.nvol + 1, 0);
    for (int64_t v = 0; v < g.nvol; ++v) {
        g.vf_ptr[v + 1] = g.vf_ptr[v] + cnt[v];
        g.max_faces = std::max<int>(g.max_faces, (int)cnt[v]);
    }
    g.vf_idx.assign(g.vf_ptr[g.nvol], 0);
    {
        std::vector<int64_t> fill(g.vf_ptr.begin(), g.vf_ptr.end() - 1);
        for (int64_t f : worder) {
            if (g.fz[g.f_fz[f]].bc == 31) continue;
            if (g.f_c0[f] >= 0) g.vf_idx[fill[g.f_c0[f]]++] = f;
            if (g.f_c1[f] >= 0) g.vf_idx[fill[g.f_c1[f]]++] = f;
        }
    }
    parallel_for((int64_t)worder.size(), [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) face_geometry(g, m, worder[i], f_loc[worder[i]]);
    });

    g.V.assign(g.nvol, 0.0);
    g.xc.assign(g.nvol * dim, 0.0);
    std::vector<int64_t> vorder;  // volumes in the reference's initialisation order
    for (size_t zi = 0; zi < m.zones.size(); ++zi) {
        const Zone &z = m.zones[zi];
        if (z.bc == 2 || z.bc == 31 || z.bc == 32) continue;
        const VZone &vz = g.vz[vslot[z.id]];
        for (int64_t j = 0; j < vz.count; ++j) {
            const int64_t v = vz.first + j;
            if (g.vol_boundary[v] && cnt[v] != 1)
                raise(PSST_ERR_FORMAT, "mesh: boundary zone " + std::to_string(z.id) +
                                           " has a face without a free side (no ghost cell)");
            if (!g.vol_boundary[v] && cnt[v] == 0) raise(PSST_ERR_FORMAT, "mesh: cell without faces");
            vorder.push_back(v);
        }
    }
    parallel_for((int64_t)vorder.size(), [&](int64_t b, int64_t e) {
        for (int64_t i = b; i < e; ++i) volume_geometry(g, m, f_loc, vorder[i]);
    });
    double mn = -1.0;  // psstAnsysGridReader.cpp:886-905
    for (int64_t v : vorder)
        if (g.vz[g.vol_vz[v]].bc == 1 && (mn > g.V[v] || mn < 0.0)) mn = g.V[v];
    g.min_vol = mn;
    green_gauss_beta(g);
    return gp.release();
}

// psstLeastSquare::initialize (psstGradCalculation.cpp:191-260). r_ is
// indexed by the cell's position inside its zone, so with several interior
// zones the last zone (ascending id) with more than i cells wins; calculate()
// reads it back the same way (:404-412). kLsqNR coefficients per index: r11,
// r12, r22 and, in 3D, r13, r23, r33 and beta, the Gram-Schmidt factors of the
// weighted (w = 1/|dx|^2) normal equations as the reference forms them.
std::vector<double> lsq_table(const psst_grid &g) {
    const int dim = g.dim;
    int64_t maxc = 0;
    for (auto &z : g.vz)
        if (z.bc == 1) maxc = std::max(maxc, z.count);
    std::vector<double> lsq_r(kLsqNR * (maxc + 1), 0.0);
    for (auto &z : g.vz) {
        if (z.bc != 1) continue;
        for (int64_t i = 0; i < z.count; ++i) {
            const int64_t v = z.first + i;
            double ca = 0.0, cb = 0.0, cd = 0.0, cc = 0.0, ce = 0.0, cg = 0.0;
            for (int64_t e = g.vf_ptr[v]; e < g.vf_ptr[v + 1]; ++e) {
                const int64_t f = g.vf_idx[e];
                const int64_t nb = g.f_c0[f] == v ? g.f_c1[f] : g.f_c0[f];
                double diff[3] = {0.0, 0.0, 0.0}, w = 0.0;
                for (int k = 0; k < dim; ++k) {
                    diff[k] = g.xc[nb * dim + k] - g.xc[v * dim + k];
                    w += diff[k] * diff[k];
                }
                const double ws = 1.0 / w;
                ca += ws * diff[0] * diff[0];
                cb += ws * diff[0] * diff[1];
                cd += ws * diff[1] * diff[1];
                if (dim == 3) {
                    cc += ws * diff[0] * diff[2];
                    ce += ws * diff[1] * diff[2];
                    cg += ws * diff[2] * diff[2];
                }
            }
            double *r = &lsq_r[kLsqNR * i];
            r[0] = std::sqrt(ca);
            r[1] = cb / r[0];
            r[2] = std::sqrt(cd - r[1] * r[1]);
            if (dim == 3) {
                r[3] = cc / r[0];
                r[4] = (ce - r[1] / r[0] * cc) / r[2];
                r[5] = std::sqrt(cg - (r[3] * r[3] + r[4] * r[4]));
                r[6] = (r[1] * r[4] - r[3] * r[2]) / (r[0] * r[2]);
            }
        }
    }
    return lsq_r;
}

}  // namespace psst
