// C ABI: errors and mesh entry points (see include/psst_b200.h).
#include <cstring>
#include <exception>
#include <new>

#include "host.hpp"

namespace psst {

static thread_local std::string g_last_error;

void raise(psst_status st, const std::string &msg) { throw Error{st, msg}; }
void set_last_error(const std::string &msg) { g_last_error = msg; }

}  // namespace psst

using namespace psst;

#define PSST_API_BEGIN try {
#define PSST_API_END                                   \
    return PSST_OK;                                    \
    }                                                  \
    catch (const Error &e) {                           \
        set_last_error(e.msg);                         \
        return e.status;                               \
    }                                                  \
    catch (const std::bad_alloc &) {                   \
        set_last_error("out of host memory");          \
        return PSST_ERR_ARG;                           \
    }                                                  \
    catch (const std::exception &e) {                  \
        set_last_error(e.what());                      \
        return PSST_ERR_ARG;                           \
    }

extern "C" const char *psst_last_error(void) { return g_last_error.c_str(); }
extern "C" int psst_abi_version(void) { return PSST_B200_ABI_VERSION; }

extern "C" psst_status psst_grid_read_fluent(const char *path, psst_grid **out) {
    PSST_API_BEGIN
    if (!path || !out) raise(PSST_ERR_ARG, "psst_grid_read_fluent: null argument");
    *out = nullptr;
    RawMesh m = read_fluent(path);
    psst_grid *g = build_grid(m);
    g->raw = std::make_shared<RawMesh>(std::move(m));
    *out = g;
    PSST_API_END
}

extern "C" psst_status psst_grid_from_fluent(const psst_fluent_desc *d, psst_grid **out) {
    PSST_API_BEGIN
    if (!d || !out) raise(PSST_ERR_ARG, "psst_grid_from_fluent: null argument");
    *out = nullptr;
    if (d->dim != 2 && d->dim != 3) raise(PSST_ERR_ARG, "dimension must be 2 or 3");
    if (d->nvert < 0 || d->nface < 0 || d->ncell < 0 || d->nzone < 0) raise(PSST_ERR_ARG, "negative size");
    if ((d->nvert && !d->verts) || (d->nface && (!d->face_ptr || !d->face_nodes || !d->face_c0 || !d->face_c1)) ||
        (d->nzone && !d->zones))
        raise(PSST_ERR_ARG, "psst_grid_from_fluent: null array");
    RawMesh m;
    m.dim = d->dim;
    m.verts.assign(d->verts, d->verts + d->nvert * d->dim);
    m.face_ptr.assign(d->face_ptr, d->face_ptr + d->nface + 1);
    if (m.face_ptr[0] != 0) raise(PSST_ERR_ARG, "face_ptr[0] must be 0");
    const int64_t nn = m.face_ptr[d->nface];
    m.face_nodes.resize(nn);
    for (int64_t i = 0; i < nn; ++i) {
        const int64_t v = d->face_nodes[i];
        if (v < 0 || v >= d->nvert) raise(PSST_ERR_ARG, "face node out of range");
        m.face_nodes[i] = v + 1;
    }
    m.face_c0.resize(d->nface);
    m.face_c1.resize(d->nface);
    for (int64_t i = 0; i < d->nface; ++i) {
        if (d->face_c0[i] < -1 || d->face_c0[i] >= d->ncell || d->face_c1[i] < -1 || d->face_c1[i] >= d->ncell)
            raise(PSST_ERR_ARG, "face cell out of range");
        m.face_c0[i] = d->face_c0[i] + 1;
        m.face_c1[i] = d->face_c1[i] + 1;
    }
    m.cell_zone.assign(d->ncell, 0);
    for (int32_t z = 0; z < d->nzone; ++z) {
        const psst_zone_desc &zd = d->zones[z];
        Zone &zz = m.zones[m.zone_slot(zd.id)];
        zz.first = zd.first;
        zz.last = zd.last;
        zz.bc = zd.bc_type;
        zz.size = zd.last - zd.first + 1;
        zz.name = zd.name ? zd.name : "";
        if (zz.size < 0) raise(PSST_ERR_ARG, "zone range is negative");
        if (zd.bc_type == 1 || zd.bc_type == 32) {
            if (zd.first < 1 || zd.last > d->ncell) raise(PSST_ERR_ARG, "cell zone range out of bounds");
            for (int64_t c = zd.first; c <= zd.last; ++c) m.cell_zone[c - 1] = zd.id;
        } else if (zd.first < 1 || zd.last > d->nface) {
            raise(PSST_ERR_ARG, "face zone range out of bounds");
        }
    }
    psst_grid *g = build_grid(m);
    g->raw = std::make_shared<RawMesh>(std::move(m));
    *out = g;
    PSST_API_END
}

extern "C" psst_status psst_grid_get_info(const psst_grid *g, psst_grid_info *out) {
    PSST_API_BEGIN
    if (!g || !out) raise(PSST_ERR_ARG, "psst_grid_get_info: null argument");
    out->dim = g->dim;
    out->nvol = g->nvol;
    out->ninterior = g->ninterior;
    out->nghost = g->nghost;
    out->nface = g->nface;
    out->max_faces_per_cell = g->max_faces;
    out->min_vol = g->min_vol;
    PSST_API_END
}

extern "C" psst_status psst_grid_get_array(const psst_grid *g, const char *name, void *out, int64_t count) {
    PSST_API_BEGIN
    if (!g || !name || !out) raise(PSST_ERR_ARG, "psst_grid_get_array: null argument");
    const std::string nm(name);
    auto put_d = [&](const std::vector<double> &v) {
        if ((int64_t)v.size() != count) raise(PSST_ERR_ARG, nm + ": expected " + std::to_string(v.size()) + " elements");
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    };
    auto put_i = [&](int64_t n, auto fn) {
        if (n != count) raise(PSST_ERR_ARG, nm + ": expected " + std::to_string(n) + " elements");
        int64_t *o = (int64_t *)out;
        for (int64_t i = 0; i < n; ++i) o[i] = fn(i);
    };
    if (nm == "vol_V")
        put_d(g->V);
    else if (nm == "vol_x")
        put_d(g->xc);
    else if (nm == "face_S")
        put_d(g->S);
    else if (nm == "face_n")
        put_d(g->n);
    else if (nm == "face_x")
        put_d(g->xf);
    else if (nm == "face_beta")
        put_d(g->beta);
    else if (nm == "face_c0")
        put_i(g->nface, [&](int64_t i) { return g->f_c0[i]; });
    else if (nm == "face_c1")
        put_i(g->nface, [&](int64_t i) { return g->f_c1[i]; });
    else if (nm == "face_zone")
        put_i(g->nface, [&](int64_t i) { return g->fz[g->f_fz[i]].id; });
    else if (nm == "vol_zone")
        put_i(g->nvol, [&](int64_t i) { return g->vz[g->vol_vz[i]].id; });
    else if (nm == "vol_boundary")
        put_i(g->nvol, [&](int64_t i) { return (int64_t)g->vol_boundary[i]; });
    else if (nm == "vol_bc")
        put_i(g->nvol, [&](int64_t i) { return g->vz[g->vol_vz[i]].bc; });
    else
        raise(PSST_ERR_ARG, "unknown grid array " + nm);
    PSST_API_END
}

extern "C" void psst_grid_free(psst_grid *g) { delete g; }
