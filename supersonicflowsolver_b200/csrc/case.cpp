// Case setup: the reference's positional text files.
//
// psstGridFV::solver_parameters (psstFiniteVolumeGrid.cpp:36-194) reads
// <case>.inp line by line with get_parameter (:20-27: a number, then the rest
// of the line is skipped), after private_initialize_field (.prop, then .par or
// .sav, :641-717) and private_load_boundary (.bvp then .btq, :403-557). This
// file reproduces those reads, including the order in which the initial field,
// the ghost states and the reference speed of psstUniformTime are formed.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "host.hpp"

namespace psst {
namespace {

struct Text {
    std::vector<char> buf;
    size_t pos = 0;
    bool eof() const { return pos >= buf.size(); }
    static bool ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }
    void skip_ws() {
        while (pos < buf.size() && ws(buf[pos])) ++pos;
    }
    bool dbl(double &x) {
        skip_ws();
        if (eof()) return false;
        buf.push_back(0);
        char *e;
        double v = std::strtod(&buf[pos], &e);
        buf.pop_back();
        if (e == &buf[pos]) return false;
        pos = (size_t)(e - buf.data());
        x = v;
        return true;
    }
    bool word(std::string &w) {
        skip_ws();
        if (eof()) return false;
        w.clear();
        while (pos < buf.size() && !ws(buf[pos])) w.push_back(buf[pos++]);
        return true;
    }
    bool integer(long &x) {
        double d;
        skip_ws();
        size_t p0 = pos;
        while (pos < buf.size() && !ws(buf[pos])) ++pos;
        std::string s(buf.begin() + p0, buf.begin() + pos);
        if (s.empty()) return false;
        char *e;
        d = std::strtod(s.c_str(), &e);
        x = (long)d;
        return e != s.c_str();
    }
    void rest_of_line() {
        while (pos < buf.size() && buf[pos++] != '\n') continue;
    }
    double parameter() {  // get_parameter (psstFiniteVolumeGrid.cpp:20-27)
        double x = 0.0;
        dbl(x);
        rest_of_line();
        return x;
    }
};

Text open_text(const std::string &path, const char *what) {
    Text t;
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) raise(PSST_ERR_IO, std::string(what) + " (" + path + ")");
    char tmp[65536];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof tmp, f)) > 0) t.buf.insert(t.buf.end(), tmp, tmp + n);
    std::fclose(f);
    return t;
}

int64_t other(const psst_grid &g, int64_t f, int64_t v) { return g.f_c0[f] == v ? g.f_c1[f] : g.f_c0[f]; }

}  // namespace

// Ghost boundary conditions on the host (setup only; the device applies them
// every stage). psstBoundaryCondition.cpp:26-37, 60-127, 197-219, 240-357.
void apply_dynamic(const psst_grid &g, const VZone &z, int64_t v, double *P, double *T, double *U) {
    const int dim = g.dim;
    const int64_t nv = g.nvol;
    const int64_t f = g.vf_idx[g.vf_ptr[v]];
    const int64_t nb = other(g, f, v);
    (void)T;
    switch (z.dyn) {
    case 26:
        for (int j = 0; j < dim; ++j) U[j * nv + v] = U[j * nv + nb];
        P[v] = P[nb];
        break;
    case 15: {
        double vn = 0.0;
        for (int j = 0; j < dim; ++j) vn += U[j * nv + nb] * g.n[f * dim + j];
        for (int j = 0; j < dim; ++j) U[j * nv + v] = U[j * nv + nb] - vn * g.n[f * dim + j];
        P[v] = P[nb];
        break;
    }
    case 25:
        for (int j = 0; j < dim; ++j) U[j * nv + v] = U[j * nv + nb];
        break;
    default:
        break;
    }
}

}  // namespace psst

using namespace psst;

extern "C" psst_status psst_case_read(psst_grid *g, const char *dir, const char *name, psst_scheme *sc,
                                      double *prim_out) {
    try {
        if (!g || !dir || !name || !sc) raise(PSST_ERR_ARG, "psst_case_read: null argument");
        const std::string base = std::string(dir) + "/" + name;
        const int dim = g->dim;
        const int64_t nv = g->nvol;
        std::memset(sc, 0, sizeof *sc);
        sc->precision = 64;
        sc->renumber = 1;
        sc->venkat_k = 5.0;
        Text inp = open_text(base + ".inp", "Error: Could not found setting file!");
        const long init_mode = (long)inp.parameter();

        // private_initialize_field
        Text prop = open_text(base + ".prop", "Error: Could not open fluid properties file");
        const double M = prop.parameter();
        const double cp = prop.parameter();
        const double R = 8.31;
        sc->rm = R / M;
        sc->cp = cp;
        sc->gamma = cp / (cp - sc->rm);
        sc->cv = cp / sc->gamma;
        std::vector<double> prim((size_t)(2 + dim) * nv, 0.0);
        double *P = prim.data(), *T = P + nv, *U = T + nv;
        std::vector<double> rho(nv, 0.0);
        if (init_mode == 0) {
            sc->iter = 1;
            Text par = open_text(base + ".par", "Error! Could not open initial parameters file!");
            double vel[3] = {0, 0, 0};
            for (int j = 0; j < dim - 1; ++j) par.dbl(vel[j]);
            vel[dim - 1] = par.parameter();
            const double Ti = par.parameter();
            const double pi = par.parameter();
            for (auto &z : g->vz) {
                if (z.bc != 1) continue;
                for (int64_t i = 0; i < z.count; ++i) {
                    const int64_t v = z.first + i;
                    for (int j = 0; j < dim; ++j) U[j * nv + v] = vel[j];
                    T[v] = Ti;
                    P[v] = pi;
                }
            }
        } else if (init_mode == 1) {
            Text sav = open_text(base + ".sav", "Error! Could not open initial parameters file!");
            long it = 0;
            sav.integer(it);
            sc->iter = it;
            while (!sav.eof()) {  // private_load_parameter (:559-604)
                long zid = 0, cnt = 0;
                if (!sav.integer(zid) || zid == 0) break;
                int32_t slot = -1;
                for (size_t s = 0; s < g->vz.size(); ++s)
                    if (g->vz[s].id == zid) slot = (int32_t)s;
                if (slot < 0) raise(PSST_ERR_FORMAT, "sav: unknown zone " + std::to_string(zid));
                sav.integer(cnt);
                if (cnt != g->vz[slot].count) raise(PSST_ERR_FORMAT, "Error! Different size of storage found!");
                for (long i = 0; i < cnt; ++i) {
                    const int64_t v = g->vz[slot].first + i;
                    sav.dbl(P[v]);
                    sav.dbl(T[v]);
                    for (int j = 0; j < dim; ++j) sav.dbl(U[j * nv + v]);
                }
            }
        } else {
            raise(PSST_ERR_FORMAT, "Error! Unknown command detected!");
        }

        // private_load_boundary: .bvp
        double ref_vel = 0.0;
        bool have_ref = false;
        for (auto &z : g->vz) z.dyn = z.therm = 0;
        auto find_zone = [&](const std::string &zn) -> VZone & {
            for (auto &z : g->vz)
                if (z.name == zn) {
                    if (z.bc == 1 || z.bc == 2 || z.bc == 31 || z.bc == 32)
                        raise(PSST_ERR_FORMAT, "Error: Could not attach boundary condition to inner zone!");
                    return z;
                }
            raise(PSST_ERR_FORMAT, "Error: Could not found zone!");
        };
        Text bvp = open_text(base + ".bvp", "Error! Could not open boundary condition file!");
        std::string zn;
        long id;
        while (!bvp.eof()) {
            if (!bvp.word(zn) || !bvp.integer(id)) break;
            VZone &z = find_zone(zn);
            z.dyn = (int)id;
            if (id == 23) {
                ref_vel = 0.0;
                for (int i = 0; i < dim; ++i) {
                    bvp.dbl(z.u[i]);
                    ref_vel += z.u[i] * z.u[i];
                }
                ref_vel = std::sqrt(ref_vel);
                have_ref = true;
                z.p = bvp.parameter();
                for (int64_t i = 0; i < z.count; ++i) {
                    const int64_t v = z.first + i;
                    P[v] = z.p;
                    for (int j = 0; j < dim; ++j) U[j * nv + v] = z.u[j];
                }
            } else if (id == 26 || id == 15) {
                for (int64_t i = 0; i < z.count; ++i) apply_dynamic(*g, z, z.first + i, P, T, U);
            } else if (id == 27) {
                raise(PSST_ERR_UNSUPPORTED, "Error: Wrong dimension!");  // psstInlet ctor always throws (:147)
            } else if (id == 25) {
                z.p = bvp.parameter();
                for (int64_t i = 0; i < z.count; ++i) {
                    P[z.first + i] = z.p;
                    apply_dynamic(*g, z, z.first + i, P, T, U);
                }
            } else {
                raise(PSST_ERR_FORMAT, "bvp: unknown boundary condition id " + std::to_string(id));
            }
        }
        // .btq
        Text btq = open_text(base + ".btq", "Error! Could not open boundary condition file!");
        while (!btq.eof()) {
            if (!btq.word(zn) || !btq.integer(id)) break;
            VZone &z = find_zone(zn);
            if (!z.dyn) raise(PSST_ERR_FORMAT, "btq: zone " + zn + " has no dynamic condition");
            z.therm = (int)id;
            if (id == 11 || id == 27) {
                z.T = btq.parameter();
                const double c = std::sqrt(sc->gamma * sc->rm * z.T);
                if (ref_vel < c) ref_vel = c;
                have_ref = true;
                for (int64_t i = 0; i < z.count; ++i) T[z.first + i] = z.T;
            } else if (id == 18 || id == 25) {
                for (int64_t i = 0; i < z.count; ++i) {
                    const int64_t v = z.first + i;
                    T[v] = T[other(*g, g->vf_idx[g->vf_ptr[v]], v)];
                }
            } else {
                raise(PSST_ERR_FORMAT, "btq: unknown thermal condition id " + std::to_string(id));
            }
        }
        (void)have_ref;

        // remaining .inp lines
        sc->cfl = inp.parameter();
        sc->lc = (int32_t)(long)inp.parameter();
        if (sc->lc < 0 || sc->lc > 2) raise(PSST_ERR_FORMAT, "inp: unknown local time step mode");
        if (sc->lc == 0 && std::fabs(ref_vel) < 1.0e-10) ref_vel = 1.0;
        sc->ref_vel = ref_vel;
        g->ref_vel = ref_vel;
        const long mx = (long)inp.parameter();
        sc->max_iter = mx + sc->iter - 1;
        sc->iter_step = (long)inp.parameter();
        sc->rk_level = (int32_t)(long)inp.parameter();
        const long rk_mode = (long)inp.parameter();
        if (rk_mode == 0) {
            static const double tab[6][5] = {{0}, {1.0}, {0.4242, 1.0}, {0.1918, 0.4929, 1.0000},
                                             {0.1084, 0.2602, 0.5052, 1.0000},
                                             {0.0695, 0.1602, 0.2898, 0.5060, 1.0000}};
            if (sc->rk_level < 1 || sc->rk_level > 5) raise(PSST_ERR_FORMAT, "Error: Unknow RK order!");
            for (int i = 0; i < sc->rk_level; ++i) sc->rk[i] = tab[sc->rk_level][i];
            inp.rest_of_line();
        } else {
            if (sc->rk_level < 1 || sc->rk_level > 16)
                raise(PSST_ERR_FORMAT, "Error! Expected Runge Kutta coefficients but empty vector found!");
            for (int i = 0; i < sc->rk_level - 1; ++i) inp.dbl(sc->rk[i]);
            sc->rk[sc->rk_level - 1] = inp.parameter();
        }
        sc->flux = (int32_t)(long)inp.parameter();
        sc->order = (int32_t)(long)inp.parameter();
        sc->grad = (int32_t)(long)inp.parameter() == 1 ? 1 : 2;
        sc->limiter = (int32_t)(long)inp.parameter();
        if (sc->flux < 1 || sc->flux > 3) raise(PSST_ERR_FORMAT, "Error: Unknow convective flow scheme!");
        if (sc->order != 1 && sc->order != 2) raise(PSST_ERR_FORMAT, "Error! Unknown scheme order!");
        g->prim0 = prim;
        if (prim_out) std::memcpy(prim_out, prim.data(), prim.size() * sizeof(double));
        return PSST_OK;
    } catch (const Error &e) {
        set_last_error(e.msg);
        return e.status;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return PSST_ERR_ARG;
    }
}

extern "C" psst_status psst_grid_set_boundary(psst_grid *g, const char *zone_name, int dyn_id, const double *u,
                                              double p, int therm_id, double T) {
    try {
        if (!g || !zone_name) raise(PSST_ERR_ARG, "psst_grid_set_boundary: null argument");
        for (auto &z : g->vz) {
            if (z.name != zone_name) continue;
            if (z.bc == 1 || z.bc == 2 || z.bc == 31 || z.bc == 32)
                raise(PSST_ERR_ARG, "Error: Could not attach boundary condition to inner zone!");
            if (!(dyn_id == 23 || dyn_id == 26 || dyn_id == 15 || dyn_id == 25))
                raise(PSST_ERR_ARG, "unknown dynamic boundary condition id");
            if (!(therm_id == 27 || therm_id == 25 || therm_id == 11 || therm_id == 18))
                raise(PSST_ERR_ARG, "unknown thermal boundary condition id");
            z.dyn = dyn_id;
            z.therm = therm_id;
            for (int j = 0; j < g->dim; ++j) z.u[j] = u ? u[j] : 0.0;
            z.p = p;
            z.T = T;
            return PSST_OK;
        }
        raise(PSST_ERR_ARG, "Error: Could not found zone!");
    } catch (const Error &e) {
        set_last_error(e.msg);
        return e.status;
    }
}
