// ref_dump: runs the compiled PSST reference (built in place from its own
// sources, see oracle/Makefile) on one case and dumps its full FP64 state.
//
// TEST INFRASTRUCTURE ONLY (the oracle's executable arm). Nothing in the
// product links or runs this.
//
// Usage (cwd = case directory holding <case>.inp/.prop/.par/.bvp/.btq):
//     ref_dump <mesh.msh> <case> <outdir>
// It follows main.cpp:9-63 (Director/Builder read, create_finite_volume_grid,
// solver_parameters, explicit_solve) and then writes .npy arrays to <outdir>:
//   vol_*  : every volume of every volume zone in std::map (zone id) order,
//            interior and ghost, i.e. the reference's storage order
//   face_* : every face of every face zone in std::map order (zone 31 kept)
// Reading goes through the public accessors of psstGridFV
// (psstFiniteVolumeGrid.h:54-65) only.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "psstAnsysGridReader.h"
#include "psstFiniteVolumeGrid.h"
#include "psstFiniteVolumeGridTools.h"
#include "psstGridReader.h"
#include "psstOutputManager.h"
#include "psstVariable.h"

static void write_npy(const std::string &path, const char *descr, size_t itemsize,
                      const void *data, size_t n) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::fprintf(stderr, "cannot write %s\n", path.c_str());
        std::exit(3);
    }
    char hdr[256];
    int len = std::snprintf(hdr, sizeof hdr,
                            "{'descr': '%s', 'fortran_order': False, 'shape': (%zu,), }",
                            descr, n);
    int total = 10 + len + 1;
    int pad = (64 - total % 64) % 64;
    unsigned short hlen = (unsigned short)(len + pad + 1);
    std::fwrite("\x93NUMPY\x01\x00", 1, 8, f);
    std::fwrite(&hlen, 2, 1, f);
    std::fwrite(hdr, 1, len, f);
    for (int i = 0; i < pad; ++i) std::fputc(' ', f);
    std::fputc('\n', f);
    if (n) std::fwrite(data, itemsize, n, f);
    std::fclose(f);
}

static void dump_d(const std::string &dir, const char *name, const std::vector<double> &v) {
    write_npy(dir + "/" + name + ".npy", "<f8", 8, v.data(), v.size());
}
static void dump_i(const std::string &dir, const char *name, const std::vector<int64_t> &v) {
    write_npy(dir + "/" + name + ".npy", "<i8", 8, v.data(), v.size());
}

int main(int argc, char **argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: ref_dump <mesh> <case> <outdir>\n");
        return 2;
    }
    const std::string mesh = argv[1], case_name = argv[2], out = argv[3];
    try {
        std::ifstream in(mesh);
        if (!in.is_open()) {
            std::fprintf(stderr, "cannot open %s\n", mesh.c_str());
            return 2;
        }
        psstInterfaceGridBuilder *builder = new psstAnsysBuilder;
        psstInterfaceGridDirector *director = new psstAnsysDirector;
        director->set_builder(builder);
        psstInterfaceInputGrid *grid = director->construct_grid(in);
        in.close();
        std::shared_ptr<psstInterfaceOutputManager> om =
            std::make_shared<psstAnsysOutputManager>(case_name);
        psstGridFV *fv = grid->create_finite_volume_grid();
        fv->attach_output_manager(om);
        fv->settings_file_name(case_name);
        fv->solver_parameters();
        fv->explicit_solve();

        const size_t dim = fv->dimension();
        std::unordered_map<const psstInterfaceVolume *, int64_t> vindex;
        std::vector<int64_t> vzone, vbc, vbnd, vnf, vfaces;
        std::vector<double> p, T, rho, u, w, pw, res, dt, gu, gp, gT, grho, V, xc;
        auto *vs = fv->volume_storage();
        for (auto &z : *vs) {
            for (size_t i = 0; i < z.second.volumes_.size(); ++i) {
                auto vol = z.second.volumes_[i];
                vindex[vol.get()] = (int64_t)vindex.size();
            }
        }
        // faces: index faces in map order to record each volume's face list
        std::unordered_map<const psstInterfaceFace *, int64_t> findex;
        auto *fs = fv->face_storage();
        for (auto &z : *fs)
            for (size_t i = 0; i < z.second.faces_.size(); ++i)
                findex[z.second.faces_[i].get()] = (int64_t)findex.size();

        for (auto &z : *vs) {
            for (size_t i = 0; i < z.second.volumes_.size(); ++i) {
                auto vol = z.second.volumes_[i];
                auto var = vol->variable();
                vzone.push_back((int64_t)z.first);
                vbc.push_back((int64_t)z.second.bc_type_id_);
                vbnd.push_back(vol->is_boundary() ? 1 : 0);
                vnf.push_back((int64_t)vol->number_of_faces());
                for (size_t j = 0; j < vol->number_of_faces(); ++j) {
                    auto fc = vol->face_ptr(j);
                    vfaces.push_back(findex.count(fc.get()) ? findex[fc.get()] : -1);
                }
                p.push_back(var->pressure());
                T.push_back(var->temperature());
                rho.push_back(var->density());
                for (size_t k = 0; k < dim; ++k) u.push_back(var->velocity(k));
                for (size_t k = 0; k < dim + 2; ++k) {
                    w.push_back(var->w(k));
                    pw.push_back(var->prev_w(k));
                    res.push_back(var->residual(k));
                }
                dt.push_back(var->time_step());
                for (size_t j = 0; j < dim; ++j)
                    for (size_t k = 0; k < dim; ++k) gu.push_back(var->grad_velocity(j)->component(k));
                for (size_t k = 0; k < dim; ++k) {
                    gp.push_back(var->grad_pressure()->component(k));
                    gT.push_back(var->grad_temperature()->component(k));
                    grho.push_back(var->grad_density()->component(k));
                }
                V.push_back(vol->volume());
                for (size_t k = 0; k < dim; ++k) xc.push_back(vol->center_vertex()->component(k));
            }
        }
        std::vector<int64_t> fzone, fbc, fc0, fc1;
        std::vector<double> S, n, xf;
        for (auto &z : *fs) {
            for (size_t i = 0; i < z.second.faces_.size(); ++i) {
                auto f = z.second.faces_[i];
                fzone.push_back((int64_t)z.first);
                fbc.push_back((int64_t)z.second.bc_type_id_);
                auto a = f->neighbour_ptr(0), b = f->neighbour_ptr(1);
                fc0.push_back(a ? vindex[a.get()] : -1);
                fc1.push_back(b ? vindex[b.get()] : -1);
                S.push_back(f->square());
                for (size_t k = 0; k < dim; ++k) n.push_back(f->normal_vector()->component(k));
                for (size_t k = 0; k < dim; ++k) xf.push_back(f->center_vertex()->component(k));
            }
        }
        dump_i(out, "dim", {(int64_t)dim});
        dump_d(out, "min_vol", {fv->min_vol()});
        dump_d(out, "gas", {fv->rm(), fv->cp(), fv->cv(), fv->gamma()});
        dump_i(out, "vol_zone", vzone);
        dump_i(out, "vol_bc", vbc);
        dump_i(out, "vol_boundary", vbnd);
        dump_i(out, "vol_nfaces", vnf);
        dump_i(out, "vol_faces", vfaces);
        dump_d(out, "vol_p", p);
        dump_d(out, "vol_T", T);
        dump_d(out, "vol_rho", rho);
        dump_d(out, "vol_u", u);
        dump_d(out, "vol_w", w);
        dump_d(out, "vol_prev_w", pw);
        dump_d(out, "vol_residual", res);
        dump_d(out, "vol_dt", dt);
        dump_d(out, "vol_grad_u", gu);
        dump_d(out, "vol_grad_p", gp);
        dump_d(out, "vol_grad_T", gT);
        dump_d(out, "vol_grad_rho", grho);
        dump_d(out, "vol_V", V);
        dump_d(out, "vol_x", xc);
        dump_i(out, "face_zone", fzone);
        dump_i(out, "face_bc", fbc);
        dump_i(out, "face_c0", fc0);
        dump_i(out, "face_c1", fc1);
        dump_d(out, "face_S", S);
        dump_d(out, "face_n", n);
        dump_d(out, "face_x", xf);
        delete fv;
        delete grid;
        delete director;
        delete builder;
    } catch (std::runtime_error &e) {
        std::fprintf(stderr, "reference error: %s\n", e.what());
        return 1;
    } catch (std::logic_error &e) {
        std::fprintf(stderr, "reference error: %s\n", e.what());
        return 1;
    }
    return 0;
}
