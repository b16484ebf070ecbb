// Fluent case and data files of a solution, byte for byte as PSST's
// psstAnsysOutputManager writes them (psstOutputManager.cpp:35-397): the .cas
// repeats the mesh as read (vertices, faces with their file neighbours, cell
// types, the cell/face trees of adapted meshes, zones), the .dat holds p, T,
// rho, u, v (, w) per volume zone in ascending zone id (ghost zones included;
// parent-cell zones skipped).
#include <cinttypes>
#include <cstdio>
#include <map>
#include <string>

#include "host.hpp"

using namespace psst;

namespace {

const char *bc_name(int64_t bc) {  // psstOutputManager.cpp:8-27
    static const std::map<int64_t, const char *> names = {
        {1, "fluid"},           {2, "interior"},           {3, "wall"},      {4, "pressure-inlet"},
        {5, "pressure-outlet"}, {7, "symmetry"},           {8, "periodic-shadow"},
        {9, "pressure-far-field"}, {10, "velocity-inlet"}, {12, "periodic"}, {14, "radiator"},
        {20, "mass-flow-inlet"}, {24, "interface"},        {31, "parent"},   {32, "parent"},
        {36, "outflow"},        {37, "axis"}};
    auto it = names.find(bc);
    if (it == names.end()) raise(PSST_ERR_ARG, "map::at");
    return it->second;
}

struct File {
    FILE *f = nullptr;
    explicit File(const std::string &path, const char *what) {
        f = std::fopen(path.c_str(), "wb");
        if (!f) raise(PSST_ERR_IO, std::string("Error: Could not open output *.") + what + " file!");
    }
    ~File() {
        if (f) std::fclose(f);
    }
};

// Fluent cell type from the number of faces (meshes given as arrays carry none).
int64_t cell_type_from_faces(int dim, int nf, bool has_tri) {
    if (dim == 2) return nf == 3 ? 1 : 3;
    if (nf == 4) return 2;
    if (nf == 6) return 4;
    return has_tri ? 6 : 5;  // 5 faces: wedge (two triangles) or pyramid
}

void write_dat(const psst_grid &g, const double *prim, const double *rho, const std::string &path) {
    File out(path, "dat");
    const int64_t nv = g.nvol;
    const struct {
        int id;
        const double *v;
    } vars[] = {{1, prim}, {3, prim + nv}, {101, rho}, {111, prim + 2 * nv}, {112, prim + 3 * nv},
                {113, g.dim == 3 ? prim + 4 * nv : nullptr}};
    for (const auto &var : vars) {
        if (!var.v) continue;
        int64_t first = 0, last = 0;
        for (const VZone &z : g.vz) {  // ascending zone id, as the reference's std::map
            if (z.bc == 32) continue;
            first = last;
            last += z.count;
            std::fprintf(out.f, "(\t 300 \t(\t %d \t %" PRId64 " \t 1 \t 0 \t 0 \t %" PRId64 " \t %" PRId64 " \t) \n(\n",
                         var.id, z.id, first + 1, last);
            for (int64_t j = 0; j < z.count; ++j) std::fprintf(out.f, "%.11f\n", var.v[z.first + j]);
            std::fprintf(out.f, ")\n\n");
        }
    }
}

// One tree section per parent zone (private_write_cell_tree / _face_tree,
// :266-351). Children hang off the parent entity whatever section listed them
// (create_finite_volume_grid, psstAnsysGridReader.cpp:788-821); a zone's child
// zone is the one the last section naming it as parent gave.
void write_trees(FILE *f, const RawMesh &m, const std::map<int64_t, const Zone *> &zones, int op) {
    const int64_t parent_bc = op == 58 ? 32 : 31;
    std::map<int64_t, std::vector<int64_t>> kids;  // parent file index -> children
    std::map<int64_t, int64_t> child_zone;
    for (const RawMesh::Tree &t : m.trees) {
        if (t.op != op) continue;
        child_zone[t.parent_zone] = t.child_zone;
        for (int64_t i = 0; i + 1 < (int64_t)t.ptr.size(); ++i) {
            std::vector<int64_t> &k = kids[t.first + i];
            k.insert(k.end(), t.kids.begin() + t.ptr[i], t.kids.begin() + t.ptr[i + 1]);
        }
    }
    bool header = false;
    for (auto &kv : zones) {
        const Zone &z = *kv.second;
        if (z.bc != parent_bc) continue;
        if (!header) std::fprintf(f, op == 58 ? "(0 \"Cells Trees:\")\n" : "(0 \"Faces Trees:\")\n");
        header = true;
        auto cz = child_zone.find(z.id);
        std::fprintf(f, "(%d (%" PRIx64 " %" PRIx64 " %" PRIx64 " %" PRIx64 ")(\n", op, z.first, z.last, z.id,
                     cz == child_zone.end() ? (int64_t)0 : cz->second);
        for (int64_t i = 0; i < z.size; ++i) {
            auto it = kids.find(z.first + i);
            const int64_t nk = it == kids.end() ? 0 : (int64_t)it->second.size();
            std::fprintf(f, " %" PRIx64, nk);
            for (int64_t j = 0; j < nk; ++j) std::fprintf(f, " %" PRIx64, it->second[j]);
            std::fprintf(f, "\n");
        }
        std::fprintf(f, "))\n\n");
    }
}

void write_cas(const psst_grid &g, const RawMesh &m, const std::string &path) {
    std::map<int64_t, const Zone *> zones;  // ascending id
    for (const Zone &z : m.zones) zones[z.id] = &z;
    File out(path, "cas");
    FILE *f = out.f;
    const int dim = m.dim;
    const int64_t nvert = (int64_t)m.verts.size() / dim;
    std::fprintf(f, "(0 \"Dimension:\")\n(2 %d)\n\n", dim);
    std::fprintf(f, "(0 \"Vertices:\")\n");
    std::fprintf(f, "(10 (0 1 %" PRIx64 " 1 %x))\n", nvert, dim);
    std::fprintf(f, "(10 (1 1 %" PRIx64 " 1 %x)(\n", nvert, dim);
    for (int64_t i = 0; i < nvert; ++i) {
        for (int k = 0; k < dim; ++k) std::fprintf(f, " %.20e ", m.verts[(size_t)i * dim + k]);
        std::fprintf(f, "\n");
    }
    std::fprintf(f, "))\n\n");
    const int64_t nfile_faces = (int64_t)m.face_c0.size();
    std::fprintf(f, "(0 \"Faces:\")\n(13 (0 1 %" PRIx64 " 0))\n", nfile_faces);
    for (auto &kv : zones) {
        const Zone &z = *kv.second;
        if (z.bc == 1 || z.bc == 32) continue;  // face zones: interior, boundary and parent faces
        std::fprintf(f, "(13 (%" PRIx64 " %" PRIx64 " %" PRIx64 " %" PRIx64 " 0)(\n", z.id, z.first, z.last, z.bc);
        for (int64_t j = 0; j < z.size; ++j) {
            const int64_t loc = z.first + j - 1;
            const int64_t b = m.face_ptr[loc], e = m.face_ptr[loc + 1];
            std::fprintf(f, " %" PRIx64 " ", e - b);
            for (int64_t q = b; q < e; ++q) std::fprintf(f, " %" PRIx64 " ", m.face_nodes[q]);
            std::fprintf(f, " %" PRIx64 "  %" PRIx64 " \n", m.face_c0[loc], m.face_c1[loc]);
        }
        std::fprintf(f, "))\n\n");
    }
    const int64_t ncell = (int64_t)m.cell_zone.size();
    std::fprintf(f, "(0 \"Cells:\")\n(12 (0 1 %" PRIx64 " 0))\n", ncell);
    std::vector<int64_t> types = m.cell_type;
    if ((int64_t)types.size() != ncell) {  // infer from the faces
        std::vector<int> nf(ncell, 0);
        std::vector<char> tri(ncell, 0);
        for (int64_t i = 0; i < nfile_faces; ++i)
            for (int64_t c : {m.face_c0[i], m.face_c1[i]})
                if (c > 0) {
                    nf[c - 1] += 1;
                    if (m.face_ptr[i + 1] - m.face_ptr[i] == 3) tri[c - 1] = 1;
                }
        types.resize(ncell);
        for (int64_t c = 0; c < ncell; ++c) types[c] = cell_type_from_faces(dim, nf[c], tri[c]);
    }
    for (auto &kv : zones) {
        const Zone &z = *kv.second;
        if (z.bc != 1 && z.bc != 32) continue;
        std::fprintf(f, "(12 (%" PRIx64 " %" PRIx64 " %" PRIx64 " %" PRIx64 " 0)(\n", z.id, z.first, z.last, z.bc);
        for (int64_t i = 0; i < z.size; ++i) {
            if (i % 9 == 0 && i != 0) std::fprintf(f, "\n");
            std::fprintf(f, " %" PRIx64, types[z.first + i - 1]);
        }
        std::fprintf(f, "\n))\n\n");
    }
    write_trees(f, m, zones, 58);
    write_trees(f, m, zones, 59);
    std::fprintf(f, "(0 \"Zones:\")\n");
    for (auto &kv : zones)
        if (kv.second->bc == 1)
            std::fprintf(f, "(39 (%" PRId64 " %s %s)())\n\n", kv.first, bc_name(1), kv.second->name.c_str());
    for (auto &kv : zones)
        if (kv.second->bc != 1 && kv.second->bc != 31 && kv.second->bc != 32)
            std::fprintf(f, "(39 (%" PRId64 " %s %s)())\n\n", kv.first, bc_name(kv.second->bc), kv.second->name.c_str());
    (void)g;
}

}  // namespace

extern "C" psst_status psst_write_fluent(const psst_grid *g, const double *prim, const double *rho,
                                         const char *prefix) {
    try {
        if (!g || !prim || !rho || !prefix) raise(PSST_ERR_ARG, "psst_write_fluent: null argument");
        if (!g->raw) raise(PSST_ERR_ARG, "psst_write_fluent: the grid carries no mesh (merged grid)");
        write_dat(*g, prim, rho, std::string(prefix) + ".dat");
        write_cas(*g, *g->raw, std::string(prefix) + ".cas");
        return PSST_OK;
    } catch (const Error &e) {
        set_last_error(e.msg);
        return e.status;
    } catch (const std::bad_alloc &) {
        set_last_error("out of host memory");
        return PSST_ERR_ARG;
    }
}
