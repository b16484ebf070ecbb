// Internal host-side data model of libpsst_b200 (not part of the C ABI).
//
// psst_grid holds the finite-volume grid in the reference's storage order
// (volume zones and face zones in ascending zone id, psstFiniteVolumeGrid.h:21-23)
// as flat arrays, plus everything the device layout is derived from.
#pragma once

#include <algorithm>
#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "psst_b200.h"

namespace psst {

// Thrown inside the library only; every C entry point converts it to a status.
struct Error {
    psst_status status;
    std::string msg;
};
[[noreturn]] void raise(psst_status st, const std::string &msg);
void set_last_error(const std::string &msg);

struct Zone {  // psstSimpleStorage (psstAnsysGridReader.h)
    int64_t id = 0, first = 0, last = 0, bc = 0, size = 0;
    std::string name;
};

// What a Fluent file says (psstAnsysInputGrid).
struct RawMesh {
    int dim = 0;
    std::vector<double> verts;            // nvert * dim
    std::vector<int64_t> face_ptr{0};     // per file face, into face_nodes
    std::vector<int64_t> face_nodes;      // 1-based vertex ids
    std::vector<int64_t> face_c0, face_c1;  // 1-based file cell ids, 0 = none
    std::vector<int64_t> cell_zone;       // per file cell
    std::vector<int64_t> cell_type;       // per file cell (Fluent type; empty when not given)
    std::vector<Zone> zones;              // file order (first appearance)
    struct Tree {                         // a 58 (cells) or 59 (faces) section
        int op = 0;
        int64_t first = 0, last = 0, parent_zone = 0, child_zone = 0;
        std::vector<int64_t> ptr, kids;   // children of parent first + i: kids[ptr[i], ptr[i+1])
    };
    std::vector<Tree> trees;
    int64_t zone_slot(int64_t id);        // find or append
};

RawMesh read_fluent(const std::string &path);

struct VZone {
    int64_t id, bc, first, count;  // volumes [first, first+count)
    std::string name;
    int dyn = 0, therm = 0;        // .bvp / .btq ids
    double u[3] = {0, 0, 0}, p = 0, T = 0;
};
struct FZone {
    int64_t id, bc, first, count;
    std::string name;
};

struct psst_grid_impl;
}  // namespace psst

struct psst_grid {
    int dim = 0;
    std::vector<psst::VZone> vz;  // ascending id
    std::vector<psst::FZone> fz;  // ascending id
    int64_t nvol = 0, nface = 0, ninterior = 0, nghost = 0;
    std::vector<uint8_t> vol_boundary;   // ghost flag
    std::vector<int32_t> vol_vz;         // volume -> vz slot
    std::vector<int64_t> vf_ptr, vf_idx; // per volume face list, reference wiring order
    std::vector<double> V, xc;           // nvol, nvol*dim
    std::vector<int64_t> f_c0, f_c1;     // nface, volume index or -1
    std::vector<int32_t> f_fz;           // face -> fz slot
    std::vector<double> S, n, xf, beta;  // nface, nface*dim, nface*dim, nface
    double min_vol = -1.0;
    int max_faces = 0;
    // initial state holder filled by psst_case_read (SoA p,T,u..)
    std::vector<double> prim0;
    double ref_vel = 0.0;
    // the mesh as read (vertices, file faces, cell types, file zone ranges):
    // what psst_write_fluent writes back; null for merged grids
    std::shared_ptr<const psst::RawMesh> raw;
    // merged grids (psst_grid_merge): volumes [case_vol_ptr[i], case_vol_ptr[i+1])
    // belong to case i; empty for a single case
    std::vector<int64_t> case_vol_ptr;
};

namespace psst {
// Runs fn(begin, end) over [0, n) split into contiguous chunks on the host
// threads (PSST_HOST_THREADS, default: the hardware threads); small ranges run
// inline. If chunks throw, the exception of the lowest failing chunk is
// rethrown after all have finished, which is the first error a sequential
// loop over [0, n) would have raised.
void parallel_for(int64_t n, const std::function<void(int64_t, int64_t)> &fn);
int host_threads();
// Runs fn(t) for t in [0, ntasks), each task on its own host thread.
void parallel_tasks(int ntasks, const std::function<void(int)> &fn);

// Sorts v by cmp, a strict total order (make keys unique, e.g. by an index,
// so that the result equals a stable sort): chunks sorted in parallel, then
// merged pairwise in parallel.
template <class T, class Cmp>
void parallel_sort(std::vector<T> &v, Cmp cmp) {
    const int64_t n = (int64_t)v.size();
    int chunks = 1;
    while (chunks * 2 <= host_threads() && n / (chunks * 2) >= 65536) chunks *= 2;
    if (chunks == 1) {
        std::sort(v.begin(), v.end(), cmp);
        return;
    }
    std::vector<int64_t> cut((size_t)chunks + 1);
    for (int i = 0; i <= chunks; ++i) cut[(size_t)i] = n * i / chunks;
    parallel_tasks(chunks, [&](int t) { std::sort(v.begin() + cut[(size_t)t], v.begin() + cut[(size_t)t + 1], cmp); });
    std::vector<T> tmp((size_t)n);
    for (int width = 1; width < chunks; width *= 2) {
        parallel_tasks(chunks / (2 * width), [&](int p) {
            const int64_t a = cut[(size_t)(2 * p * width)], m = cut[(size_t)((2 * p + 1) * width)],
                          b = cut[(size_t)((2 * p + 2) * width)];
            std::merge(v.begin() + a, v.begin() + m, v.begin() + m, v.begin() + b, tmp.begin() + a, cmp);
        });
        v.swap(tmp);
    }
}
psst_grid *build_grid(const RawMesh &m);
constexpr int kLsqNR = 7;  // least-squares coefficients per cell: r11 r12 r22 (2D), + r13 r23 r33 beta (3D)
std::vector<double> lsq_table(const psst_grid &g);  // kLsqNR per zone-local interior index
}  // namespace psst
