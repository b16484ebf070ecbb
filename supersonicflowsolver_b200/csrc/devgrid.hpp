// Device-side views shared by the host driver (solver.cpp) and the kernels.
// Plain structs of device pointers, passed to kernels by value.
#pragma once
#include <cstdint>

namespace psst {

struct DevGrid {
    int32_t nint;     // interior cells: device ids [0, nint)
    int32_t nghost;   // ghost cells: device ids [nint, nint + nghost)
    int32_t nall;     // nint + nghost
    int32_t nface;    // active faces (zone 31 excluded); interior faces first
    int32_t nfi;      // interior faces: device ids [0, nfi)
    const int32_t *c0, *c1;   // [nface] device cell ids of neighbour 0 / 1
    const double *S;          // [nface] face area
    const double *n;          // [dim][nface] unit normal, neighbour 1 -> neighbour 0
    const double *xf;         // [dim][nface] face centre
    const double *beta;       // [nface] Green-Gauss interpolation weight (reference table)
    const double *V;          // [nint] cell volume
    const double *xc;         // [dim][nall] centroid (ghost: its face centre)
    const int32_t *csr_ptr;   // [nint+1]
    const int32_t *csr_ent;   // face << 1 | side, sorted by the reference's face-loop order
    const uint64_t *wperm;    // [nint] 4-bit slots: k-th face of the cell's own face order
    const double *lsq_r;      // [3][nint] 2D least-squares coefficients (reference table)
    const double *vk_eps2;    // [nint] Venkatakrishnan epsilon^2 = (K h)^3, h = V^(1/dim)
    const int32_t *rank;      // [nint] position in the reference's interior update order
    const int32_t *g_nb;      // [nghost] interior neighbour of each ghost
    const int32_t *g_face;    // [nghost] face of each ghost
    const int32_t *g_zone;    // [nghost] boundary zone slot
    const int32_t *z_dyn, *z_therm;  // [nzone] boundary ids
    const double *z_u;        // [nzone][3]
    const double *z_p, *z_T;  // [nzone]
    const int32_t *lvl_cells; // [nint] cells grouped by level (sequential LocalAccTime1)
    const int32_t *lvl_ptr;   // [nlevels+1]
    int32_t nlevels;
};

template <typename R>
struct DevState {
    R *p, *T, *rho, *u;  // [nall], u: [dim][nall]
};

template <typename R>
struct DevWork {
    double *w, *pw;      // [dim+2][nint] conservative state, previous-stage state
    R *grad;             // [dim+2][dim][nint] gradients of u.., p, T
    R *lim;              // [dim+2][nint] cell limiter (limiters 4/5)
    R *fs;               // [dim+2][nface] flux * area per face
    R *res;              // [dim+2][nint] residual (stage-by-stage API only)
    double *dt;          // [nint]
    unsigned long long *linf;  // [n_iter][dim+2] max |res| (bit pattern of a non-negative double)
    double *l2part;      // [nblocks][dim+2] partial sums of res^2
    double *l2;          // [n_iter][dim+2]
    int32_t *err;        // [4] error word, face id, cell id, code
};

struct Gas {
    double rm, cp, cv, gamma;
};

}  // namespace psst
