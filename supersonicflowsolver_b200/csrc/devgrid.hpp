// Device-side views shared by the host driver (solver.cpp) and the kernels.
// Plain structs of device pointers, passed to kernels by value.
//
// Per-cell and per-face data that kernels gather through an index are stored
// as 16-byte-aligned records (one or a few 128-bit loads per gather); data
// read only at the thread's own index stay structure-of-arrays (coalesced).
#pragma once
#include <cstdint>

namespace psst {

// Primitive state of a volume: p, T, rho, u0, u1, (u2), padding.
template <typename R>
struct alignas(16) CellRec {
    R v[8];
};
enum { RP = 0, RT = 1, RRHO = 2, RU = 3 };

// Gradients of u.., p, T (g[var * DIM + k]); with a cell limiter (MUSCL,
// limiters 4/5) each variable's gradient is stored already multiplied by its
// limiter psi. 64 bytes in 3D FP32 (15 values + padding).
template <typename R, int DIM>
struct alignas(16) GradRec {
    R g[(DIM + 2) * DIM];
};

// Face: neighbours (device ids), area, unit normal (FP64: geometry is kept in
// FP64 on both paths), and the reconstruction offsets: x_f - x_c0 and
// x_f - x_c1 for cell-limited MUSCL, or x_c0 - x_c1 in o0 for the
// Darwish-Moukalled reconstruction. Offsets are formed in FP64 on the host
// and rounded once to R (exact on the FP64 path).
template <typename R, int DIM>
struct alignas(16) FaceRec {
    int32_t c0, c1;
    double S;
    double n[DIM];
    R o0[DIM];
    R o1[DIM];
};

// Output of the face pass for one face: flux * area (DIM+2), then the face's
// local-time-step terms: for LocalAccTime1 the two neighbours' normal
// velocities and the mean sound speed (the face area comes from
// DevGrid::csr_s); for LocalAccTime2 S |n_k| (DIM values from Q0). The normal
// velocities are kept per component (u_k n_k, NQ = DIM per side) on the FP64
// path, because the reference adds the neighbour's components one at a time
// onto a value carried over from the previous face
// (psstLocalTimeCalculation.cpp:117-124), and as their sums (NQ = 1) on the
// FP32 path: 12 values (96 bytes) in FP64, 8 (32 bytes) in FP32.
#ifndef PSST_FACEOUT_COMPACT
#define PSST_FACEOUT_COMPACT 1
#endif
template <typename R, int DIM>
struct alignas(16) FaceOut {
    static constexpr bool COMPACT = sizeof(R) == 4 && PSST_FACEOUT_COMPACT;
    static constexpr int NV = DIM + 2;
    static constexpr int NQ = COMPACT ? 1 : DIM;
    static constexpr int Q0 = NV, Q1 = NV + NQ, CN = NV + 2 * NQ;
    R v[COMPACT ? 8 : 12];
};

struct DevGrid {
    int32_t nint;     // interior cells: device ids [0, nint)
    int32_t nghost;   // ghost cells: device ids [nint, nint + nghost)
    int32_t nall;     // nint + nghost
    int32_t nface;    // active faces (zone 31 excluded); interior faces first
    int32_t nfi;      // interior faces: device ids [0, nfi)
    const void *frec;         // [nface] FaceRec<R, DIM>
    const double *beta;       // [nface] Green-Gauss interpolation weight (reference table)
    const double *V;          // [nint] cell volume
    const double *xc;         // [dim][nall] centroid (ghost: its face centre); least squares only
    const int32_t *csr_ptr;   // [nint+1]
    int32_t kuni;             // K if every interior cell has K CSR entries (csr_ptr[c] = K c), else 0
    const int32_t *csr_ent;   // face << 1 | side, sorted by the reference's face-loop order
    const int32_t *csr_nb;    // the cell across each csr_ent face (saves a dependent load)
    const void *csr_s;        // R per csr_ent: the face's area, rounded to R (LocalAccTime1)
    const uint64_t *wperm;    // [nint] 4-bit slots: k-th face of the cell's own face order
    const double *lsq_r;      // [3 (2D) or 7 (3D)][nint] least-squares coefficients (reference table)
    const double *vk_eps2;    // [nint] Venkatakrishnan epsilon^2 = (K h)^3, h = V^(1/dim)
    // Green-Gauss on meshes of 4 faces per cell (tets, quads), else null; per
    // CSR entry of cell c (slots 4c..4c+3), component-major [comp][4 nint]:
    //  FP32 [2 dim + 1]: sign * S/V * n_k (dim values, sign -1 on side 0), the
    //    weight of the neighbour's value in the face value (1 - beta on side 0,
    //    beta on side 1), the face offsets x_f - x_c of the cell's side;
    //  FP64 [2 dim + 2]: sign * (S / V), n_k (dim values), beta, the offsets --
    //    the values the face records hold, so the arithmetic is unchanged
    const void *gcoef;
    const int32_t *rank;      // [nint] position in the reference's interior update order
    const int32_t *gptr;      // [nint+1] ghosts of each interior cell (ghost index space)
    const int32_t *g_nb;      // [nghost] interior neighbour of each ghost
    const int32_t *g_face;    // [nghost] face of each ghost
    const int32_t *g_zone;    // [nghost] boundary zone slot
    const int32_t *z_dyn, *z_therm;  // [nzone] boundary ids
    const double *z_u;        // [nzone][3]
    const double *z_p, *z_T;  // [nzone]
    const int32_t *lvl_cells; // [nint] cells grouped by level (sequential LocalAccTime1)
    const int32_t *lvl_ptr;   // [nlevels+1]
    int32_t nlevels;
    // launch shapes (threads per block: 64, 128 or 256) of the gradient, face
    // and cell passes; set by the solver, tuned by psst_solver_autotune
    int32_t blk_grad, blk_face, blk_cell;
    // merged grids only (null otherwise): case of every cell (ghosts included)
    // and the per-case run flag; cells of a stopped case keep their state
    int32_t ncase;
    const int32_t *cell_case;    // [nall]
    const int32_t *face_case;    // [nface]
    const int32_t *case_active;  // [ncase]
};

template <typename R>
struct DevState {
    CellRec<R> *rec;  // [nall]
};

template <typename R>
struct DevWork {
    double *w, *pw;      // [dim+2][nint] conservative state, previous-stage state
    void *grec;          // [nint] GradRec<R, DIM>
    void *fout;          // [nface] FaceOut<R, DIM>, written by the face pass
    R *res;              // [dim+2][nint] residual (stage-by-stage API only)
    double *dt;          // [nint]
    double *linf;        // [n_iter][dim+2] max over stages and cells of |res|
    double *l2;          // [n_iter][dim+2]
    double *l2part;      // [stages][nblocks][2][dim+2] per-block sum of res^2 and max |res|
    double *l2mid;       // [kNormReduceBlocks][stages][2][dim+2] first level of k_norm_reduce
    unsigned int *ticket;  // [1] blocks of k_norm_reduce finished in the current launch
    int32_t *err;        // [4] error word, face id, cell id, code
    unsigned long long *case_linf;  // merged grids: [n_iter][ncase][dim+2] max |res| (bits of a
                                    // non-negative double, so integer max = numeric max)
};

struct Gas {
    double rm, cp, cv, gamma;
};

// Per-case stop rule of merged grids, evaluated on the device after every
// iteration: each component of a case's residual column is normalised by its
// maximum over the case's first scale_iters iterations (or by a given
// scale); the case stops at the first iteration where every normalised
// component is <= drop, or when it has run cap iterations.
struct CaseStop {
    double drop;
    int32_t scale_iters;  // 0: the scales are given
    int32_t *active;      // [ncase] the run flags the kernels read (DevGrid::case_active)
    int32_t *rows;        // [ncase] iterations run under the rule
    int32_t *conv_at;     // [ncase] iteration of the drop, 0 while not reached
    const int32_t *cap;   // [ncase] most iterations a case runs
    double *scale;        // [ncase][dim+2]
};

// Device-side state of a run-to-stop launch (psst_solver_run_to_stop): a CUDA
// graph whose while-loop node repeats a captured block of iterations; the
// block's last kernel appends its residual columns to the history, counts
// the iterations and sets the loop condition.
struct LoopCtl {
    int64_t done;                 // iterations run by this launch so far
    int64_t max_iter;             // no further block once done >= max_iter
    int64_t cap_rows;             // rows of the history
    double *hist_linf, *hist_l2;  // [cap_rows][dim+2]
};

// Wavefront schedule of the sequential LocalAccTime1 (the reference's in-loop
// order, psstFiniteVolumeGrid.cpp:317-323) over many RK stages in one
// persistent launch. Cell c's level exceeds the level of every interior
// neighbour updated before it; D is the largest level difference across an
// interior face and P = D + 1. Operation m of the call (a gradient or an RK
// stage) of cell c runs at step P m + level(c): every input it needs -- the
// previous operation of each neighbour and this operation of each earlier
// neighbour -- is then at least one step (one grid barrier) old. Work items
// are chunks (at most one block) of one level; they are ordered by level mod
// P, then level, so the items of one step are contiguous.
struct WfSched {
    int32_t period;          // P
    int32_t nlevels, nitems;
    const int32_t *cells32;     // [nitems][32] the cells of each item (-1: empty slot)
    const uint32_t *lowmask;    // [nint] bit q: the cell across CSR entry q was updated
                                // before this cell in the reference's order
    const int32_t *item_level;  // [nitems]
    const int32_t *lvl_items;   // [2 nlevels] item range [first, end) of each level
    double *ipart;              // [2][nitems][2 NV] per item: sum res^2, max |res| (by operation parity)
    double *acc;                // [nacc][2 NV] per RK stage: the same over the levels folded so far
    int32_t nacc;
    void *grec2;                // second gradient buffer (gradients by iteration parity)
    unsigned *sync;             // grid barrier: arrivals, generation, abort flag (one 128-byte line each)
};

template <typename R>
struct WfArgs {
    DevGrid g;
    CellRec<R> *buf[2];  // state buffers; a stage reads one and writes the other
    DevWork<R> wk;
    void *gbuf[2];       // gradient buffers of the iterations n-1, n-3, .. ([0]) and n-2, .. ([1])
    WfSched sc;
    Gas gas;
    double cfl;
    double alpha[16];
    int32_t nst;      // RK stages per iteration
    int32_t nopi;     // operations per iteration: nst, + 1 with a gradient
    int64_t nops;     // operations of the call
    int32_t n_iter;
    int32_t flux, grad, celllim;
    int32_t in_buf;   // buffer holding the call's input state
    uint64_t wait_ns; // bound of each grid-barrier wait (0: do not wait)
};

}  // namespace psst
