/* psst_b200.h — C ABI of libpsst_b200.so, the B200 (sm_100a) implementation of
 * PSST's explicit finite-volume residual/update loop.
 *
 * The reference exposes this path as C++ strategy interfaces selected by the
 * factory in psstGridFV::solver_parameters (psstFiniteVolumeGrid.cpp:36-194)
 * and driven by psstGridFV::explicit_solve (psstFiniteVolumeGrid.cpp:248-401).
 * Per-face virtual calls cannot cross a host/device boundary, so this ABI cuts
 * at stage and iteration granularity. Every entry point below names the
 * reference interface it replaces.
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, status codes. No exceptions cross the
 *    ABI; a failing call returns a non-zero psst_status and psst_last_error()
 *    returns its message (thread-local). Messages reuse the reference's texts
 *    where the reference reports the same condition.
 *  - Buffers passed in are caller-owned and copied; buffers passed out are
 *    caller-allocated with the stated size.
 *  - Volumes are numbered in the reference's storage order: all volume zones in
 *    ascending zone id (std::map order), interior cells and ghost cells alike,
 *    each zone in its own index order (psstFiniteVolumeGrid.h:23). Faces are
 *    numbered in the reference's face-loop order: face zones in ascending id,
 *    each in file order (psstFiniteVolumeGrid.h:21).
 *  - Primitive state arrays are SoA: p[nvol], T[nvol], u[dim][nvol] packed as
 *    prim[(2 + dim) * nvol] = {p..., T..., u0..., u1..., (u2...)}.
 *  - A psst_solver owns its device memory and one CUDA stream; it is not
 *    thread-safe. Calls on one solver are stream-ordered.
 */
#ifndef PSST_B200_H
#define PSST_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSST_B200_ABI_VERSION 1

typedef enum psst_status {
    PSST_OK = 0,
    PSST_ERR_ARG = 1,         /* invalid argument (reference: std::invalid_argument) */
    PSST_ERR_IO = 2,          /* file missing/unreadable */
    PSST_ERR_FORMAT = 3,      /* malformed mesh or setup file */
    PSST_ERR_CUDA = 4,        /* CUDA runtime error, or no usable device */
    PSST_ERR_NONFINITE = 5,   /* non-finite residual or state detected on the device */
    PSST_ERR_FLUX = 6,        /* HLL/HLLC wave speeds not ordered (ConvectiveFlow.cpp:283-286, 582-585) */
    PSST_ERR_TIMEOUT = 7,     /* a bounded device-side wait ran out */
    PSST_ERR_UNSUPPORTED = 8, /* option the reference does not support either */
    PSST_ERR_STATE = 9        /* call order violated (e.g. no state set) */
} psst_status;

typedef struct psst_grid psst_grid;     /* host mesh + geometry, reference storage order */
typedef struct psst_solver psst_solver; /* device state for one case */

/* Message of the last failing call on this thread ("" if none). */
const char *psst_last_error(void);
int psst_abi_version(void);

/* ------------------------------------------------------------------------ */
/* Mesh                                                                      */
/* ------------------------------------------------------------------------ */

/* Reads a Fluent ASCII mesh (.msh/.cas; LF or CRLF) and builds the finite-volume
 * grid: ghost cell per boundary face, face/volume wiring, FP64 geometry.
 * Replaces psstAnsysDirector::construct_grid (psstAnsysGridReader.cpp:1308-1317)
 * + psstAnsysInputGrid::create_finite_volume_grid (psstAnsysGridReader.cpp:688-907)
 * + psstFace::initialize / psstVolume::initialize
 *   (psstFiniteVolumeGridTools.cpp:397-505, 709-827). */
psst_status psst_grid_read_fluent(const char *path, psst_grid **out);

/* Same grid from in-memory Fluent-style arrays (for callers that already hold
 * the mesh, e.g. a reference-side shim or a mesh generator). Faces are given in
 * file order grouped in zones; cells are given per cell zone.
 *  face_nodes: 0-based vertex ids, face_ptr[nface+1] offsets into it;
 *  face_c0/face_c1: 0-based cell ids, -1 = none (Fluent's 0);
 *  zones: for each zone in file order, id, Fluent bc type, first and last
 *  1-based index (cells or faces, per bc type) and a name. */
typedef struct psst_zone_desc {
    int64_t id, bc_type, first, last;
    const char *name;
} psst_zone_desc;

typedef struct psst_fluent_desc {
    int32_t dim;
    int64_t nvert;
    const double *verts; /* nvert * dim */
    int64_t nface;
    const int64_t *face_ptr;   /* nface + 1 */
    const int64_t *face_nodes; /* face_ptr[nface] */
    const int64_t *face_c0, *face_c1;
    int64_t ncell;
    int32_t nzone;
    const psst_zone_desc *zones;
} psst_fluent_desc;

psst_status psst_grid_from_fluent(const psst_fluent_desc *desc, psst_grid **out);

typedef struct psst_grid_info {
    int32_t dim;
    int64_t nvol;      /* all volumes (interior + ghost) */
    int64_t ninterior; /* volumes of interior cell zones (bc 1) */
    int64_t nghost;    /* ghost volumes (one per boundary face) */
    int64_t nface;     /* all faces of all face zones */
    int32_t max_faces_per_cell;
    double min_vol; /* psstGridFV::min_vol (psstAnsysGridReader.cpp:886-905) */
} psst_grid_info;

psst_status psst_grid_get_info(const psst_grid *g, psst_grid_info *out);

/* Copies a named array in reference order. Doubles: "vol_V", "vol_x"[nvol*dim],
 * "face_S", "face_n"[nface*dim], "face_x"[nface*dim], "face_beta". Int64:
 * "face_c0", "face_c1" (volume index, -1 none), "vol_zone", "vol_boundary",
 * "vol_bc" (zone type: 1 interior, 32 parent cell, else a ghost's boundary
 * type), "face_zone". count = element count of the out buffer. */
psst_status psst_grid_get_array(const psst_grid *g, const char *name, void *out, int64_t count);

void psst_grid_free(psst_grid *g);

/* Writes <prefix>.cas and <prefix>.dat as psstAnsysOutputManager::output_data
 * does (psstOutputManager.cpp:35-397): the mesh as read (vertices, faces with
 * their file neighbours, cell types, zones) and p, T, rho, u.. of every
 * volume zone. prim: state in the layout of psst_solver_get_state; rho[nvol]:
 * densities (psst_solver_get_array "rho"). Grids built by psst_grid_merge
 * carry no mesh and are rejected. */
psst_status psst_write_fluent(const psst_grid *g, const double *prim, const double *rho, const char *prefix);

/* No counterpart in the reference (it solves one case per process). Merges n
 * case grids, each already set up by psst_case_read, into one grid that is
 * their disjoint union, so that one solver advances all of them with every
 * launch. Volumes, faces and zones follow case after case, each case in its
 * own reference order; zone id z of case i becomes i*1000000 + z and its name
 * gets "#i". Each case keeps its own geometry, boundary values and initial
 * state (returned in the merged prim layout by psst_case_read's holder), so
 * it evolves as it would alone. The inputs stay owned by the caller. Merged
 * grids need Green-Gauss gradients (the reference's least-squares table is
 * indexed across zones) and, for LocalAccTime1, lc1_mode JACOBI. */
psst_status psst_grid_merge(const psst_grid *const *grids, int32_t n, psst_grid **out);

/* Number of cases of a grid (1 unless merged) and, if case_vol_ptr is not
 * NULL, the ncase+1 volume offsets of the cases. */
psst_status psst_grid_case_count(const psst_grid *g, int32_t *ncase, int64_t *case_vol_ptr);

/* Initial state of a merged grid in the prim layout of psst_solver_set_state
 * (the cases' psst_case_read states, concatenated per variable); count =
 * (2+dim)*nvol. */
psst_status psst_grid_initial_state(const psst_grid *g, double *prim, int64_t count);

/* ------------------------------------------------------------------------ */
/* Case setup                                                                */
/* ------------------------------------------------------------------------ */

enum { PSST_FLUX_AUSM = 1, PSST_FLUX_HLL = 2, PSST_FLUX_HLLC = 3 };
enum { PSST_GRAD_GREEN_GAUSS = 1, PSST_GRAD_LEAST_SQUARES = 2 };
/* 1..3 are the reference's psstScalarLimiters (DM reconstruction); 4 and 5 are
 * cell-based MUSCL limiters the reference does not have. */
enum {
    PSST_LIMITER_VANALBADA = 1,
    PSST_LIMITER_MINMOD = 2,
    PSST_LIMITER_VANLEER = 3,
    PSST_LIMITER_BARTH_JESPERSEN = 4,
    PSST_LIMITER_VENKATAKRISHNAN = 5
};
/* Local time step: 0 psstUniformTime, 1 psstLocalAccTime1, 2 psstLocalAccTime2 */
enum { PSST_TIME_UNIFORM = 0, PSST_TIME_LOCAL1 = 1, PSST_TIME_LOCAL2 = 2 };
/* lc1_mode for PSST_TIME_LOCAL1: the reference evaluates it inside the update
 * loop, so each cell sees neighbours already updated in the same stage
 * (psstFiniteVolumeGrid.cpp:323). SEQUENTIAL reproduces that exactly with a
 * level schedule; JACOBI uses stage-start values for every cell. */
enum { PSST_LC1_SEQUENTIAL = 0, PSST_LC1_JACOBI = 1 };

typedef struct psst_scheme {
    int32_t flux, order, grad, limiter;
    int32_t lc, lc1_mode;
    int32_t rk_level;
    double rk[16];
    double cfl;
    double rm, cp, cv, gamma; /* gas constants as psstGridFV derives them */
    double ref_vel;           /* psstUniformTime reference speed */
    double venkat_k;          /* Venkatakrishnan K (limiter 5) */
    int32_t precision;        /* 64: FP64 parity path; 32: FP32 production path */
    int32_t renumber;         /* 1: reorder cells along a Hilbert curve on the device */
    int64_t iter, max_iter, iter_step; /* reference counters (.inp lines 4-5, .sav) */
} psst_scheme;

/* Reads <dir>/<name>.inp/.prop/.par (or .sav)/.bvp/.btq exactly as
 * psstGridFV::solver_parameters does (psstFiniteVolumeGrid.cpp:36-194,
 * 403-557, 559-604, 641-717). Boundary conditions are attached to the grid;
 * the scheme is returned; prim (may be NULL) receives the initial primitive
 * state of every volume including ghosts ((2+dim)*nvol doubles). */
psst_status psst_case_read(psst_grid *g, const char *dir, const char *name, psst_scheme *scheme,
                           double *prim);

/* Boundary conditions set directly (same ids as .bvp/.btq): dynamic 23, 26, 15,
 * 25; thermal 27, 25, 11, 18. u has dim entries (23), p (23, 25), T (27, 11). */
psst_status psst_grid_set_boundary(psst_grid *g, const char *zone_name, int dyn_id, const double *u,
                                   double p, int therm_id, double T);

/* ------------------------------------------------------------------------ */
/* Solver                                                                    */
/* ------------------------------------------------------------------------ */

/* Uploads grid and scheme to `device`. Replaces the strategy construction and
 * initialize() calls in solver_parameters (psstFiniteVolumeGrid.cpp:50-192). */
psst_status psst_solver_create(const psst_grid *g, const psst_scheme *scheme, int device,
                               psst_solver **out);

/* Sets the primitive state of all volumes and forms w as the explicit_solve
 * prologue does (psstFiniteVolumeGrid.cpp:279-300). */
psst_status psst_solver_set_state(psst_solver *s, const double *prim);

/* Reads back primitives ((2+dim)*nvol) and, if w != NULL, the conservative
 * state w[(dim+2)*nvol] (rho*u.., rho, rho*E; zero for ghosts). */
psst_status psst_solver_get_state(psst_solver *s, double *prim, double *w);

/* Binary checkpoint, next to the reference's .sav (psstFiniteVolumeGrid.cpp:
 * 606-639, read back at :559-604). The .sav keeps 11 decimals of p, T, u and
 * the restart recomputes rho and w, so a run resumed from it does not continue
 * exactly. The checkpoint holds, at full precision, the primitive records (p,
 * T, rho, u..) of every volume as the solver holds them, the FP64 conservative
 * state w and the iteration counter: N iterations, save, load into a solver
 * of the same grid, scheme and precision, M iterations equals N + M
 * iterations bit for bit. Format (native byte order): "PSSTCKP1", int32 dim,
 * int32 precision, int64 nvol, nint, iter; then doubles prim[(2+dim)*nvol]
 * (layout of psst_solver_get_state), rho[nvol], w[nvol*(dim+2)]. Loading
 * checks grid size and precision (PSST_ERR_FORMAT otherwise). */
psst_status psst_solver_save_checkpoint(psst_solver *s, const char *path);
psst_status psst_solver_load_checkpoint(psst_solver *s, const char *path);

/* psstInterfaceGradientCalc::calculate (psstGradCalculation.h:20;
 * psstGreenGauss .cpp:80-177, psstLeastSquare .cpp:268-368). For limiters 4/5
 * this also evaluates the cell limiter. */
psst_status psst_gradient_calculate(psst_solver *s);

/* psstInterfaceConvectiveFlow::calculate (psstConvectiveFlow.h:22): face fluxes
 * with the selected reconstruction/limiter, accumulated into per-cell residuals
 * in the reference's face-loop order. */
psst_status psst_convective_calculate(psst_solver *s);

/* Stage k of psstRungeKutta (psstFiniteVolumeGrid.cpp:312-366): local time
 * step (psstInterfaceLocalTime::calculate_at), w = prev_w - dt*a_k*res/V,
 * primitives, then ghost boundary conditions
 * (psstInterfaceBoundaryCondition::calculate_at). res_linf (may be NULL)
 * receives max|residual| per component over interior cells. */
psst_status psst_stage_update(psst_solver *s, int k, double *res_linf);

/* n_iter iterations of the explicit_solve loop body (psstFiniteVolumeGrid.cpp:
 * 305-367), launched back to back on the solver's stream. res_linf/res_l2 (may
 * be NULL) receive n_iter*(dim+2) values: the reference's residual columns
 * (max over stages and cells of |residual|) and RMS residuals. */
psst_status psst_explicit_solve(psst_solver *s, int n_iter, double *res_linf, double *res_l2);

/* Reads of device arrays, reference volume order: "rho"[nvol] (density of
 * every volume, ghosts included, as psst_write_fluent needs it),
 * "residual"[(dim+2)*nvol], "dt"[nvol], "grad_u"[nvol*dim*dim],
 * "grad_p"[nvol*dim], "grad_T"[nvol*dim] (with limiters 4/5 each gradient
 * multiplied by its cell limiter psi, the form the MUSCL reconstruction uses). */
psst_status psst_solver_get_array(psst_solver *s, const char *name, double *out, int64_t count);

/* Runs the solver's work on the given CUDA stream (cudaStream_t passed as a
 * pointer) instead of its own; NULL restores its own (non-blocking) stream,
 * so the legacy default stream is selected by its explicit handle,
 * cudaStreamLegacy. */
psst_status psst_solver_set_stream(psst_solver *s, void *stream);

/* Kernel launches issued by the last psst_explicit_solve call, and the
 * device-side duration (ms) of that call measured with CUDA events. */
psst_status psst_solver_last_stats(const psst_solver *s, int64_t *launches, double *device_ms);

/* Runs n_iter iterations like psst_explicit_solve, with a CUDA event pair
 * around every kernel launch, and returns per kernel kind the summed device
 * time (ms) and the launch count. Kinds: 0 gradient (+cell limiter), 1 face
 * pass (fluxes and time-step terms), 2 cell pass (residual, time step, RK
 * update; in the parallel modes also ghosts and the norms' block partials;
 * in the sequential mode's persistent launch the whole call), 3 ghost update
 * (stage-by-stage sequential mode), 4 residual norms (the parallel modes'
 * per-iteration reduction, the merged grids' stop rule, the stage-by-stage
 * sequential mode's per-stage finish). */
#define PSST_KERNEL_KINDS 5
psst_status psst_solver_profile(psst_solver *s, int n_iter, double *ms_per_kind, int64_t *launches_per_kind);

/* No counterpart in the reference (its loop is serial). Launch-shape tuner:
 * times n_iter iterations at 64, 128 and 256 threads per block on the
 * solver's own mesh and state, keeps the fastest shape for each of the
 * gradient, face and cell passes, and restores the state and iteration count,
 * so the next psst_explicit_solve continues from where it was. blocks (may be
 * NULL) receives the chosen shapes {gradient, face, cell}. The shapes change
 * no result except the last bits of the RMS column (its block partials follow
 * the cell-pass shape). Allocates a state-sized snapshot for the call. */
psst_status psst_solver_autotune(psst_solver *s, int n_iter, int *blocks);

/* Sets (set != NULL; 0 keeps an entry) and/or reads (get != NULL) the launch
 * shapes {gradient, face, cell}: 64, 128 or 256 threads per block (default
 * 256). */
psst_status psst_solver_launch_shape(psst_solver *s, const int *set, int *get);

/* ------------------------------------------------------------------------ */
/* Residual without any allocation                                           */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference. For callers that cannot allocate device
 * memory -- code running under an application or framework that owns every
 * device allocation (a pool or arena it hands out), or a solver embedded in a
 * host that forbids growing the device footprint after start-up -- and so
 * cannot create a solver object, since psst_solver_create allocates.
 *
 * Computes the first-order convective residual (the result of
 * psst_convective_calculate for order 1: HLL/HLLC/AUSM fluxes of unreconstructed
 * cell states, ghost physical flux on boundary faces, per-cell sums in the
 * order of each cell's CSR) from caller-owned DEVICE arrays into a
 * caller-owned device array. It calls no cudaMalloc/cudaFree and no allocating
 * library routine: the per-face flux buffer it needs is a fixed array compiled
 * into the library, sized for PSST_STATIC_MAX_FACES faces (5.24 MB, held on
 * every GPU that loads the library until the process exits). Larger meshes are
 * rejected with PSST_ERR_ARG.
 *
 *  volumes: interior cells are [0, nint), ghost cells [nint, nall);
 *  face_c0/face_c1 [nface]: neighbour volumes (a face with a ghost side is a
 *    boundary face); face_S [nface]; face_n [dim][nface] unit normals pointing
 *    from neighbour 1 into neighbour 0;
 *  csr_ptr [nint+1], csr_ent: per interior cell, (face << 1 | side) entries in
 *    the order the residual is summed (the reference's face-loop order);
 *  prim [(3+dim)][nall]: p, T, rho, u0, u1, (u2);
 *  residual [(dim+2)][nint] (output): rho*u.., rho, rho*E components.
 *
 * The first call on a device looks up the device address of the fixed buffer
 * (cudaGetSymbolAddress, with that device current); make that first call
 * before any stream capture. Every call shares the buffer and it keeps the
 * last call's contents; calls that overlap on the GPU (on different streams or
 * threads) race on it. The call synchronises `stream` (a cudaStream_t, NULL =
 * legacy default stream) to report a failed wave-speed ordering as
 * PSST_ERR_FLUX, like psst_convective_calculate. */
#define PSST_STATIC_MAX_FACES 131072
psst_status psst_convective_residual_static(int32_t dim, int32_t flux, int32_t nint, int32_t nall, int32_t nface,
                                            const int32_t *face_c0, const int32_t *face_c1, const double *face_S,
                                            const double *face_n, const int32_t *csr_ptr, const int32_t *csr_ent,
                                            const double *prim, double rm, double cp, double cv, double gamma,
                                            double *residual, void *stream);

/* No counterpart in the reference. With on != 0, each psst_explicit_solve
 * call is captured once as a CUDA graph (per iteration count and state-buffer
 * parity) and replayed afterwards: one launch per call instead of one per
 * kernel, for meshes small enough that launch latency dominates. Changing the
 * launch shapes drops the captured graphs. */
psst_status psst_solver_use_graphs(psst_solver *s, int on);

/* Merged grids only. Sets the run flag of every case (active[ncase], non-zero =
 * run): kernels skip the cells and faces of stopped cases, which keep their
 * state, and their residual columns read 0. */
psst_status psst_solver_set_active(psst_solver *s, const int32_t *active);

/* Merged grids only; no counterpart in the reference (it runs one case per
 * process until max_iter). A stop rule evaluated on the device after every
 * iteration, inside the launch sequence (and so inside a captured graph):
 * each component of a case's residual column (as psst_solver_case_residuals
 * returns it) is divided by its maximum over the case's first scale_iters
 * iterations under the rule -- or by scales[case][dim+2] when scales is not
 * NULL -- and the case stops at the first iteration where every component is
 * <= drop, or after caps[case] iterations (caps may be NULL: no cap). A
 * stopped case is skipped by every later launch, so no case runs past its
 * stopping iteration whatever the length of the psst_explicit_solve calls.
 * Setting the rule resets every case's counters and run flags (a case with
 * cap <= 0 starts stopped); drop <= 0 switches the rule off. */
psst_status psst_solver_set_stop_rule(psst_solver *s, double drop, int32_t scale_iters, const double *scales,
                                      const int32_t *caps);

/* Merged grids with a stop rule set; no counterpart in the reference. Runs
 * iterations until every case has stopped, a kernel has raised an error, or
 * max_iter iterations have run -- as ONE launch of a CUDA graph whose
 * while-loop node repeats a captured block of `chunk` iterations; the block's
 * last kernel sets the loop condition on the device from the cases' run
 * flags, the error word and the iteration count, so the host takes no part
 * until the end (at most ceil(max_iter / chunk) blocks run). chunk times the
 * RK stage count must be even. *iterations receives the iterations run
 * (whole blocks); res_linf / res_l2 (may be NULL) receive the residual
 * columns of the first min(*iterations, max_iter) of them, [n][dim+2] as
 * psst_explicit_solve returns them. Per-case residuals are not kept
 * (psst_solver_case_status gives each case's stopping iteration). */
psst_status psst_solver_run_to_stop(psst_solver *s, int64_t max_iter, int chunk, int64_t *iterations,
                                    double *res_linf, double *res_l2);

/* Merged grids only. Per case (each argument may be NULL): run flag, iterations
 * run under the stop rule, iteration at which the drop was reached (0: not
 * reached), and the normalisation in use [ncase][dim+2]. */
psst_status psst_solver_case_status(psst_solver *s, int32_t *active, int32_t *iterations, int32_t *converged_at,
                                    double *scales);

/* Merged grids only. Per-case residual columns of the last psst_explicit_solve
 * call: out[n_iter][ncase][dim+2], each the max over RK stages and the case's
 * cells of |res| (the reference's column, per case). n_iter <= that call's. */
psst_status psst_solver_case_residuals(psst_solver *s, int n_iter, double *out);

/* Sequential LocalAccTime1 (lc1_mode SEQUENTIAL, FP64, single grids): the
 * reference's in-loop order (psstFiniteVolumeGrid.cpp:317-323) as a wavefront.
 * With on != 0 (the default) each psst_explicit_solve call runs as ONE
 * persistent cooperative launch: operation m (a gradient or an RK stage) of a
 * cell at level L runs at step P m + L, so the operations of many iterations
 * overlap along the level chain, every cell keeps the reference's inputs and
 * results are bit-identical to the level-by-level walk (on == 0, one launch
 * sequence per stage, also the path of the stage-by-stage API). Calls are not
 * captured as CUDA graphs in this mode. */
psst_status psst_solver_use_wavefront(psst_solver *s, int on);

/* Bound of each device-side wait of the persistent launch (its grid
 * barriers), in nanoseconds; < 0 restores the default (10 s). A wait that runs
 * out stops the launch and the call returns PSST_ERR_TIMEOUT; the solver stays
 * usable, its state is undefined until the next psst_solver_set_state. 0 makes
 * every wait run out at once (used to test that path). */
psst_status psst_solver_set_wait_limit(psst_solver *s, int64_t nanoseconds);

/* Schedule of the sequential LocalAccTime1: info[5] = {wavefront active (0/1),
 * period P, levels, work items, CTAs of the persistent launch}. */
psst_status psst_solver_schedule_info(const psst_solver *s, int64_t *info);

/* Reference counter psstGridFV::iter_ after the calls so far. */
int64_t psst_solver_iter(const psst_solver *s);

void psst_solver_destroy(psst_solver *s);

/* ------------------------------------------------------------------------ */
/* Learned warm start: coordinate MLP (no counterpart in the reference)      */
/* ------------------------------------------------------------------------ */

/* A 6-layer MLP of width 256 mapping (Mach, ramp angle, x, y), each normalised
 * to [-1, 1], through 124 Fourier features (sin/cos(2^j pi v), j < 15, and v
 * itself) to 4 outputs (normalised rho, u, v, p). Hidden layers use SiLU. The
 * five hidden GEMMs of the forward and backward passes run on the tensor cores
 * (tcgen05, BF16 operands, FP32 accumulation); master weights, gradients and
 * Adam state are FP32. Input and target arrays are DEVICE pointers, row-major
 * [B][4] FP32, on the network's device. */
typedef struct psst_mlp psst_mlp;
psst_status psst_mlp_create(int device, uint64_t seed, psst_mlp **out);
int64_t psst_mlp_param_count(const psst_mlp *m);
/* Parameters as one FP32 array: for each layer W [out][in] then b [out]. */
psst_status psst_mlp_get_params(psst_mlp *m, float *out, int64_t n);
psst_status psst_mlp_set_params(psst_mlp *m, const float *in, int64_t n); /* also resets Adam */
psst_status psst_mlp_forward(psst_mlp *m, const float *x, int B, float *y);
/* Loss (mean squared error over B x 4) and its gradient (host array, layout of
 * psst_mlp_get_params) without changing the parameters. */
psst_status psst_mlp_gradients(psst_mlp *m, const float *x, const float *t, int B, float *grads, float *loss);
/* One Adam step (beta 0.9/0.999, eps 1e-8) at learning rate lr; returns the loss
 * before the step. */
psst_status psst_mlp_train_step(psst_mlp *m, const float *x, const float *t, int B, float lr, float *loss);
/* The network's kernels run on `stream` (a cudaStream_t; NULL: its own
 * non-blocking stream, which is not ordered with the legacy default stream --
 * select that one by its explicit handle, cudaStreamLegacy). x, t and y are
 * device arrays read and written in stream order: inputs produced on another
 * stream must be complete before a call, and y of psst_mlp_forward is
 * complete only in `stream`'s order. */
psst_status psst_mlp_set_stream(psst_mlp *m, void *stream);
void psst_mlp_destroy(psst_mlp *m);

/* The tensor-core GEMM on its own: D[z][m][n] = sum over k of split z of
 * A[m][k] * B[n][k], BF16 device operands given by element strides
 * (A[m][k] = A[m*a_sm + k*a_sk], B[n][k] = B[n*b_sn + k*b_sk]), FP32 device
 * output with row stride d_sm, z over ceil(K / k_split) splits (plain element
 * sum of the splits = the full product). Synchronises the stream. Operands
 * 16-byte aligned with a row stride of a multiple of 8 elements, contiguous
 * along K (a_sk or b_sk == 1) or along M/N (a_sm or b_sn == 1), with split
 * ranges of whole 64-wide chunks (k_split % 64 == 0, or one split), are
 * loaded by TMA (tensor maps encoded per call); other operands are staged
 * through registers (16-byte vectors where aligned, else element by element). */
psst_status psst_tc_gemm_bf16(const void *A, int64_t a_sm, int64_t a_sk, const void *B, int64_t b_sn, int64_t b_sk,
                              int M, int N, int K, int k_split, float *D, int64_t d_sm, void *stream);

/* psst_tc_gemm_bf16 timed: one launch outside the timing, then reps launches
 * captured as one CUDA graph on a private stream (ordered after `stream`) and
 * replayed between two CUDA events; *ms receives the mean device time of one
 * launch, with no host time between launches. */
psst_status psst_tc_gemm_bf16_time(const void *A, int64_t a_sm, int64_t a_sk, const void *B, int64_t b_sn,
                                   int64_t b_sk, int M, int N, int K, int k_split, float *D, int64_t d_sm,
                                   void *stream, int reps, double *ms);

/* psst_tc_gemm_bf16 with the bound of its first mbarrier wait that runs out
 * given in polls (< 0: the default, about a second; 0: that wait gives up at
 * once). A wait that runs out makes the call return PSST_ERR_TIMEOUT after
 * full-length waits for the tensor-core work and the TMA copies in flight, so
 * no MMA or copy is running when the kernel frees its tensor memory and its
 * shared memory; D is then undefined. Used to test the timeout path without
 * stalling a GPU. */
psst_status psst_tc_gemm_bf16_wait(const void *A, int64_t a_sm, int64_t a_sk, const void *B, int64_t b_sn,
                                   int64_t b_sk, int M, int N, int K, int k_split, float *D, int64_t d_sm,
                                   void *stream, int64_t wait_polls);

#ifdef __cplusplus
}
#endif
#endif
