/* psst_oracle: CPU restatement of the PSST explicit finite-volume loop.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker that the CUDA path is compared
 * against; it is built into oracle/_build/ and is used only by tests/,
 * __graft_entry__.smoke() and the cpu_baseline leg of bench.py. The product
 * library never links or calls it.
 *
 * It reads a Fluent ASCII mesh and the reference's setup files and reproduces,
 * operation by operation and in the same order, what the reference does in
 *   psstAnsysDirector/psstAnsysBuilder/create_finite_volume_grid
 *       (psstAnsysGridReader.cpp:688-907, 937-1116, 1138-1317)
 *   psstFace::initialize / psstVolume::initialize
 *       (psstFiniteVolumeGridTools.cpp:397-505, 709-827)
 *   psstGridFV::solver_parameters / explicit_solve
 *       (psstFiniteVolumeGrid.cpp:36-194, 248-401, 403-557, 641-717)
 * and the strategies they select (gradients, reconstruction, limiters,
 * convective fluxes, local time step, Runge-Kutta, boundary conditions).
 *
 * Extensions the reference does not have (their results are "parity
 * unpinned", i.e. checked only against this restatement):
 *   - lc1_jacobi: LocalAccTime1 evaluated from stage-start values (Jacobi),
 *   - limiter 4 = Barth-Jespersen, 5 = Venkatakrishnan (cell-based MUSCL),
 *   - RMS (L2) residual norms.
 */
#ifndef PSST_ORACLE_H
#define PSST_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle oracle_t;

/* Opens mesh + case (cwd-independent: files are <case_dir>/<case_name>.*).
 * Returns NULL on error and writes the message into err. */
oracle_t *oracle_open(const char *mesh_path, const char *case_dir, const char *case_name,
                      char *err, int errlen);

/* Overrides applied after setup: "lc1_jacobi" (0/1), "limiter" (1..5),
 * "venkat_k" (Venkatakrishnan K), "max_iter". Returns 0 on success. */
int oracle_set(oracle_t *o, const char *key, double value);

/* Runs n_iter iterations of the explicit_solve loop body. res_linf and res_l2
 * (may be NULL) receive n_iter x (dim+2) values: per iteration, per component
 * (rho*u.., rho, rho*E) the max over RK stages of max|residual| and of the RMS
 * residual over interior cells. Returns 0, or -1 with oracle_error() set. */
int oracle_run(oracle_t *o, int n_iter, double *res_linf, double *res_l2);

/* One stage's convective residual of the current state (gradients first for
 * second order), without updating anything: read it as "vol_res"
 * [nvol x (dim+2)]. Returns 0, or -1 with oracle_error() set. */
int oracle_convective(oracle_t *o);

const char *oracle_error(const oracle_t *o);
int oracle_dim(const oracle_t *o);
int oracle_nvol(const oracle_t *o);   /* all volumes (interior + ghost), storage order */
int oracle_nface(const oracle_t *o);  /* all faces of all face zones, map order */
int oracle_iter(const oracle_t *o);   /* the reference's iter_ counter */

/* Copies a named per-volume / per-face array (layout as oracle/ref_dump.cpp):
 *  vol_p vol_T vol_rho vol_u[dim] vol_w[dim+2] vol_prev_w[dim+2] vol_dt vol_res[dim+2] vol_V
 *  vol_x[dim] vol_grad_u[dim*dim] vol_grad_p[dim] vol_grad_T[dim]
 *  vol_grad_rho[dim] vol_zone vol_bc vol_boundary
 *  face_S face_n[dim] face_x[dim] face_beta face_zone face_bc face_c0 face_c1
 * Integer arrays are returned as doubles. Returns the element count, or -1. */
long oracle_get(const oracle_t *o, const char *name, double *out, long cap);

/* Sets the primitive state (p, T, u[dim]) of every volume in storage order and
 * recomputes rho = p/(rm*T) and w as the explicit_solve prologue does. */
int oracle_set_prim(oracle_t *o, const double *p, const double *T, const double *u);

/* Writes <path> in the reference's .sav format (psstFiniteVolumeGrid.cpp:606-639). */
int oracle_write_sav(const oracle_t *o, const char *path);

void oracle_close(oracle_t *o);

#ifdef __cplusplus
}
#endif
#endif
