// Kernel launchers, one set per state precision (explicitly instantiated in
// kernels_f64.cu and kernels_f32.cu). Host code (solver.cpp) calls only these.
#pragma once
#include <cstddef>

#include <cuda_runtime_api.h>

#include "devgrid.hpp"

namespace psst {

constexpr int kBlock = 256;
constexpr int kMinBlock = 64;  // smallest launch shape the tuner may pick
constexpr int kWfBlock = 128;  // threads per CTA of k_wavefront
constexpr int kWfLanes = 4;    // lanes per cell in k_wavefront's RK stages (cells per work item: 32)
constexpr int kWfSyncWords = 96;  // k_wavefront's grid-barrier words (three 128-byte lines)
constexpr int kNormReduceBlocks = 296;  // blocks of k_norm_reduce (first level of its two-level sum): two per SM
inline int nblocks(int64_t n, int b = kBlock) { return (int)((n + b - 1) / b); }

template <typename R>
struct Ops {
    // sizes of the records for a dimension (host allocation)
    static size_t face_rec_bytes(int dim);
    static size_t grad_rec_bytes(int dim);
    static size_t face_out_bytes(int dim);
    static void prologue(int dim, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk, const Gas &gas,
                         cudaStream_t s);
    // state <-> the reference's volume order on the device: prim is SoA
    // p[nvol], T[nvol], u[dim][nvol] (FP64), vol[d] the volume of device cell d
    static void gather_prim(int dim, const DevGrid &g, const DevState<R> &st, const double *prim,
                            const int32_t *vol, int64_t nvol, cudaStream_t s);
    static void scatter_prim(int dim, const DevGrid &g, const DevState<R> &st, double *prim, const int32_t *vol,
                             int64_t nvol, cudaStream_t s);
    // exact state (records incl. rho, and w) from reference-ordered FP64 arrays
    static void set_exact(int dim, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk,
                          const double *prim, const double *rho, const double *w, const int32_t *vol, int64_t nvol,
                          cudaStream_t s);
    // w[v][dim+2] per volume (interior cells only)
    static void scatter_w(int dim, const DevGrid &g, const DevWork<R> &wk, double *w, const int32_t *vol,
                          cudaStream_t s);
    // grad: 1 Green-Gauss, 2 least squares; celllim: 0, 4 (Barth-Jespersen), 5 (Venkatakrishnan)
    static void gradient(int dim, int grad, int celllim, const DevGrid &g, const DevState<R> &st,
                         const DevWork<R> &wk, cudaStream_t s);
    // face pass: rec 0 first order, 1 DM with limiter lim (1..3), 2 cell-limited
    // MUSCL; lc selects the time-step terms written with each face's flux
    static void face(int dim, int flux, int rec, int lim, int lc, const DevGrid &g, const DevState<R> &st,
                     const DevWork<R> &wk, const Gas &gas, cudaStream_t s);
    // cell pass of the parallel modes (lc 0, 2, 1 from stage-start values):
    // residual, time step, RK update, ghosts, block norm partials of stage kstage
    static void cell(int dim, int lc, const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt,
                     const DevWork<R> &wk, const Gas &gas, double cfl, double dt_uniform, double alpha,
                     int stage, int kstage, int it_slot, cudaStream_t s);  // stage: 1 first, 2 last (bits)
    // the iteration's residual columns from the cell passes' partials of nstage stages
    static void norm_reduce(int dim, const DevGrid &g, const DevWork<R> &wk, int nstage, int it_slot,
                            cudaStream_t s);
    static void residual(int dim, const DevGrid &g, const DevWork<R> &wk, cudaStream_t s);
    // cell update from face outputs (gather) or from wk.res; seq: the
    // sequential LocalAccTime1 (single block over levels); norms by norm_finish
    static void cell_update(int dim, int lc, bool seq, bool gather, const DevGrid &g, const DevState<R> &cur,
                            const DevState<R> &nxt, const DevWork<R> &wk, const Gas &gas, double cfl,
                            double dt_uniform, double alpha, int first_stage, cudaStream_t s);
    static void ghost_update(int dim, const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt,
                             const Gas &gas, cudaStream_t s);
    static void norm_finish(int dim, const DevWork<R> &wk, int nblk, int32_t nint, int it_slot, cudaStream_t s);
    // merged grids: the per-case stop rule after iteration it_slot
    static void case_stop(int dim, const DevGrid &g, const DevWork<R> &wk, const CaseStop &cs, int it_slot,
                          cudaStream_t s);
    // the last kernel of a run-to-stop block of `chunk` iterations: history,
    // iteration count and the while-loop condition `h`
    static void loop_control(int dim, const DevGrid &g, const DevWork<R> &wk, const CaseStop &cs, LoopCtl *ctl,
                             int chunk, cudaGraphConditionalHandle h, cudaStream_t s);
    // Sequential LocalAccTime1 over a whole call as one cooperative launch of
    // nblocks CTAs (k_wavefront; FP64 only, cudaErrorNotSupported otherwise).
    static cudaError_t wavefront(int dim, int rec, int lim, const WfArgs<R> &a, int nblocks, cudaStream_t s);
    // co-resident CTAs of that kernel on the current device (0: not built)
    static int wavefront_max_blocks(int dim, int rec, int lim);
};

}  // namespace psst
