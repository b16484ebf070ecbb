// Launcher bodies for Ops<R>: template dispatch from runtime scheme options to
// kernel instantiations. Included by kernels_f64.cu / kernels_f32.cu only.
#pragma once
#include <algorithm>

#include "kernels.cuh"
#include "ops.hpp"
#include "wavefront.cuh"

namespace psst {

template <typename R>
size_t Ops<R>::face_rec_bytes(int dim) {
    return dim == 2 ? sizeof(FaceRec<R, 2>) : sizeof(FaceRec<R, 3>);
}
template <typename R>
size_t Ops<R>::grad_rec_bytes(int dim) {
    return dim == 2 ? sizeof(GradRec<R, 2>) : sizeof(GradRec<R, 3>);
}
template <typename R>
size_t Ops<R>::face_out_bytes(int dim) {
    return dim == 2 ? sizeof(FaceOut<R, 2>) : sizeof(FaceOut<R, 3>);
}

template <typename R>
void Ops<R>::prologue(int dim, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk, const Gas &gas,
                      cudaStream_t s) {
    if (g.nall == 0) return;
    if (dim == 2)
        k_prologue<R, 2><<<nblocks(g.nall), kBlock, 0, s>>>(g, st, wk, gas);
    else
        k_prologue<R, 3><<<nblocks(g.nall), kBlock, 0, s>>>(g, st, wk, gas);
}

template <typename R>
void Ops<R>::gather_prim(int dim, const DevGrid &g, const DevState<R> &st, const double *prim, const int32_t *vol,
                         int64_t nvol, cudaStream_t s) {
    if (g.nall == 0) return;
    if (dim == 2)
        k_gather_prim<R, 2><<<nblocks(g.nall), kBlock, 0, s>>>(g.nall, st, prim, vol, nvol);
    else
        k_gather_prim<R, 3><<<nblocks(g.nall), kBlock, 0, s>>>(g.nall, st, prim, vol, nvol);
}

template <typename R>
void Ops<R>::scatter_prim(int dim, const DevGrid &g, const DevState<R> &st, double *prim, const int32_t *vol,
                          int64_t nvol, cudaStream_t s) {
    if (g.nall == 0) return;
    if (dim == 2)
        k_scatter_prim<R, 2><<<nblocks(g.nall), kBlock, 0, s>>>(g.nall, st, prim, vol, nvol);
    else
        k_scatter_prim<R, 3><<<nblocks(g.nall), kBlock, 0, s>>>(g.nall, st, prim, vol, nvol);
}

template <typename R>
void Ops<R>::set_exact(int dim, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk, const double *prim,
                       const double *rho, const double *w, const int32_t *vol, int64_t nvol, cudaStream_t s) {
    if (g.nall == 0) return;
    if (dim == 2)
        k_set_exact<R, 2><<<nblocks(g.nall), kBlock, 0, s>>>(g.nall, g.nint, st, wk.w, prim, rho, w, vol, nvol);
    else
        k_set_exact<R, 3><<<nblocks(g.nall), kBlock, 0, s>>>(g.nall, g.nint, st, wk.w, prim, rho, w, vol, nvol);
}

template <typename R>
void Ops<R>::scatter_w(int dim, const DevGrid &g, const DevWork<R> &wk, double *w, const int32_t *vol,
                       cudaStream_t s) {
    if (g.nint == 0) return;
    k_scatter_w<R><<<nblocks(g.nint), kBlock, 0, s>>>(g.nint, dim + 2, wk.w, w, vol);
}

template <typename R, int DIM>
static void gradient_dim(int grad, int celllim, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk,
                         cudaStream_t s) {
    const int bs = g.blk_grad, nb = nblocks(g.nint, bs);
    if (grad == 1) {
        if (celllim == 4)
            k_gradient<R, DIM, 1, 4><<<nb, bs, 0, s>>>(g, st, wk);
        else if (celllim == 5)
            k_gradient<R, DIM, 1, 5><<<nb, bs, 0, s>>>(g, st, wk);
        else
            k_gradient<R, DIM, 1, 0><<<nb, bs, 0, s>>>(g, st, wk);
    } else {
        if (celllim == 4)
            k_gradient<R, DIM, 2, 4><<<nb, bs, 0, s>>>(g, st, wk);
        else if (celllim == 5)
            k_gradient<R, DIM, 2, 5><<<nb, bs, 0, s>>>(g, st, wk);
        else
            k_gradient<R, DIM, 2, 0><<<nb, bs, 0, s>>>(g, st, wk);
    }
}

template <typename R>
void Ops<R>::gradient(int dim, int grad, int celllim, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk,
                      cudaStream_t s) {
    if (g.nint == 0) return;
    if (dim == 2)
        gradient_dim<R, 2>(grad, celllim, g, st, wk, s);
    else
        gradient_dim<R, 3>(grad, celllim, g, st, wk, s);
}

// ---- face pass: DIM x FLUX x (REC, LIM) x LC ----
template <typename R, int DIM, int FLUX, int REC, int LIM>
static void face_l(int lc, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk, const Gas &gas,
                   cudaStream_t s) {
    const int bs = g.blk_face, nb = nblocks(g.nface, bs);
    if (lc == 1)
        k_face<R, DIM, FLUX, REC, LIM, 1><<<nb, bs, 0, s>>>(g, st, wk, gas);
    else if (lc == 2)
        k_face<R, DIM, FLUX, REC, LIM, 2><<<nb, bs, 0, s>>>(g, st, wk, gas);
    else
        k_face<R, DIM, FLUX, REC, LIM, 0><<<nb, bs, 0, s>>>(g, st, wk, gas);
}

template <typename R, int DIM, int FLUX>
static void face_r(int rec, int lim, int lc, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk,
                   const Gas &gas, cudaStream_t s) {
    if (rec == 0)
        face_l<R, DIM, FLUX, 0, 1>(lc, g, st, wk, gas, s);
    else if (rec == 2)
        face_l<R, DIM, FLUX, 2, 1>(lc, g, st, wk, gas, s);
    else if (lim == 1)
        face_l<R, DIM, FLUX, 1, 1>(lc, g, st, wk, gas, s);
    else if (lim == 2)
        face_l<R, DIM, FLUX, 1, 2>(lc, g, st, wk, gas, s);
    else
        face_l<R, DIM, FLUX, 1, 3>(lc, g, st, wk, gas, s);
}

template <typename R, int DIM>
static void face_f(int flux, int rec, int lim, int lc, const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk,
                   const Gas &gas, cudaStream_t s) {
    if (flux == 1)
        face_r<R, DIM, 1>(rec, lim, lc, g, st, wk, gas, s);
    else if (flux == 2)
        face_r<R, DIM, 2>(rec, lim, lc, g, st, wk, gas, s);
    else
        face_r<R, DIM, 3>(rec, lim, lc, g, st, wk, gas, s);
}

template <typename R>
void Ops<R>::face(int dim, int flux, int rec, int lim, int lc, const DevGrid &g, const DevState<R> &st,
                  const DevWork<R> &wk, const Gas &gas, cudaStream_t s) {
    if (g.nface == 0) return;
    if (dim == 2)
        face_f<R, 2>(flux, rec, lim, lc, g, st, wk, gas, s);
    else
        face_f<R, 3>(flux, rec, lim, lc, g, st, wk, gas, s);
}

// ---- cell pass (parallel modes) ----
template <typename R, int DIM>
static void cell_d(int lc, const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt, const DevWork<R> &wk,
                   const Gas &gas, double cfl, double dtu, double alpha, int first, int ks, int it, cudaStream_t s) {
    const int bs = g.blk_cell, nb = nblocks(g.nint, bs);
    if (g.cell_case) {  // merged grids: per-case run flags and residual columns
        if (lc == 1)
            k_cell<R, DIM, 1, true><<<nb, bs, 0, s>>>(g, cur, nxt, wk, gas, cfl, dtu, alpha, first, ks, it);
        else if (lc == 2)
            k_cell<R, DIM, 2, true><<<nb, bs, 0, s>>>(g, cur, nxt, wk, gas, cfl, dtu, alpha, first, ks, it);
        else
            k_cell<R, DIM, 0, true><<<nb, bs, 0, s>>>(g, cur, nxt, wk, gas, cfl, dtu, alpha, first, ks, it);
        return;
    }
    if (lc == 1)
        k_cell<R, DIM, 1, false><<<nb, bs, 0, s>>>(g, cur, nxt, wk, gas, cfl, dtu, alpha, first, ks, it);
    else if (lc == 2)
        k_cell<R, DIM, 2, false><<<nb, bs, 0, s>>>(g, cur, nxt, wk, gas, cfl, dtu, alpha, first, ks, it);
    else
        k_cell<R, DIM, 0, false><<<nb, bs, 0, s>>>(g, cur, nxt, wk, gas, cfl, dtu, alpha, first, ks, it);
}

template <typename R>
void Ops<R>::cell(int dim, int lc, const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt,
                  const DevWork<R> &wk, const Gas &gas, double cfl, double dt_uniform, double alpha, int stage,
                  int kstage, int it_slot, cudaStream_t s) {
    if (g.nint == 0) return;
    if (dim == 2)
        cell_d<R, 2>(lc, g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, stage, kstage, it_slot, s);
    else
        cell_d<R, 3>(lc, g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, stage, kstage, it_slot, s);
}

template <typename R>
void Ops<R>::norm_reduce(int dim, const DevGrid &g, const DevWork<R> &wk, int nstage, int it_slot, cudaStream_t s) {
    if (g.nint == 0) return;
    const int nblk = nblocks(g.nint, g.blk_cell);
    const dim3 grid((unsigned)std::min(nblk, kNormReduceBlocks), (unsigned)nstage);
    if (dim == 2)
        k_norm_reduce<4><<<grid, 64 * 4, 0, s>>>(wk.l2part, nblk, nstage, g.nint, wk.l2mid, wk.ticket, wk.linf, wk.l2,
                                                 it_slot);
    else
        k_norm_reduce<5><<<grid, 64 * 5, 0, s>>>(wk.l2part, nblk, nstage, g.nint, wk.l2mid, wk.ticket, wk.linf, wk.l2,
                                                 it_slot);
}

template <typename R>
void Ops<R>::residual(int dim, const DevGrid &g, const DevWork<R> &wk, cudaStream_t s) {
    if (g.nint == 0) return;
    if (dim == 2)
        k_residual<R, 2><<<nblocks(g.nint), kBlock, 0, s>>>(g, wk);
    else
        k_residual<R, 3><<<nblocks(g.nint), kBlock, 0, s>>>(g, wk);
}

template <typename R, int DIM, bool GATHER>
static void cell_update_g(int lc, bool seq, const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt,
                          const DevWork<R> &wk, const Gas &gas, double cfl, double dt_uniform, double alpha,
                          int first_stage, cudaStream_t s) {
    if (seq) {
        k_cell_update_seq<R, DIM, GATHER><<<1, 1024, 0, s>>>(g, cur, nxt, wk, gas, cfl, alpha, first_stage);
        return;
    }
    const int nb = nblocks(g.nint);
    if (lc == 0)
        k_cell_update<R, DIM, 0, GATHER><<<nb, kBlock, 0, s>>>(g, cur, nxt, wk, gas, cfl, dt_uniform, alpha,
                                                               first_stage);
    else if (lc == 1)
        k_cell_update<R, DIM, 1, GATHER><<<nb, kBlock, 0, s>>>(g, cur, nxt, wk, gas, cfl, dt_uniform, alpha,
                                                               first_stage);
    else
        k_cell_update<R, DIM, 2, GATHER><<<nb, kBlock, 0, s>>>(g, cur, nxt, wk, gas, cfl, dt_uniform, alpha,
                                                               first_stage);
}

template <typename R>
void Ops<R>::cell_update(int dim, int lc, bool seq, bool gather, const DevGrid &g, const DevState<R> &cur,
                         const DevState<R> &nxt, const DevWork<R> &wk, const Gas &gas, double cfl, double dt_uniform,
                         double alpha, int first_stage, cudaStream_t s) {
    if (g.nint == 0) return;
    if (dim == 2) {
        if (gather)
            cell_update_g<R, 2, true>(lc, seq, g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, first_stage, s);
        else
            cell_update_g<R, 2, false>(lc, seq, g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, first_stage, s);
    } else {
        if (gather)
            cell_update_g<R, 3, true>(lc, seq, g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, first_stage, s);
        else
            cell_update_g<R, 3, false>(lc, seq, g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, first_stage, s);
    }
}

template <typename R>
void Ops<R>::ghost_update(int dim, const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt, const Gas &gas,
                          cudaStream_t s) {
    if (g.nghost == 0) return;
    if (dim == 2)
        k_ghost_update<R, 2><<<nblocks(g.nghost), kBlock, 0, s>>>(g, cur, nxt, gas);
    else
        k_ghost_update<R, 3><<<nblocks(g.nghost), kBlock, 0, s>>>(g, cur, nxt, gas);
}

template <typename R>
void Ops<R>::norm_finish(int dim, const DevWork<R> &wk, int nblk, int32_t nint, int it_slot, cudaStream_t s) {
    if (dim == 2)
        k_norm_finish<4><<<1, 256, 0, s>>>(wk.l2part, nblk, nint, wk.linf, wk.l2, it_slot);
    else
        k_norm_finish<5><<<1, 256, 0, s>>>(wk.l2part, nblk, nint, wk.linf, wk.l2, it_slot);
}

template <typename R>
void Ops<R>::case_stop(int dim, const DevGrid &g, const DevWork<R> &wk, const CaseStop &cs, int it_slot,
                       cudaStream_t s) {
    const unsigned long long *cl = wk.case_linf + (int64_t)it_slot * g.ncase * (dim + 2);
    if (dim == 2)
        k_case_stop<4><<<nblocks(g.ncase), kBlock, 0, s>>>(cs, cl, g.ncase);
    else
        k_case_stop<5><<<nblocks(g.ncase), kBlock, 0, s>>>(cs, cl, g.ncase);
}

template <typename R>
void Ops<R>::loop_control(int dim, const DevGrid &g, const DevWork<R> &wk, const CaseStop &cs, LoopCtl *ctl,
                          int chunk, cudaGraphConditionalHandle h, cudaStream_t s) {
    if (dim == 2)
        k_loop_control<4><<<1, kBlock, 0, s>>>(cs, g.ncase, wk.err, ctl, wk.linf, wk.l2, chunk, h);
    else
        k_loop_control<5><<<1, kBlock, 0, s>>>(cs, g.ncase, wk.err, ctl, wk.linf, wk.l2, chunk, h);
}

// ---- sequential LocalAccTime1 as one persistent launch (FP64 only) ----
template <typename R, int DIM>
static cudaError_t wavefront_d(int rec, int lim, const WfArgs<R> &a, int nb, cudaStream_t s) {
    if (rec == 0) return wf_launch<R, DIM, 0, 1>(a, nb, s);
    if (rec == 2) return wf_launch<R, DIM, 2, 1>(a, nb, s);
    if (lim == 1) return wf_launch<R, DIM, 1, 1>(a, nb, s);
    if (lim == 2) return wf_launch<R, DIM, 1, 2>(a, nb, s);
    return wf_launch<R, DIM, 1, 3>(a, nb, s);
}
template <typename R, int DIM>
static int wavefront_max_d(int rec, int lim) {
    if (rec == 0) return wf_max_blocks<R, DIM, 0, 1>();
    if (rec == 2) return wf_max_blocks<R, DIM, 2, 1>();
    if (lim == 1) return wf_max_blocks<R, DIM, 1, 1>();
    if (lim == 2) return wf_max_blocks<R, DIM, 1, 2>();
    return wf_max_blocks<R, DIM, 1, 3>();
}

template <typename R>
cudaError_t Ops<R>::wavefront(int dim, int rec, int lim, const WfArgs<R> &a, int nb, cudaStream_t s) {
    if constexpr (sizeof(R) == 8) {
        return dim == 2 ? wavefront_d<R, 2>(rec, lim, a, nb, s) : wavefront_d<R, 3>(rec, lim, a, nb, s);
    } else {
        (void)dim, (void)rec, (void)lim, (void)a, (void)nb, (void)s;
        return cudaErrorNotSupported;
    }
}

template <typename R>
int Ops<R>::wavefront_max_blocks(int dim, int rec, int lim) {
    if constexpr (sizeof(R) == 8) {
        return dim == 2 ? wavefront_max_d<R, 2>(rec, lim) : wavefront_max_d<R, 3>(rec, lim);
    } else {
        (void)dim, (void)rec, (void)lim;
        return 0;
    }
}

}  // namespace psst
