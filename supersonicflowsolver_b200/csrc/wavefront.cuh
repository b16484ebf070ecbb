// Sequential LocalAccTime1 as one persistent, cooperative launch per call.
//
// The reference evaluates LocalAccTime1 inside its update loop
// (psstFiniteVolumeGrid.cpp:317-323), so within a stage each cell sees the
// neighbours updated before it in storage order: a Gauss-Seidel chain.
// Walking it level by level costs one barrier per level per stage. Here the
// operations of a whole call (per iteration an optional gradient, then the RK
// stages) are pipelined as a wavefront: operation m of cell c runs at step
// P m + level(c) (WfSched in devgrid.hpp), so later operations start on the
// early levels while earlier ones are still finishing the late levels; a call
// of n iterations takes P (n ops/iteration - 1) + nlevels + 1 steps instead of
// n ops/iteration x nlevels. Every value a cell operation computes -- fluxes
// of its faces (each interior face is computed by both of its cells, with the
// same arithmetic and so the same bits), the time step from the neighbours
// the reference's order gives it, the RK update, its ghosts -- is the
// reference's, bit for bit.
//
// Buffers: states by stage parity, gradients by iteration parity, norm
// partials by operation parity (the schedule keeps every reader of a slot
// before its next writer). Residual norms are folded per level in level
// order, so they do not depend on which CTA ran which item.
//
// The grid barrier between steps is bounded: a wait longer than wait_ns sets
// the abort flag and ERR_TIMEOUT, and every CTA leaves at its next barrier.
#pragma once
#include "kernels.cuh"
#include "ops.hpp"

// CTAs per SM the wavefront kernel is built for (register cap 65536 / (128 x
// this)): more co-resident CTAs take more of a step's work items at once. 2D:
// three without spills; 3D: two (three would spill).
#ifndef PSST_WF_MINB_2D
#define PSST_WF_MINB_2D 3
#endif
#ifndef PSST_WF_MINB_3D
#define PSST_WF_MINB_3D 2
#endif
// pause between two polls of the grid barrier's generation (ns)
#ifndef PSST_WF_POLL_NS
#define PSST_WF_POLL_NS 32
#endif

namespace psst {

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Grid barrier of a cooperative launch (all CTAs co-resident). sync[0]
// counts arrivals, sync[kSyncGen] is the generation, sync[kSyncAbort] the
// abort flag, each on its own 128-byte line so that the CTAs polling the
// generation do not slow the arrivals' atomics. The last CTA to arrive resets
// the count and releases the next generation; the others poll it for at most
// wait_ns (0: not at all). Returns false when the launch is aborted (here or
// in another CTA).
constexpr int kSyncGen = 32, kSyncAbort = 64;
static_assert(kSyncAbort < kWfSyncWords, "barrier words");
__device__ __forceinline__ bool grid_barrier(unsigned *sync, unsigned &gen, uint64_t wait_ns, int32_t *err,
                                             int64_t step) {
    __shared__ int s_go;
    __syncthreads();
    if (threadIdx.x == 0) {
        int go = 1;
        const unsigned g0 = gen;
        __threadfence();  // this CTA's writes (ordered before by the CTA barrier) before its arrival
        if (atomicAdd(&sync[0], 1u) == gridDim.x - 1) {
            sync[0] = 0u;
            st_release_gpu(&sync[kSyncGen], g0 + 1u);
        } else {
            const uint64_t t0 = global_ns();
            for (;;) {
                if (ld_acquire_gpu(&sync[kSyncGen]) != g0) break;
                __nanosleep(PSST_WF_POLL_NS);  // fewer polls competing with the arrivals for L2
                if (ld_acquire_gpu(&sync[kSyncAbort]) != 0u) {
                    go = 0;
                    break;
                }
                if (wait_ns == 0 || global_ns() - t0 > wait_ns) {
                    atomicExch(&sync[kSyncAbort], 1u);
                    flag_error(err, ERR_TIMEOUT, (int)step);
                    go = 0;
                    break;
                }
            }
        }
        if (go && ld_acquire_gpu(&sync[kSyncAbort]) != 0u) go = 0;
        gen = g0 + 1u;
        s_go = go;
    }
    __syncthreads();
    return s_go != 0;
}

template <typename R, int NV>
__device__ __forceinline__ RkIn<NV> rk_load_cg(const DevGrid &g, const DevWork<R> &wk, int first_stage, int32_t c) {
    RkIn<NV> in;
    const double *src = first_stage ? wk.w : wk.pw;
#pragma unroll
    for (int v = 0; v < NV; ++v) in.pw[v] = ldcg(src + (int64_t)v * g.nint + c);
    in.vol = g.V[c];
    return in;
}

// Riemann flux with the flux kind chosen at run time (uniform over the launch).
template <typename R, int DIM, int REC, int LIM>
__device__ __forceinline__ bool wf_interior_flux(int flux, Prim<R, DIM> r[2], const GradRec<R, DIM> *g0,
                                                 const GradRec<R, DIM> *g1, const FaceRec<R, DIM> &fr,
                                                 const R nn[DIM], const Gas &gas, R flow[DIM + 2]) {
    if (flux == 1) return interior_flux<R, DIM, 1, REC, LIM>(r, g0, g1, fr, nn, gas, flow);
    if (flux == 2) return interior_flux<R, DIM, 2, REC, LIM>(r, g0, g1, fr, nn, gas, flow);
    return interior_flux<R, DIM, 3, REC, LIM>(r, g0, g1, fr, nn, gas, flow);
}

// Gradient (and cell limiter) of cell c by the four lanes of a quad: lane q
// forms the contributions of the faces q, q+4, .. -- Green-Gauss in the
// face-loop order (psstGradCalculation.cpp:80-177), least squares in the
// cell's own order (:268-368; 3D as the corrected restatement of
// gradient_cell) -- as the products gradient_cell forms, and the quad adds
// them face by face in that order through shuffles, so the sums are
// gradient_cell's bit for bit. The neighbour min/max and the Barth-Jespersen
// / Venkatakrishnan limiter are minima and maxima (order-free). Lane 0 stores
// the record.
template <typename R, int DIM, int GRAD, int CELLLIM>
__device__ __forceinline__ void wf_gradient_quad(const DevGrid &g, const CellRec<R> *rec, GradRec<R, DIM> *gout,
                                                 int32_t c, int q, int qbase) {
    constexpr int NVAR = DIM + 2;
    const unsigned qmask = 0xFu << qbase;
    const FaceRec<R, DIM> *frec = reinterpret_cast<const FaceRec<R, DIM> *>(g.frec);
    const int32_t b = g.kuni ? c * g.kuni : g.csr_ptr[c], K = g.kuni ? g.kuni : g.csr_ptr[c + 1] - b;
    const uint64_t perm = g.wperm[c];
    const Prim<R, DIM> own = unpack<R, DIM>(ldcg(rec + c));
    R gr[NVAR][DIM], mx[NVAR], mn[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) {
        mx[i] = mn[i] = pvar<R, DIM>(own, i);
#pragma unroll
        for (int k = 0; k < DIM; ++k) gr[i][k] = (R)0;
    }
    const double V = g.V[c];
    constexpr int NR = DIM == 2 ? 3 : 7;
    R lr[NR], xo[DIM];
    if (GRAD == 2) {
#pragma unroll
        for (int t = 0; t < NR; ++t) lr[t] = (R)g.lsq_r[(int64_t)t * g.nint + c];
#pragma unroll
        for (int k = 0; k < DIM; ++k) xo[k] = (R)g.xc[(int64_t)k * g.nall + c];
    }
    for (int r0 = 0; r0 < K; r0 += kWfLanes) {
        const int j = r0 + q;
        R term[NVAR][DIM];
#pragma unroll
        for (int i = 0; i < NVAR; ++i)
#pragma unroll
            for (int k = 0; k < DIM; ++k) term[i][k] = (R)0;
        if (j < K) {
            Prim<R, DIM> oth;
            if (GRAD == 1) {  // face-loop order
                const int32_t ent = g.csr_ent[b + j];
                const FaceRec<R, DIM> fr = ldg(frec + (ent >> 1));
                oth = unpack<R, DIM>(ldcg(rec + g.csr_nb[b + j]));
                const R beta = (R)g.beta[ent >> 1];
                const int side = ent & 1;
                const R rbeta = (R)1 - beta;
                const R gp = (R)(fr.S / V);
                const R sgn = side ? (R)1 : (R)-1;
#pragma unroll
                for (int i = 0; i < NVAR; ++i) {
                    const R av = pvar<R, DIM>(own, i), ov = pvar<R, DIM>(oth, i);
                    const R phi0 = side ? ov : av, phi1 = side ? av : ov;
                    const R tv = beta * phi0 + rbeta * phi1;
#pragma unroll
                    for (int k = 0; k < DIM; ++k) term[i][k] = sgn * tv * gp * (R)fr.n[k];
                }
            } else {  // the cell's own order
                const int32_t slot = b + (int32_t)((perm >> (4 * j)) & 15);
                const int32_t nb = g.csr_nb[slot];
                oth = unpack<R, DIM>(ldcg(rec + nb));
                R diff[DIM];
                R w = (R)0;
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    diff[k] = (R)g.xc[(int64_t)k * g.nall + nb] - xo[k];
                    w += diff[k] * diff[k];
                }
                const R ws = (R)1 / w;
                const R al0 = diff[0] / (lr[0] * lr[0]);
                const R al1 = (diff[1] - lr[1] / lr[0] * diff[0]) / (lr[2] * lr[2]);
                R th[DIM];
                th[0] = al0 - lr[1] / lr[0] * al1;
                th[1] = al1;
                if constexpr (DIM == 3) {
                    const R al2 = (diff[2] - lr[4] / lr[2] * diff[1] + lr[6] * diff[0]) / (lr[5] * lr[5]);
                    th[0] += al2 * lr[6];
                    th[1] -= lr[4] / lr[2] * al2;
                    th[2] = al2;
                }
#pragma unroll
                for (int i = 0; i < NVAR; ++i) {
                    const R phi = (pvar<R, DIM>(oth, i) - pvar<R, DIM>(own, i));
#pragma unroll
                    for (int k = 0; k < DIM; ++k) term[i][k] = ws * th[k] * phi;
                }
            }
            if (CELLLIM)
#pragma unroll
                for (int i = 0; i < NVAR; ++i) {
                    const R v = pvar<R, DIM>(oth, i);
                    if (v > mx[i]) mx[i] = v;
                    if (v < mn[i]) mn[i] = v;
                }
        }
        for (int jj = 0; jj < kWfLanes && r0 + jj < K; ++jj)
#pragma unroll
            for (int i = 0; i < NVAR; ++i)
#pragma unroll
                for (int k = 0; k < DIM; ++k) gr[i][k] += __shfl_sync(qmask, term[i][k], qbase + jj);
    }
    R lim[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) lim[i] = (R)1;
    if (CELLLIM) {
#pragma unroll
        for (int i = 0; i < NVAR; ++i)
#pragma unroll
            for (int o = 1; o < kWfLanes; o <<= 1) {
                const R a = __shfl_xor_sync(qmask, mx[i], o), d = __shfl_xor_sync(qmask, mn[i], o);
                if (a > mx[i]) mx[i] = a;
                if (d < mn[i]) mn[i] = d;
            }
        const R eps2 = CELLLIM == 5 ? (R)g.vk_eps2[c] : (R)0;
        for (int j = q; j < K; j += kWfLanes) {
            const int32_t ent = g.csr_ent[b + j];
            R off[DIM];
            face_offsets<R, DIM>(frec + (ent >> 1), ent & 1, off);
#pragma unroll
            for (int i = 0; i < NVAR; ++i) {
                const R phic = pvar<R, DIM>(own, i);
                R dm = (R)0;
#pragma unroll
                for (int k = 0; k < DIM; ++k) dm += gr[i][k] * off[k];
                R pf = (R)1;
                if (dm != (R)0) {
                    const R dp = dm > (R)0 ? mx[i] - phic : mn[i] - phic;
                    if (CELLLIM == 4) {
                        const R y = dp / dm;
                        pf = y < (R)1 ? y : (R)1;
                    } else {
                        const R num = (dp * dp + eps2) + (R)2 * dm * dp;
                        const R den = dp * dp + (R)2 * dm * dm + dm * dp + eps2;
                        pf = num / den;
                    }
                }
                if (pf < lim[i]) lim[i] = pf;
            }
        }
#pragma unroll
        for (int i = 0; i < NVAR; ++i)
#pragma unroll
            for (int o = 1; o < kWfLanes; o <<= 1) {
                const R a = __shfl_xor_sync(qmask, lim[i], o);
                if (a < lim[i]) lim[i] = a;
            }
    }
    if (q != 0) return;
    GradRec<R, DIM> outr;
#pragma unroll
    for (int i = 0; i < NVAR; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) outr.g[i * DIM + k] = CELLLIM ? gr[i][k] * lim[i] : gr[i][k];
    st16(gout + c, outr);
}

// Gradient operation of iteration k for cell c (psstFiniteVolumeGrid.cpp:307-308), by a quad.
template <typename R, int DIM, int REC>
__device__ __forceinline__ void wf_gradient(const WfArgs<R> &a, int64_t k, int32_t c, int q, int qbase) {
    const CellRec<R> *in = a.buf[(a.in_buf + k * a.nst) & 1];
    GradRec<R, DIM> *out = reinterpret_cast<GradRec<R, DIM> *>(a.gbuf[(a.n_iter - 1 - k) & 1]);
    if constexpr (REC == 1) {
        if (a.grad == 1)
            wf_gradient_quad<R, DIM, 1, 0>(a.g, in, out, c, q, qbase);
        else
            wf_gradient_quad<R, DIM, 2, 0>(a.g, in, out, c, q, qbase);
    } else if constexpr (REC == 2) {
        if (a.grad == 1) {
            if (a.celllim == 4)
                wf_gradient_quad<R, DIM, 1, 4>(a.g, in, out, c, q, qbase);
            else
                wf_gradient_quad<R, DIM, 1, 5>(a.g, in, out, c, q, qbase);
        } else {
            if (a.celllim == 4)
                wf_gradient_quad<R, DIM, 2, 4>(a.g, in, out, c, q, qbase);
            else
                wf_gradient_quad<R, DIM, 2, 5>(a.g, in, out, c, q, qbase);
        }
    }
}

// RK stage s (stage `stage` of iteration k) for cell c, by the four lanes of a
// quad (kWfLanes): lane q takes the cell's faces q, q+4, .. in the reference's
// face-loop order for the fluxes (psstConvectiveFlow.cpp:289-299 as a per-cell
// sum) and the faces q, q+4, .. of the cell's own order for the local time
// step's neighbour terms (psstLocalTimeCalculation.cpp:90-131, neighbours
// updated earlier in the reference's order read from this stage's output);
// the quad then forms the residual sum and the time step's running sums face
// by face in the reference's order through shuffles (every lane the same
// values, in the same order, so the bits are the single-thread ones). Lane 0
// does the RK update and primitives (psstFiniteVolumeGrid.cpp:324-346) and
// the cell's ghosts (:351-366). qbase: the quad's first lane in the warp.
template <typename R, int DIM, int REC, int LIM>
__device__ __forceinline__ void wf_stage_quad(const WfArgs<R> &a, int64_t s, int64_t k, int stage, int32_t c, int q,
                                              int qbase, double sq[DIM + 2], double mx[DIM + 2]) {
    constexpr int NV = DIM + 2;
    const unsigned qmask = 0xFu << qbase;
    const DevGrid &g = a.g;
    const CellRec<R> *in = a.buf[(a.in_buf + s) & 1];
    CellRec<R> *out = a.buf[(a.in_buf + s + 1) & 1];
    const GradRec<R, DIM> *gr = reinterpret_cast<const GradRec<R, DIM> *>(a.gbuf[(a.n_iter - 1 - k) & 1]);
    const FaceRec<R, DIM> *frec = reinterpret_cast<const FaceRec<R, DIM> *>(g.frec);
    const int first = stage == 0;
    // uniform meshes (all quads, all tets): the CSR range follows from c
    const int32_t b = g.kuni ? c * g.kuni : g.csr_ptr[c], K = g.kuni ? g.kuni : g.csr_ptr[c + 1] - b;
    const uint64_t perm = g.wperm[c];
    const uint32_t low = a.sc.lowmask[c];
    const Prim<R, DIM> own = unpack<R, DIM>(ldcg(in + c));
    const R grm = (R)a.gas.gamma * (R)a.gas.rm;
    const R cc = sqrt(grm * own.T);
    R res[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) res[v] = (R)0;
    R den = (R)0, nnb = (R)0;
    for (int r0 = 0; r0 < K; r0 += kWfLanes) {
        const int j = r0 + q;
        int32_t ent = 0;
        R o[NV], pu[DIM], nvj = (R)0, cnj = (R)0, sj = (R)0;
        if (j < K) {
            // flux of the j-th face in face-loop order (the face pass's output value);
            // the cell across it from the CSR, so the state load does not wait
            // for the face record
            ent = g.csr_ent[b + j];
            const int32_t f = ent >> 1;
            const Prim<R, DIM> oth = unpack<R, DIM>(ldcg(in + g.csr_nb[b + j]));
            // own-order position j: its neighbour for the time step, from this
            // stage's output if the reference updates it before this cell
            const int32_t slot2 = (int32_t)((perm >> (4 * j)) & 15);
            const int32_t ent2 = g.csr_ent[b + slot2];
            const CellRec<R> *src = ((low >> slot2) & 1u) ? out : in;
            const Prim<R, DIM> on = unpack<R, DIM>(ldcg(src + g.csr_nb[b + slot2]));
            const FaceRec<R, DIM> fr = ldg(frec + f);
            const FaceRec<R, DIM> fr2 = ent2 == ent ? fr : ldg(frec + (ent2 >> 1));
            R nn[DIM];
#pragma unroll
            for (int k2 = 0; k2 < DIM; ++k2) nn[k2] = (R)fr.n[k2];
            const Prim<R, DIM> p0 = (ent & 1) ? oth : own;  // this cell is neighbour (ent & 1)
            const Prim<R, DIM> p1 = (ent & 1) ? own : oth;
            R flow[NV];
            if (f < g.nfi) {
                GradRec<R, DIM> g0, g1;
                if (REC) {
                    g0 = ldcg(gr + fr.c0);
                    g1 = ldcg(gr + fr.c1);
                }
                Prim<R, DIM> r[2] = {p0, p1};
                if (!wf_interior_flux<R, DIM, REC, LIM>(a.flux, r, &g0, &g1, fr, nn, a.gas, flow)) {
                    flag_error(a.wk.err, a.flux == 2 ? ERR_HLL : ERR_HLLC, f);
#pragma unroll
                    for (int v = 0; v < NV; ++v) flow[v] = (R)0;
                }
            } else {
                boundary_flux<R, DIM>(oth, nn, a.gas, flow);  // the ghost side
            }
            const R S = (R)fr.S;
#pragma unroll
            for (int v = 0; v < NV; ++v) o[v] = flow[v] * S;
            // the time step's terms of this face: products in the reference's
            // expressions, sums left to the in-order pass below
            cnj = (sqrt(grm * on.T) + cc) * (R)0.5;
#pragma unroll
            for (int k2 = 0; k2 < DIM; ++k2) {
                const R t = (R)fr2.n[k2];
                nvj += own.u[k2] * t;
                pu[k2] = on.u[k2] * t;
            }
            sj = (R)fr2.S;
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) o[v] = (R)0;
#pragma unroll
            for (int k2 = 0; k2 < DIM; ++k2) pu[k2] = (R)0;
        }
        // in-order pass over faces r0 .. r0+3 (every lane of the quad)
        for (int jj = 0; jj < kWfLanes && r0 + jj < K; ++jj) {
            const int sl = qbase + jj;
            const int32_t e = __shfl_sync(qmask, ent, sl);
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const R ov = __shfl_sync(qmask, o[v], sl);
                if (e & 1)
                    res[v] += ov;
                else
                    res[v] -= ov;
            }
#pragma unroll
            for (int k2 = 0; k2 < DIM; ++k2) nnb += __shfl_sync(qmask, pu[k2], sl);
            const R nvs = __shfl_sync(qmask, nvj, sl);
            nnb = (nnb + nvs) * (R)0.5;
            den += (fabs(nnb) + __shfl_sync(qmask, cnj, sl)) * __shfl_sync(qmask, sj, sl);
        }
    }
    if (q != 0) return;
    const RkIn<NV> rin = rk_load_cg<R, NV>(g, a.wk, first, c);
    const double dt = (double)((R)a.cfl * (R)g.V[c] / den);
    const CellRec<R> nrec =
        rk_update<R, DIM>(g, a.wk, a.gas, rin, dt, a.alpha[stage], first, stage == a.nst - 1, c, res, sq, mx);
    st16(out + c, nrec);
    const int32_t gh0 = g.gptr[c], gh1 = g.gptr[c + 1];
    if (gh1 > gh0) {
        const Prim<R, DIM> np = unpack<R, DIM>(nrec);
        for (int32_t i = gh0; i < gh1; ++i) {
            const int32_t gc = g.nint + i;
            st16(out + gc, ghost_state<R, DIM>(g, ldcg(in + gc), np, i, a.gas));
        }
    }
}

// Sum of res^2 and max |res| over the cells of one item (fixed pattern: warp
// trees, then the warps in order), written to out[2 NV]. Whole CTA.
template <int NV>
__device__ __forceinline__ void wf_item_partials(double sq[NV], double mx[NV], double *out) {
    __shared__ double red[2 * NV][kWfBlock / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double x = sq[v], m = mx[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_down_sync(FULL, x, o);
            m = fmax(m, __shfl_down_sync(FULL, m, o));
        }
        if (lane == 0) {
            red[v][wid] = x;
            red[NV + v][wid] = m;
        }
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0, m = 0.0;
        for (int i = 0; i < kWfBlock / 32; ++i) {
            s += red[threadIdx.x][i];
            m = fmax(m, red[NV + threadIdx.x][i]);
        }
        out[threadIdx.x] = s;
        out[NV + threadIdx.x] = m;
    }
    __syncthreads();  // red is reused by the CTA's next item
}

// Item i at step T (whole CTA; the quad of lanes 4t..4t+3 takes the item's
// t-th cell).
template <typename R, int DIM, int REC, int LIM>
__device__ __forceinline__ void wf_item(const WfArgs<R> &a, int64_t T, int32_t i) {
    constexpr int NV = DIM + 2;
    const WfSched &w = a.sc;
    const int32_t l = w.item_level[i];
    const int64_t m = (T - l) / w.period;
    const int j = (int)(m % a.nopi), gofs = a.nopi - a.nst;
    const int64_t k = m / a.nopi;
    const int slot = (int)threadIdx.x / kWfLanes, q = (int)threadIdx.x % kWfLanes;
    const int32_t c = w.cells32[(size_t)i * (kWfBlock / kWfLanes) + slot];  // the same for the quad
    const int qbase = ((int)threadIdx.x & 31) & ~(kWfLanes - 1);
    if (j < gofs) {  // the iteration's gradient
        if (c >= 0) wf_gradient<R, DIM, REC>(a, k, c, q, qbase);
        return;
    }
    const int stage = j - gofs;
    double sq[NV], mx[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) sq[v] = mx[v] = 0.0;
    if (c >= 0)
        wf_stage_quad<R, DIM, REC, LIM>(a, k * a.nst + stage, k, stage, c, q, qbase, sq, mx);
    wf_item_partials<NV>(sq, mx, w.ipart + ((size_t)(m & 1) * w.nitems + i) * 2 * NV);
}

// Block 0 (which takes no work items), after the barrier that ends step T:
// folds the item partials of the levels completed at step T into their
// stage's running norms, in level order;
// the last level finishes the stage: RMS and max folded into the iteration's
// columns as max over stages (the columns of k_norm_finish). (Spreading the
// levels over all CTAs, a thread each, measured three times slower per step.)
template <typename R, int NV>
__device__ __forceinline__ void wf_fold(const WfArgs<R> &a, int64_t T) {
    const WfSched &w = a.sc;
    const int64_t P = w.period, r = T % P;
    const int64_t lmax = T < w.nlevels - 1 ? T : (int64_t)w.nlevels - 1;
    if (lmax < r) return;
    const int64_t lhi = r + (lmax - r) / P * P;
    const int64_t t0 = T - P * (a.nops - 1);
    const int64_t llo = t0 > r ? t0 : r;
    for (int64_t l = llo + P * (int64_t)threadIdx.x; l <= lhi; l += P * (int64_t)blockDim.x) {
        const int64_t m = (T - l) / P;
        const int j = (int)(m % a.nopi), gofs = a.nopi - a.nst;
        if (j < gofs) continue;  // gradient operation: no residual
        const int64_t s = (m / a.nopi) * a.nst + (j - gofs);
        double sum[NV], mx[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) sum[v] = mx[v] = 0.0;
        const double *part = w.ipart + (size_t)(m & 1) * w.nitems * 2 * NV;
        for (int32_t q = w.lvl_items[2 * l]; q < w.lvl_items[2 * l + 1]; ++q)
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                sum[v] += ldcg(part + (size_t)q * 2 * NV + v);
                mx[v] = fmax(mx[v], ldcg(part + (size_t)q * 2 * NV + NV + v));
            }
        double *acc = w.acc + (size_t)(s % w.nacc) * 2 * NV;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            if (l == 0) {
                acc[v] = sum[v];
                acc[NV + v] = mx[v];
            } else {
                acc[v] += sum[v];
                acc[NV + v] = fmax(acc[NV + v], mx[v]);
            }
        }
        if (l == w.nlevels - 1) {
            const int64_t it = s / a.nst;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const double rms = sqrt(acc[v] / (double)(a.g.nint > 0 ? a.g.nint : 1));
                if (rms > a.wk.l2[it * NV + v]) a.wk.l2[it * NV + v] = rms;
                if (a.wk.linf[it * NV + v] < acc[NV + v]) a.wk.linf[it * NV + v] = acc[NV + v];
            }
        }
    }
}

template <typename R, int DIM, int REC, int LIM>
__global__ void __launch_bounds__(kWfBlock, DIM == 2 ? PSST_WF_MINB_2D : PSST_WF_MINB_3D) k_wavefront(const __grid_constant__ WfArgs<R> a) {
    constexpr int NV = DIM + 2;
    const WfSched &w = a.sc;
    const int64_t P = w.period;
    const int64_t tend = P * (a.nops - 1) + w.nlevels + 1;
    unsigned gen = 0;
    for (int64_t T = 0; T < tend; ++T) {
        if (blockIdx.x == 0 && T > 0) wf_fold<R, NV>(a, T - 1);
        // items of step T: levels l = T (mod P) whose operation (T - l) / P is in [0, nops)
        const int64_t r = T % P;
        const int64_t lmax = T < w.nlevels - 1 ? T : (int64_t)w.nlevels - 1;
        if (lmax >= r) {
            const int64_t lhi = r + (lmax - r) / P * P;
            const int64_t t0 = T - P * (a.nops - 1);
            const int64_t llo = t0 > r ? t0 : r;
            if (llo <= lhi && blockIdx.x > 0) {  // CTA 0 folds the norms instead
                const int32_t i0 = w.lvl_items[2 * llo], i1 = w.lvl_items[2 * lhi + 1];
                for (int32_t i = i0 + (int32_t)blockIdx.x - 1; i < i1; i += (int32_t)gridDim.x - 1)
                    wf_item<R, DIM, REC, LIM>(a, T, i);
            }
        }
        if (T + 1 < tend && !grid_barrier(w.sync, gen, a.wait_ns, a.wk.err, T)) return;
    }
}

template <typename R, int DIM, int REC, int LIM>
cudaError_t wf_launch(const WfArgs<R> &a, int nblocks, cudaStream_t s) {
    void *args[] = {const_cast<WfArgs<R> *>(&a)};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void *>(&k_wavefront<R, DIM, REC, LIM>), dim3(nblocks),
                                       dim3(kWfBlock), args, 0, s);
}

template <typename R, int DIM, int REC, int LIM>
int wf_max_blocks() {
    int dev = 0, nsm = 0, occ = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wavefront<R, DIM, REC, LIM>, kWfBlock, 0) !=
        cudaSuccess)
        return 0;
    return occ * nsm;
}

}  // namespace psst
