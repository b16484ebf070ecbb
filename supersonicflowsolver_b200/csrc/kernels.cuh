// Kernels of the explicit finite-volume loop, templated on the state type R.
//
// This file is compiled twice: kernels_f64.cu (R = double, -fmad=false, the
// parity path) and kernels_f32.cu (R = float, FMA contraction allowed, the
// production path; geometry stays FP64 and is converted per use, the RK state
// w and the residual norms are FP64).
//
// Every expression keeps the reference's operand order and association; with
// FMA contraction off, FP64 results equal the reference's bit for bit. The
// accumulation order per cell is the reference's face-loop order (the CSR is
// sorted by it) for residuals and Green-Gauss gradients, and the cell's own face
// order (the 4-bit permutation wperm) for the local time step and the
// least-squares gradient.
#pragma once
#include <cstdint>

#include "devgrid.hpp"

namespace psst {

enum ErrCode { ERR_HLL = 1, ERR_HLLC = 2, ERR_NONFINITE_RES = 3, ERR_BAD_STATE = 4 };

__device__ __forceinline__ void flag_error(int32_t *err, int code, int id) {
    if (atomicCAS(&err[0], 0, code) == 0) err[1] = id;
}

// psstScalarLimiters.cpp:17-93
template <int LIM, typename R>
__device__ __forceinline__ R limiter_value(R num, R den) {
    const R eps = (R)1.0e-10;
    if ((num > (R)0 && den < (R)0) || (num < (R)0 && den > (R)0)) return (R)0;
    if (fabs(den) < eps) return LIM == 3 ? (R)2 : (R)1;
    R r = num / den;
    if (LIM == 1) return (r * r + r) / (r * r + (R)1);
    if (LIM == 2) return r > (R)1 ? (R)1 : r;
    return (R)2 * r / ((R)1 + r);
}

template <typename R, int DIM>
struct FaceState {
    R p, T, rho, u[DIM];
};

template <typename R, int DIM>
__device__ __forceinline__ void load_state(const DevState<R> &s, int32_t nall, int32_t c, FaceState<R, DIM> &o) {
    o.p = s.p[c];
    o.T = s.T[c];
    o.rho = s.rho[c];
#pragma unroll
    for (int k = 0; k < DIM; ++k) o.u[k] = s.u[(int64_t)k * nall + c];
}

template <typename R, int DIM>
__device__ __forceinline__ R state_var(const FaceState<R, DIM> &s, int i) {
    return i < DIM ? s.u[i] : (i == DIM ? s.p : s.T);
}
template <typename R, int DIM>
__device__ __forceinline__ R &state_var_ref(FaceState<R, DIM> &s, int i) {
    return i < DIM ? s.u[i] : (i == DIM ? s.p : s.T);
}

// psstConvectiveFlow.cpp:13-24
template <typename R>
__device__ __forceinline__ R roe_avg(R lv, R rv, R ld, R rd) {
    R l = sqrt(ld), r = sqrt(rd);
    R num = lv * l + rv * r;
    R den = (l + r);
    return num / den;
}

// One interior face: reconstruction (REC 0 first order, 1 Darwish-Moukalled
// with limiter LIM, 2 cell-limited MUSCL) and the Riemann flux FLUX
// (1 AUSM, 2 HLL, 3 HLLC). Returns false when the wave speeds cannot be
// ordered (the reference throws there).
template <typename R, int DIM, int FLUX, int REC, int LIM>
__device__ __forceinline__ bool interior_flux(const DevGrid &g, const DevState<R> &st, const DevWork<R> &wk,
                                              const Gas &gas, int32_t f, const R nn[DIM], R flow[DIM + 2]) {
    const int32_t c0 = g.c0[f], c1 = g.c1[f];
    FaceState<R, DIM> r[2];
    load_state<R, DIM>(st, g.nall, c0, r[0]);
    load_state<R, DIM>(st, g.nall, c1, r[1]);
    const R rm = (R)gas.rm;
    if (REC == 1) {  // psstReconstructorDM::reconstruct_vals (psstValueReconstructor.cpp:70-134)
        R Rv[DIM];
#pragma unroll
        for (int j = 0; j < DIM; ++j) Rv[j] = (R)(g.xc[(int64_t)j * g.nall + c0] - g.xc[(int64_t)j * g.nall + c1]);
#pragma unroll
        for (int i = 0; i < DIM + 2; ++i) {
            R dl = (R)0, dr = (R)0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                dl += wk.grad[((int64_t)i * DIM + k) * g.nint + c1] * Rv[k];
                dr += wk.grad[((int64_t)i * DIM + k) * g.nint + c0] * Rv[k];
            }
            const R v0 = state_var<R, DIM>(r[0], i), v1 = state_var<R, DIM>(r[1], i);
            const R vlm = v1 - ((R)2 * dl - (v0 - v1));
            const R vlp = v0;
            const R vrm = v1;
            const R vrp = v0 + ((R)2 * dr - (v0 - v1));
            const R nl = vlp - v1, dnl = v1 - vlm;
            const R nr = vrm - v0, dnr = v0 - vrp;
            state_var_ref<R, DIM>(r[0], i) += (R)0.5 * limiter_value<LIM, R>(nr, dnr) * dnr;
            state_var_ref<R, DIM>(r[1], i) += (R)0.5 * limiter_value<LIM, R>(nl, dnl) * dnl;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) r[j].rho = r[j].p / (rm * r[j].T);
    } else if (REC == 2) {  // cell-limited MUSCL (limiters 4, 5)
        const int32_t cc[2] = {c0, c1};
#pragma unroll
        for (int j = 0; j < 2; ++j) {
#pragma unroll
            for (int i = 0; i < DIM + 2; ++i) {
                R d = (R)0;
#pragma unroll
                for (int k = 0; k < DIM; ++k)
                    d += wk.grad[((int64_t)i * DIM + k) * g.nint + cc[j]] *
                         (R)(g.xf[(int64_t)k * g.nface + f] - g.xc[(int64_t)k * g.nall + cc[j]]);
                state_var_ref<R, DIM>(r[j], i) += wk.lim[(int64_t)i * g.nint + cc[j]] * d;
            }
            r[j].rho = r[j].p / (rm * r[j].T);
        }
    }
    const R cp = (R)gas.cp, cv = (R)gas.cv, gamma = (R)gas.gamma;
    R vn[2], a[2], H[2], M[2];
    R fi[2][DIM + 2], wi[2][DIM + 2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        vn[j] = (R)0;
        R vs = (R)0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            vn[j] += r[j].u[k] * nn[k];
            vs += r[j].u[k] * r[j].u[k];
        }
        a[j] = sqrt(gamma * rm * r[j].T);
        H[j] = cp * r[j].T + (R)0.5 * vs;
        if (FLUX == 1) {
            M[j] = vn[j] / a[j];
        } else {
            const R E = cv * r[j].T + (R)0.5 * vs;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                fi[j][k] = r[j].rho * r[j].u[k] * vn[j] + r[j].p * nn[k];
                wi[j][k] = r[j].rho * r[j].u[k];
            }
            wi[j][DIM] = r[j].rho;
            wi[j][DIM + 1] = r[j].rho * E;
            fi[j][DIM] = r[j].rho * vn[j];
            fi[j][DIM + 1] = r[j].rho * vn[j] * H[j];
        }
    }
    if (FLUX == 1) {  // psstConvectiveAUSM::calculate (psstConvectiveFlow.cpp:804-851)
        R Ms1, ps1, Ms0, ps0;
        if (M[1] >= (R)1) {
            Ms1 = M[1];
            ps1 = r[1].p;
        } else if (M[1] <= (R)-1) {
            Ms1 = (R)0;
            ps1 = (R)0;
        } else {
            Ms1 = (R)0.25 * (M[1] + (R)1) * (M[1] + (R)1);
            ps1 = (R)0.25 * r[1].p * (M[1] + (R)1) * (M[1] + (R)1) * ((R)2 - M[1]);
        }
        if (M[0] >= (R)1) {
            Ms0 = (R)0;
            ps0 = (R)0;
        } else if (M[0] <= (R)-1) {
            Ms0 = M[0];
            ps0 = r[0].p;
        } else {
            Ms0 = (R)-0.25 * (M[0] - (R)1) * (M[0] - (R)1);
            ps0 = (R)0.25 * r[0].p * (M[0] - (R)1) * (M[0] - (R)1) * ((R)2 + M[0]);
        }
        const R Mf = Ms0 + Ms1, pf = ps0 + ps1;
        const int sd = Mf > (R)0 ? 1 : 0;
        const R t = Mf * a[sd] * r[sd].rho;
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            const R pfl = pf * nn[j];
            flow[j] = t * r[sd].u[j] + pfl;
        }
        flow[DIM] = t;
        flow[DIM + 1] = t * H[sd];
        return true;
    }
    // Roe-averaged wave speeds (psstConvectiveFlow.cpp:247-266, 531-550)
    const R HR = roe_avg<R>(H[1], H[0], r[1].rho, r[0].rho);
    R vRn = (R)0, vs = (R)0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const R vR = roe_avg<R>(r[1].u[k], r[0].u[k], r[1].rho, r[0].rho);
        vRn += vR * nn[k];
        vs += vR * vR;
    }
    const R aR = sqrt((gamma - (R)1) * (HR - (R)0.5 * vs));
    R s0, s1, t;
    s1 = vn[1] - a[1];
    t = vRn - aR;
    if (s1 > t) s1 = t;
    s0 = vn[0] + a[0];
    t = vRn + aR;
    if (s0 < t) s0 = t;
    if (FLUX == 2) {  // HLL (psstConvectiveFlow.cpp:268-286)
        if (s1 >= (R)0) {
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = fi[1][j];
        } else if (s1 <= (R)0 && s0 >= (R)0) {
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j)
                flow[j] = (s0 * fi[1][j] - s1 * fi[0][j] + s0 * s1 * (wi[0][j] - wi[1][j])) / (s0 - s1);
        } else if (s0 <= (R)0) {
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = fi[0][j];
        } else {
            return false;
        }
        return true;
    }
    // HLLC (psstConvectiveFlow.cpp:552-585)
    const R p0 = r[0].p, p1 = r[1].p, d0 = r[0].rho, d1 = r[1].rho;
    const R sh = (p0 - p1 + d1 * vn[1] * (s1 - vn[1]) - d0 * vn[0] * (s0 - vn[0])) /
                 (d1 * (s1 - vn[1]) - d0 * (s0 - vn[0]));
    if (s1 >= (R)0) {
#pragma unroll
        for (int j = 0; j < DIM + 2; ++j) flow[j] = fi[1][j];
    } else if ((s1 <= (R)0 && sh >= (R)0) || (sh <= (R)0 && s0 >= (R)0)) {
        const int sd = (s1 <= (R)0 && sh >= (R)0) ? 1 : 0;
        const R ss = sd ? s1 : s0;
        const R tt = ss - sh;
        const R pr = r[sd].p, dd = r[sd].rho, vv = vn[sd];
#pragma unroll
        for (int j = 0; j < DIM; ++j)
            flow[j] = (sh * (ss * wi[sd][j] - fi[sd][j]) + ss * (pr + dd * (ss - vv) * (sh - vv)) * nn[j]) / tt;
        flow[DIM] = (sh * (ss * wi[sd][DIM] - fi[sd][DIM])) / tt;
        flow[DIM + 1] = (sh * (ss * wi[sd][DIM + 1] - fi[sd][DIM + 1]) + ss * (pr + dd * (ss - vv) * (sh - vv)) * sh) / tt;
    } else if (s0 <= (R)0) {
#pragma unroll
        for (int j = 0; j < DIM + 2; ++j) flow[j] = fi[0][j];
    } else {
        return false;
    }
    return true;
}

// Face pass: flux * area for every active face (interior faces first, then
// boundary faces whose flux is the physical flux of the ghost state,
// psstConvectiveFlow.cpp:123-202). Output fs[v][f].
template <typename R, int DIM, int FLUX, int REC, int LIM>
__global__ void __launch_bounds__(256) k_face_flux(DevGrid g, DevState<R> st, DevWork<R> wk, Gas gas) {
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nface) return;
    R nn[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) nn[k] = (R)g.n[(int64_t)k * g.nface + f];
    const R S = (R)g.S[f];
    R flow[DIM + 2];
    if (f < g.nfi) {
        if (!interior_flux<R, DIM, FLUX, REC, LIM>(g, st, wk, gas, f, nn, flow)) {
            flag_error(wk.err, FLUX == 2 ? ERR_HLL : ERR_HLLC, f);
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = (R)0;
        }
    } else {
        const int32_t c0 = g.c0[f];
        const int32_t gh = c0 >= g.nint ? c0 : g.c1[f];
        FaceState<R, DIM> s;
        load_state<R, DIM>(st, g.nall, gh, s);
        R vn = (R)0, vs = (R)0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            vn += s.u[k] * nn[k];
            vs += s.u[k] * s.u[k];
        }
        const R H = (R)gas.cp * s.T + (R)0.5 * vs;
#pragma unroll
        for (int k = 0; k < DIM; ++k) flow[k] = s.rho * s.u[k] * vn + s.p * nn[k];
        flow[DIM] = s.rho * vn;
        flow[DIM + 1] = s.rho * vn * H;
    }
#pragma unroll
    for (int j = 0; j < DIM + 2; ++j) wk.fs[(int64_t)j * g.nface + f] = flow[j] * S;
}

template <typename R>
__device__ __forceinline__ R cell_var(const DevState<R> &st, int32_t nall, int DIM, int i, int32_t c) {
    return i < DIM ? st.u[(int64_t)i * nall + c] : (i == DIM ? st.p[c] : st.T[c]);
}

// psstGreenGauss::calculate (psstGradCalculation.cpp:80-177) as a per-cell
// gather: grad_c += sign * (beta*phi0 + (1-beta)*phi1) * S/V_c * n, sign -1 on
// side 0, +1 on side 1, faces in the reference's loop order. Followed, for
// limiters 4/5, by the Barth-Jespersen / Venkatakrishnan cell limiter.
template <typename R, int DIM, int GRAD, int CELLLIM>
__global__ void __launch_bounds__(256) k_gradient(DevGrid g, DevState<R> st, DevWork<R> wk) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nint) return;
    constexpr int NVAR = DIM + 2;
    R gr[NVAR][DIM];
#pragma unroll
    for (int i = 0; i < NVAR; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) gr[i][k] = (R)0;
    const int32_t b = g.csr_ptr[c], e = g.csr_ptr[c + 1];
    if (GRAD == 1) {
        const double V = g.V[c];
        for (int32_t q = b; q < e; ++q) {
            const int32_t ent = g.csr_ent[q];
            const int32_t f = ent >> 1, side = ent & 1;
            const int32_t c0 = g.c0[f], c1 = g.c1[f];
            const R beta = (R)g.beta[f];
            const R rbeta = (R)1 - beta;
            const R gp = (R)(g.S[f] / V);
            const R sgn = side ? (R)1 : (R)-1;
            R nk[DIM];
#pragma unroll
            for (int k = 0; k < DIM; ++k) nk[k] = (R)g.n[(int64_t)k * g.nface + f];
#pragma unroll
            for (int i = 0; i < NVAR; ++i) {
                const R tv = beta * cell_var<R>(st, g.nall, DIM, i, c0) + rbeta * cell_var<R>(st, g.nall, DIM, i, c1);
#pragma unroll
                for (int k = 0; k < DIM; ++k) gr[i][k] += sgn * tv * gp * nk[k];
            }
        }
    } else {  // psstLeastSquare::calculate (:268-368), 2D, cell's own face order
        const R r0 = (R)g.lsq_r[c], r1 = (R)g.lsq_r[(int64_t)g.nint + c], r2 = (R)g.lsq_r[2 * (int64_t)g.nint + c];
        const uint64_t perm = g.wperm[c];
        const R xc0 = (R)g.xc[c], xc1 = (R)g.xc[(int64_t)g.nall + c];
        for (int32_t j = 0; j < e - b; ++j) {
            const int32_t ent = g.csr_ent[b + (int32_t)((perm >> (4 * j)) & 15)];
            const int32_t f = ent >> 1, side = ent & 1;
            const int32_t nb = side ? g.c0[f] : g.c1[f];
            R diff[2];
            diff[0] = (R)g.xc[nb] - xc0;
            diff[1] = (R)g.xc[(int64_t)g.nall + nb] - xc1;
            R w = (R)0;
            w += diff[0] * diff[0];
            w += diff[1] * diff[1];
            const R ws = (R)1 / w;
            const R al0 = diff[0] / (r0 * r0);
            const R al1 = (diff[1] - r1 / r0 * diff[0]) / (r2 * r2);
            const R th[2] = {al0 - r1 / r0 * al1, al1};
#pragma unroll
            for (int i = 0; i < NVAR; ++i) {
                const R phi = (cell_var<R>(st, g.nall, DIM, i, nb) - cell_var<R>(st, g.nall, DIM, i, c));
#pragma unroll
                for (int k = 0; k < 2; ++k) gr[i][k] += ws * th[k] * phi;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NVAR; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) wk.grad[((int64_t)i * DIM + k) * g.nint + c] = gr[i][k];
    if (CELLLIM) {
        // Barth & Jespersen (AIAA 89-0366) / Venkatakrishnan (AIAA 93-0880):
        // psi = min over faces of phi(Delta+, Delta-), Delta- = grad . (x_f - x_c)
        const R eps2 = CELLLIM == 5 ? (R)g.vk_eps2[c] : (R)0;
        const uint64_t perm = g.wperm[c];
#pragma unroll
        for (int i = 0; i < NVAR; ++i) {
            const R phic = cell_var<R>(st, g.nall, DIM, i, c);
            R mx = phic, mn = phic;
            for (int32_t q = b; q < e; ++q) {
                const int32_t ent = g.csr_ent[q];
                const int32_t nb = (ent & 1) ? g.c0[ent >> 1] : g.c1[ent >> 1];
                const R v = cell_var<R>(st, g.nall, DIM, i, nb);
                if (v > mx) mx = v;
                if (v < mn) mn = v;
            }
            R psi = (R)1;
            for (int32_t j = 0; j < e - b; ++j) {
                const int32_t f = g.csr_ent[b + (int32_t)((perm >> (4 * j)) & 15)] >> 1;
                R dm = (R)0;
#pragma unroll
                for (int k = 0; k < DIM; ++k)
                    dm += gr[i][k] * (R)(g.xf[(int64_t)k * g.nface + f] - g.xc[(int64_t)k * g.nall + c]);
                R pf = (R)1;
                if (dm != (R)0) {
                    const R dp = dm > (R)0 ? mx - phic : mn - phic;
                    if (CELLLIM == 4) {
                        const R y = dp / dm;
                        pf = y < (R)1 ? y : (R)1;
                    } else {
                        const R num = (dp * dp + eps2) + (R)2 * dm * dp;
                        const R den = dp * dp + (R)2 * dm * dm + dm * dp + eps2;
                        pf = num / den;
                    }
                }
                if (pf < psi) psi = pf;
            }
            wk.lim[(int64_t)i * g.nint + c] = psi;
        }
    }
}

// Local time step of one cell (psstLocalTimeCalculation.cpp:90-131, 175-213),
// faces in the cell's own order. nbP chooses the state each neighbour is read
// from (the sequential mode reads already-updated neighbours from `nxt`).
template <typename R, int DIM, int LC, bool SEQ>
__device__ __forceinline__ double local_time(const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt,
                                             const Gas &gas, double cfl, double dt_uniform, int32_t c) {
    if (LC == 0) return dt_uniform;
    const int32_t b = g.csr_ptr[c], e = g.csr_ptr[c + 1];
    const uint64_t perm = g.wperm[c];
    const R gr = (R)gas.gamma * (R)gas.rm;
    const R Tc = cur.T[c];
    const R cc = sqrt(gr * Tc);
    R uc[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) uc[k] = cur.u[(int64_t)k * g.nall + c];
    R den = (R)0;
    if (LC == 1) {
        R nnb = (R)0;
        int32_t myrank = 0;
        if (SEQ) myrank = g.rank[c];
        for (int32_t j = 0; j < e - b; ++j) {
            const int32_t ent = g.csr_ent[b + (int32_t)((perm >> (4 * j)) & 15)];
            const int32_t f = ent >> 1;
            const int32_t nb = (ent & 1) ? g.c0[f] : g.c1[f];
            const DevState<R> &src = (SEQ && nb < g.nint && g.rank[nb] < myrank) ? nxt : cur;
            const R cn = (sqrt(gr * src.T[nb]) + cc) * (R)0.5;
            R nv = (R)0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                const R t = (R)g.n[(int64_t)k * g.nface + f];
                nv += uc[k] * t;
                nnb += src.u[(int64_t)k * g.nall + nb] * t;
            }
            nnb = (nnb + nv) * (R)0.5;
            den += (fabs(nnb) + cn) * (R)g.S[f];
        }
    } else {
        R s[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) s[k] = (R)0;
        for (int32_t j = 0; j < e - b; ++j) {
            const int32_t f = g.csr_ent[b + (int32_t)((perm >> (4 * j)) & 15)] >> 1;
            const R S = (R)g.S[f];
#pragma unroll
            for (int k = 0; k < DIM; ++k) s[k] += S * fabs((R)g.n[(int64_t)k * g.nface + f]);
        }
#pragma unroll
        for (int k = 0; k < DIM; ++k) den += (fabs(uc[k]) + cc) * s[k] * (R)0.5;
    }
    return (double)((R)cfl * (R)g.V[c] / den);
}

template <typename R>
__device__ __forceinline__ void atomic_max_pos(unsigned long long *addr, R v) {
    const double d = fabs((double)v);
    if (d == d) atomicMax(addr, (unsigned long long)__double_as_longlong(d));
}

// Cell pass of one RK stage for one cell (psstFiniteVolumeGrid.cpp:317-347):
// residual gather in face-loop order, local time step, w = prev_w - dt*a*res/V,
// max|res|, primitives. Writes the next primitive buffer.
template <typename R, int DIM, int LC, bool SEQ, bool GATHER>
__device__ __forceinline__ void update_cell(const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt,
                                            const DevWork<R> &wk, const Gas &gas, double cfl, double dt_uniform,
                                            double alpha, int first_stage, int it_slot, int32_t c, double sq[DIM + 2]) {
    constexpr int NV = DIM + 2;
    R res[NV];
    if (GATHER) {
#pragma unroll
        for (int v = 0; v < NV; ++v) res[v] = (R)0;
        const int32_t b = g.csr_ptr[c], e = g.csr_ptr[c + 1];
        for (int32_t q = b; q < e; ++q) {
            const int32_t ent = g.csr_ent[q];
            const int32_t f = ent >> 1;
            if (ent & 1) {
#pragma unroll
                for (int v = 0; v < NV; ++v) res[v] += wk.fs[(int64_t)v * g.nface + f];
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) res[v] -= wk.fs[(int64_t)v * g.nface + f];
            }
        }
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) res[v] = wk.res[(int64_t)v * g.nint + c];
    }
    const double dt = local_time<R, DIM, LC, SEQ>(g, cur, nxt, gas, cfl, dt_uniform, c);
    wk.dt[c] = dt;
    const double vol = g.V[c];
    double w[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const int64_t idx = (int64_t)v * g.nint + c;
        double pw;
        if (first_stage) {
            pw = wk.w[idx];
            wk.pw[idx] = pw;
        } else {
            pw = wk.pw[idx];
        }
        w[v] = pw - dt * alpha * (double)res[v] / vol;
        wk.w[idx] = w[v];
        atomic_max_pos<R>(&wk.linf[it_slot * NV + v], res[v]);
        const double rv = (double)res[v];
        sq[v] += rv * rv;
        if (!(rv - rv == 0.0)) flag_error(wk.err, ERR_NONFINITE_RES, c);
    }
    const double rho = w[DIM];
    double vs = 0.0;
    double u[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        u[k] = w[k] / rho;
        vs += u[k] * u[k];
    }
    const double T = ((w[DIM + 1] / rho) - (vs * 0.5)) / gas.cv;
    const double p = rho * gas.rm * T;
    if (!(rho > 0.0 && T > 0.0)) flag_error(wk.err, ERR_BAD_STATE, c);
    nxt.rho[c] = (R)rho;
#pragma unroll
    for (int k = 0; k < DIM; ++k) nxt.u[(int64_t)k * g.nall + c] = (R)u[k];
    nxt.T[c] = (R)T;
    nxt.p[c] = (R)p;
}

template <int NV>
__device__ __forceinline__ void block_sum_sq(double sq[NV], double *l2part) {
    __shared__ double red[NV][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double x = sq[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (lane == 0) red[v][wid] = x;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        const int nw = (blockDim.x + 31) >> 5;
        for (int i = 0; i < nw; ++i) s += red[threadIdx.x][i];
        l2part[(int64_t)blockIdx.x * NV + threadIdx.x] = s;
    }
}

template <typename R, int DIM, int LC, bool GATHER>
__global__ void __launch_bounds__(256) k_cell_update(DevGrid g, DevState<R> cur, DevState<R> nxt, DevWork<R> wk, Gas gas,
                                                     double cfl, double dt_uniform, double alpha, int first_stage,
                                                     int it_slot) {
    constexpr int NV = DIM + 2;
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    double sq[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) sq[v] = 0.0;
    if (c < g.nint)
        update_cell<R, DIM, LC, false, GATHER>(g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, first_stage, it_slot, c, sq);
    block_sum_sq<NV>(sq, wk.l2part);
}

// Sequential LocalAccTime1 (the reference's in-loop evaluation order,
// psstFiniteVolumeGrid.cpp:317-323): cells grouped into levels so that every
// cell's earlier-ranked neighbours sit in lower levels; one block walks the
// levels with a barrier between them, and each cell reads earlier-ranked
// neighbours from the next buffer and the others from the current one.
template <typename R, int DIM, bool GATHER>
__global__ void __launch_bounds__(1024) k_cell_update_seq(DevGrid g, DevState<R> cur, DevState<R> nxt, DevWork<R> wk,
                                                          Gas gas, double cfl, double alpha, int first_stage, int it_slot) {
    constexpr int NV = DIM + 2;
    double sq[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) sq[v] = 0.0;
    for (int32_t l = 0; l < g.nlevels; ++l) {
        const int32_t b = g.lvl_ptr[l], e = g.lvl_ptr[l + 1];
        for (int32_t i = b + threadIdx.x; i < e; i += blockDim.x)
            update_cell<R, DIM, 1, true, GATHER>(g, cur, nxt, wk, gas, cfl, 0.0, alpha, first_stage, it_slot,
                                                 g.lvl_cells[i], sq);
        __threadfence_block();
        __syncthreads();
    }
    block_sum_sq<NV>(sq, wk.l2part);
}

// Ghost cells after the interior update (psstFiniteVolumeGrid.cpp:351-366):
// dynamic condition, thermal condition, rho = p/(T*rm).
template <typename R, int DIM>
__global__ void __launch_bounds__(256) k_ghost_update(DevGrid g, DevState<R> cur, DevState<R> nxt, Gas gas) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nghost) return;
    const int32_t c = g.nint + i;
    const int32_t nb = g.g_nb[i], f = g.g_face[i], z = g.g_zone[i];
    R p = cur.p[c], T = cur.T[c], u[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) u[k] = cur.u[(int64_t)k * g.nall + c];
    const int dyn = g.z_dyn[z], th = g.z_therm[z];
    if (dyn == 26) {  // psstSupersonicOutlet (psstBoundaryCondition.cpp:72-80)
#pragma unroll
        for (int k = 0; k < DIM; ++k) u[k] = nxt.u[(int64_t)k * g.nall + nb];
        p = nxt.p[nb];
    } else if (dyn == 15) {  // psstInviscidWall (:108-127)
        R vn = (R)0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) vn += nxt.u[(int64_t)k * g.nall + nb] * (R)g.n[(int64_t)k * g.nface + f];
#pragma unroll
        for (int k = 0; k < DIM; ++k)
            u[k] = nxt.u[(int64_t)k * g.nall + nb] - vn * (R)g.n[(int64_t)k * g.nface + f];
        p = nxt.p[nb];
    } else if (dyn == 25) {  // psstOutlet (:212-219)
#pragma unroll
        for (int k = 0; k < DIM; ++k) u[k] = nxt.u[(int64_t)k * g.nall + nb];
    }
    if (th == 25 || th == 18) T = nxt.T[nb];  // (:285-288, :354-357)
    nxt.p[c] = p;
    nxt.T[c] = T;
#pragma unroll
    for (int k = 0; k < DIM; ++k) nxt.u[(int64_t)k * g.nall + c] = u[k];
    nxt.rho[c] = p / (T * (R)gas.rm);
}

// residual gather into wk.res (stage-by-stage API)
template <typename R, int DIM>
__global__ void __launch_bounds__(256) k_residual(DevGrid g, DevWork<R> wk) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nint) return;
    constexpr int NV = DIM + 2;
    R res[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) res[v] = (R)0;
    for (int32_t q = g.csr_ptr[c]; q < g.csr_ptr[c + 1]; ++q) {
        const int32_t ent = g.csr_ent[q];
        const int32_t f = ent >> 1;
        if (ent & 1) {
#pragma unroll
            for (int v = 0; v < NV; ++v) res[v] += wk.fs[(int64_t)v * g.nface + f];
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) res[v] -= wk.fs[(int64_t)v * g.nface + f];
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) wk.res[(int64_t)v * g.nint + c] = res[v];
}

// RMS of one stage from the block partials, folded into the iteration's max.
template <int NV>
__global__ void k_l2_finish(const double *l2part, int nblocks, int32_t nint, double *l2, int it_slot) {
    const int v = threadIdx.x;
    if (v >= NV) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += l2part[(int64_t)b * NV + v];
    const double r = sqrt(s / (double)(nint > 0 ? nint : 1));
    if (r > l2[it_slot * NV + v]) l2[it_slot * NV + v] = r;
}

// explicit_solve prologue (psstFiniteVolumeGrid.cpp:279-300) for interior cells,
// plus rho = p/(rm*T) for every volume.
template <typename R, int DIM>
__global__ void k_prologue(DevGrid g, DevState<R> st, DevWork<R> wk, Gas gas) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nall) return;
    const double p = (double)st.p[c], T = (double)st.T[c];
    const double rho = p / (gas.rm * T);
    st.rho[c] = (R)rho;
    if (c >= g.nint) return;
    double vs = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const double t = (double)st.u[(int64_t)k * g.nall + c];
        wk.w[(int64_t)k * g.nint + c] = rho * t;
        vs += t * t;
    }
    const double E = gas.cv * T + 0.5 * vs;
    wk.w[(int64_t)DIM * g.nint + c] = rho;
    wk.w[(int64_t)(DIM + 1) * g.nint + c] = rho * E;
}

}  // namespace psst
