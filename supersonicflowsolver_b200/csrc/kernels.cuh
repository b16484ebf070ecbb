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
//
// One RK stage (parallel modes) is two launches: k_face (one thread per face:
// reconstruction + flux, written as a per-face output record together with the
// face's local-time-step terms) and k_cell (one thread per interior cell:
// in-order gather of its faces' records, time step, RK update, its ghosts,
// norms). Each interior face's flux is computed once.
#pragma once
#include <cstddef>
#include <cstdint>

#include "devgrid.hpp"

// Register budgets of the three hot kernels on the FP32 path (compile-time
// tuning; the values are the measured best on the 6M-tet benchmark): k_face
// register cap, k_cell and k_gradient minimum resident 256-thread blocks per
// SM (gradient: 3, room for the pipelined loop's next-face records). The
// FP64 instantiations (twice the registers per value) get budgets that do
// not spill.
#ifndef PSST_FACE_MAXNREG
#define PSST_FACE_MAXNREG 48
#endif
#ifndef PSST_FACE_MAXNREG_DM  // the DM reconstruction holds both neighbours' projections
#define PSST_FACE_MAXNREG_DM 56
#endif
#ifndef PSST_CELL_MINB
#define PSST_CELL_MINB 4
#endif
#ifndef PSST_GRAD_MINB
#define PSST_GRAD_MINB 3
#endif
#define PSST_BUDGET(R, f32, f64) (sizeof(R) == 8 ? (f64) : (f32))
#ifndef PSST_GRAD_PIPE
#define PSST_GRAD_PIPE 1  // software-pipelined Green-Gauss loop on all-tet meshes
#endif

namespace psst {

enum ErrCode { ERR_HLL = 1, ERR_HLLC = 2, ERR_NONFINITE_RES = 3, ERR_BAD_STATE = 4, ERR_TIMEOUT = 5 };

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ void flag_error(int32_t *err, int code, int id) {
    if (atomicCAS(&err[0], 0, code) == 0) err[1] = id;
}

// Record loads and stores. Record arrays start on cudaMalloc boundaries, so a
// record whose size is a multiple of 32 bytes is 32-byte aligned and moves
// with 256-bit accesses (sm_100 ld/st.global.v8.b32: one L1 request per
// record instead of two for the 32-byte cell records and face outputs);
// other records with 128-bit ones.
//
// ldg: for records the running kernel does not write (the asm has no memory
// dependence, so the compiler may schedule it freely).
template <typename T>
__device__ __forceinline__ T ldg(const T *p) {
    static_assert(sizeof(T) % 16 == 0, "record size must be a multiple of 16 bytes");
    union U {
        T t;
        uint32_t w[sizeof(T) / 4];
        int4 v[sizeof(T) / 16];
        __device__ U() {}
    } u;
    if constexpr (sizeof(T) % 32 == 0) {
        const char *q = reinterpret_cast<const char *>(p);
#pragma unroll
        for (int i = 0; i < (int)(sizeof(T) / 32); ++i)
            asm("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                : "=r"(u.w[8 * i]), "=r"(u.w[8 * i + 1]), "=r"(u.w[8 * i + 2]), "=r"(u.w[8 * i + 3]),
                  "=r"(u.w[8 * i + 4]), "=r"(u.w[8 * i + 5]), "=r"(u.w[8 * i + 6]), "=r"(u.w[8 * i + 7])
                : "l"(q + 32 * i));
    } else {
        const int4 *q = reinterpret_cast<const int4 *>(p);
#pragma unroll
        for (int i = 0; i < (int)(sizeof(T) / 16); ++i) u.v[i] = q[i];
    }
    return u.t;
}

// The reconstruction offsets x_f - x_c of one side of a face record, reading
// only the record's tail that holds them (the 32- or 16-byte chunks from the
// one containing o0 to the end).
template <typename R, int DIM>
__device__ __forceinline__ void face_offsets(const FaceRec<R, DIM> *p, int side, R off[DIM]) {
    using F = FaceRec<R, DIM>;
    constexpr size_t CH = sizeof(F) % 32 == 0 ? 32 : 16;
    constexpr size_t FROM = offsetof(F, o0) / CH * CH;
    constexpr int NW = (int)((sizeof(F) - FROM) / 4);
    union U {
        uint32_t w[NW];
        unsigned char b[NW * 4];
        __device__ U() {}
    } u;
    const char *q = reinterpret_cast<const char *>(p) + FROM;
    if constexpr (CH == 32) {
#pragma unroll
        for (int i = 0; i < NW / 8; ++i)
            asm("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                : "=r"(u.w[8 * i]), "=r"(u.w[8 * i + 1]), "=r"(u.w[8 * i + 2]), "=r"(u.w[8 * i + 3]),
                  "=r"(u.w[8 * i + 4]), "=r"(u.w[8 * i + 5]), "=r"(u.w[8 * i + 6]), "=r"(u.w[8 * i + 7])
                : "l"(q + 32 * i));
    } else {
#pragma unroll
        for (int i = 0; i < NW / 4; ++i) {
            const int4 v = *reinterpret_cast<const int4 *>(q + 16 * i);
            u.w[4 * i] = (uint32_t)v.x, u.w[4 * i + 1] = (uint32_t)v.y, u.w[4 * i + 2] = (uint32_t)v.z,
                   u.w[4 * i + 3] = (uint32_t)v.w;
        }
    }
    constexpr size_t A0 = offsetof(F, o0) - FROM, A1 = offsetof(F, o1) - FROM;  // constant: stays in registers
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        R x0, x1;
        memcpy(&x0, u.b + A0 + k * sizeof(R), sizeof(R));
        memcpy(&x1, u.b + A1 + k * sizeof(R), sizeof(R));
        off[k] = side ? x1 : x0;
    }
}

// ld16: plain 128-bit loads, for records that other threads of the same
// kernel may have written before a barrier (sequential LocalAccTime1).
template <typename T>
__device__ __forceinline__ T ld16(const T *p) {
    static_assert(sizeof(T) % 16 == 0, "record size must be a multiple of 16 bytes");
    union U {
        T t;
        int4 v[sizeof(T) / 16];
        __device__ U() {}
    } u;
    const int4 *q = reinterpret_cast<const int4 *>(p);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 16); ++i) u.v[i] = q[i];
    return u.t;
}
// ldcg: 128-bit loads through L2 only (ld.global.cg), for records that other
// CTAs of a persistent launch write between its grid barriers: an L1-cached
// load could return a line this SM kept from before the write. Volatile, so
// the compiler neither merges nor hoists it across steps.
template <typename T>
__device__ __forceinline__ T ldcg(const T *p) {
    static_assert(sizeof(T) % 16 == 0, "record size must be a multiple of 16 bytes");
    union U {
        T t;
        uint32_t w[sizeof(T) / 4];
        __device__ U() {}
    } u;
    const char *q = reinterpret_cast<const char *>(p);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(T) / 16); ++i)
        asm volatile("ld.global.cg.v4.b32 {%0,%1,%2,%3}, [%4];"
                     : "=r"(u.w[4 * i]), "=r"(u.w[4 * i + 1]), "=r"(u.w[4 * i + 2]), "=r"(u.w[4 * i + 3])
                     : "l"(q + 16 * i));
    return u.t;
}
__device__ __forceinline__ double ldcg(const double *p) {
    double v;
    asm volatile("ld.global.cg.f64 %0, [%1];" : "=d"(v) : "l"(p));
    return v;
}
// state and gradient records: ldg in the pass kernels, ldcg in the persistent one
template <bool CG, typename T>
__device__ __forceinline__ T ldst(const T *p) {
    if constexpr (CG)
        return ldcg(p);
    else
        return ldg(p);
}

template <typename T>
__device__ __forceinline__ void st16(T *p, const T &t) {
    static_assert(sizeof(T) % 16 == 0, "record size must be a multiple of 16 bytes");
    union U {
        T t;
        uint32_t w[sizeof(T) / 4];
        int4 v[sizeof(T) / 16];
        __device__ U() {}
    } u;
    u.t = t;
    if constexpr (sizeof(T) % 32 == 0) {
        char *q = reinterpret_cast<char *>(p);
#pragma unroll
        for (int i = 0; i < (int)(sizeof(T) / 32); ++i)
            asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(q + 32 * i), "r"(u.w[8 * i]),
                         "r"(u.w[8 * i + 1]), "r"(u.w[8 * i + 2]), "r"(u.w[8 * i + 3]), "r"(u.w[8 * i + 4]),
                         "r"(u.w[8 * i + 5]), "r"(u.w[8 * i + 6]), "r"(u.w[8 * i + 7])
                         : "memory");
    } else {
        int4 *q = reinterpret_cast<int4 *>(p);
#pragma unroll
        for (int i = 0; i < (int)(sizeof(T) / 16); ++i) q[i] = u.v[i];
    }
}

// psstScalarLimiters.cpp:17-93, r = num / den. FP64 (parity): the
// reference's expressions. FP32: each limiter with num and den multiplied
// through (they have the same sign and |den| >= eps here), one fast division:
// VanAlbada (num^2 + num den) / (num^2 + den^2), MinMod min(num / den, 1),
// VanLeer 2 num / (den + num).
template <int LIM, typename R>
__device__ __forceinline__ R limiter_value(R num, R den) {
    const R eps = (R)1.0e-10;
    if ((num > (R)0 && den < (R)0) || (num < (R)0 && den > (R)0)) return (R)0;
    if (fabs(den) < eps) return LIM == 3 ? (R)2 : (R)1;
    if constexpr (sizeof(R) == 4) {
        if (LIM == 1) return __fdividef(num * num + num * den, num * num + den * den);
        if (LIM == 2) return fabsf(num) > fabsf(den) ? 1.0f : __fdividef(num, den);
        return __fdividef(2.0f * num, den + num);
    }
    R r = num / den;
    if (LIM == 1) return (r * r + r) / (r * r + (R)1);
    if (LIM == 2) return r > (R)1 ? (R)1 : r;
    return (R)2 * r / ((R)1 + r);
}

template <typename R, int DIM>
struct Prim {
    R p, T, rho, u[DIM];
};

template <typename R, int DIM>
__device__ __forceinline__ Prim<R, DIM> unpack(const CellRec<R> &c) {
    Prim<R, DIM> o;
    o.p = c.v[RP];
    o.T = c.v[RT];
    o.rho = c.v[RRHO];
#pragma unroll
    for (int k = 0; k < DIM; ++k) o.u[k] = c.v[RU + k];
    return o;
}
template <typename R, int DIM>
__device__ __forceinline__ CellRec<R> pack(R p, R T, R rho, const R *u) {
    CellRec<R> c;
#pragma unroll
    for (int i = 0; i < 8; ++i) c.v[i] = (R)0;
    c.v[RP] = p;
    c.v[RT] = T;
    c.v[RRHO] = rho;
#pragma unroll
    for (int k = 0; k < DIM; ++k) c.v[RU + k] = u[k];
    return c;
}

// variable i of the reconstructed set: u.. (i < DIM), p (DIM), T (DIM+1)
template <typename R, int DIM>
__device__ __forceinline__ R &pvar(Prim<R, DIM> &s, int i) {
    return i < DIM ? s.u[i] : (i == DIM ? s.p : s.T);
}
template <typename R, int DIM>
__device__ __forceinline__ R pvar(const Prim<R, DIM> &s, int i) {
    return i < DIM ? s.u[i] : (i == DIM ? s.p : s.T);
}

// Division of several numerators by one denominator: FP32, one reciprocal
// and a product each; FP64 (parity), the reference's division each.
template <typename R>
struct SharedDen {
    R d, r;
    __device__ __forceinline__ explicit SharedDen(R den) : d(den), r(sizeof(R) == 4 ? (R)1 / den : (R)0) {}
    __device__ __forceinline__ R operator()(R num) const { return sizeof(R) == 4 ? num * r : num / d; }
};

// psstConvectiveFlow.cpp:13-24
template <typename R>
__device__ __forceinline__ R roe_avg(R lv, R rv, R ld, R rd) {
    R l = sqrt(ld), r = sqrt(rd);
    R num = lv * l + rv * r;
    R den = (l + r);
    return num / den;
}

// Physical flux of a ghost state through a boundary face (psstConvectiveFlow.cpp:123-202).
template <typename R, int DIM>
__device__ __forceinline__ void boundary_flux(const Prim<R, DIM> &s, const R nn[DIM], const Gas &gas, R flow[DIM + 2]) {
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

// One side of the cell-limited MUSCL reconstruction: phi_f = phi_c +
// (psi_c grad(phi)_c) . (x_f - x_c), the record holding psi_c grad(phi)_c;
// rho_f = p_f / (R T_f) as in the DM reconstruction.
template <typename R, int DIM>
__device__ __forceinline__ void muscl_side(Prim<R, DIM> &r, const GradRec<R, DIM> &gr, const R off[DIM], R rm) {
#pragma unroll
    for (int i = 0; i < DIM + 2; ++i) {
        R d = (R)0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) d += gr.g[i * DIM + k] * off[k];
        pvar<R, DIM>(r, i) += d;
    }
    r.rho = r.p / (rm * r.T);
}

// Interior face: reconstruction (REC 0 first order, 1 Darwish-Moukalled with
// limiter LIM, 2 cell-limited MUSCL) and the Riemann flux FLUX (1 AUSM, 2 HLL,
// 3 HLLC). r[0] is neighbour 0 (c0), r[1] neighbour 1. Returns false when the
// wave speeds cannot be ordered (the reference throws there).
template <typename R, int DIM, int FLUX, int REC, int LIM>
__device__ __forceinline__ bool interior_flux(Prim<R, DIM> r[2], const GradRec<R, DIM> *gr0,
                                              const GradRec<R, DIM> *gr1, const FaceRec<R, DIM> &fr,
                                              const R nn[DIM], const Gas &gas, R flow[DIM + 2]) {
    const R rm = (R)gas.rm;
    if (REC == 1) {  // psstReconstructorDM::reconstruct_vals (psstValueReconstructor.cpp:70-134)
        // projections of neighbour 0's gradients first, then neighbour 1's (same
        // sums), so one gradient record is dead before the other is read
        R dra[DIM + 2], dla[DIM + 2];
#pragma unroll
        for (int i = 0; i < DIM + 2; ++i) {
            R dr = (R)0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) dr += gr0->g[i * DIM + k] * fr.o0[k];
            dra[i] = dr;
        }
#pragma unroll
        for (int i = 0; i < DIM + 2; ++i) {
            R dl = (R)0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) dl += gr1->g[i * DIM + k] * fr.o0[k];
            dla[i] = dl;
        }
#pragma unroll
        for (int i = 0; i < DIM + 2; ++i) {
            const R dl = dla[i], dr = dra[i];
            const R v0 = pvar<R, DIM>(r[0], i), v1 = pvar<R, DIM>(r[1], i);
            const R vlm = v1 - ((R)2 * dl - (v0 - v1));
            const R vlp = v0;
            const R vrm = v1;
            const R vrp = v0 + ((R)2 * dr - (v0 - v1));
            const R nl = vlp - v1, dnl = v1 - vlm;
            const R nr = vrm - v0, dnr = v0 - vrp;
            pvar<R, DIM>(r[0], i) += (R)0.5 * limiter_value<LIM, R>(nr, dnr) * dnr;
            pvar<R, DIM>(r[1], i) += (R)0.5 * limiter_value<LIM, R>(nl, dnl) * dnl;
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) r[j].rho = r[j].p / (rm * r[j].T);
    } else if (REC == 2) {  // cell-limited MUSCL (limiters 4, 5)
        muscl_side<R, DIM>(r[0], *gr0, fr.o0, rm);
        muscl_side<R, DIM>(r[1], *gr1, fr.o1, rm);
    }
    const R cp = (R)gas.cp, cv = (R)gas.cv, gamma = (R)gas.gamma;
    R vn[2], a[2], H[2], M[2], vsq[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        vn[j] = (R)0;
        R vs = (R)0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            vn[j] += r[j].u[k] * nn[k];
            vs += r[j].u[k] * r[j].u[k];
        }
        vsq[j] = vs;
        a[j] = sqrt(gamma * rm * r[j].T);
        H[j] = cp * r[j].T + (R)0.5 * vs;
        if (FLUX == 1) M[j] = vn[j] / a[j];
    }
    // physical flux f and conserved state w of side j, formed only in the
    // branch that uses them (same expressions, so the same bits)
    auto side = [&](int j, R f[DIM + 2], R w[DIM + 2]) {
        const R E = cv * r[j].T + (R)0.5 * vsq[j];
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            f[k] = r[j].rho * r[j].u[k] * vn[j] + r[j].p * nn[k];
            w[k] = r[j].rho * r[j].u[k];
        }
        w[DIM] = r[j].rho;
        w[DIM + 1] = r[j].rho * E;
        f[DIM] = r[j].rho * vn[j];
        f[DIM + 1] = r[j].rho * vn[j] * H[j];
    };
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
        const bool sd = Mf > (R)0;  // upwind side: 1 if Mf > 0
        const R t = Mf * (sd ? a[1] : a[0]) * (sd ? r[1].rho : r[0].rho);
#pragma unroll
        for (int j = 0; j < DIM; ++j) {
            const R pfl = pf * nn[j];
            flow[j] = t * (sd ? r[1].u[j] : r[0].u[j]) + pfl;
        }
        flow[DIM] = t;
        flow[DIM + 1] = t * (sd ? H[1] : H[0]);
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
        R f0[DIM + 2], w0[DIM + 2], f1[DIM + 2], w1[DIM + 2];
        if (s1 >= (R)0) {
            side(1, f1, w1);
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = f1[j];
        } else if (s1 <= (R)0 && s0 >= (R)0) {
            side(0, f0, w0);
            side(1, f1, w1);
            const SharedDen<R> q(s0 - s1);
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = q(s0 * f1[j] - s1 * f0[j] + s0 * s1 * (w0[j] - w1[j]));
        } else if (s0 <= (R)0) {
            side(0, f0, w0);
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = f0[j];
        } else {
            return false;
        }
        return true;
    }
    // HLLC (psstConvectiveFlow.cpp:552-585)
    const R p0 = r[0].p, p1 = r[1].p, d0 = r[0].rho, d1 = r[1].rho;
    const R sh = (p0 - p1 + d1 * vn[1] * (s1 - vn[1]) - d0 * vn[0] * (s0 - vn[0])) /
                 (d1 * (s1 - vn[1]) - d0 * (s0 - vn[0]));
    R fs[DIM + 2], ws[DIM + 2];
    if (s1 >= (R)0) {
        side(1, fs, ws);
#pragma unroll
        for (int j = 0; j < DIM + 2; ++j) flow[j] = fs[j];
    } else if ((s1 <= (R)0 && sh >= (R)0) || (sh <= (R)0 && s0 >= (R)0)) {
        const bool sd = (s1 <= (R)0 && sh >= (R)0);  // star state of side 1, else side 0
        const R ss = sd ? s1 : s0;
        const R tt = ss - sh;
        const R pr = sd ? r[1].p : r[0].p, dd = sd ? r[1].rho : r[0].rho, vv = sd ? vn[1] : vn[0];
        if (sd)  // constant side indices: no dynamically indexed (local-memory) arrays
            side(1, fs, ws);
        else
            side(0, fs, ws);
        const SharedDen<R> q(tt);
#pragma unroll
        for (int j = 0; j < DIM + 2; ++j) {
            const R wj = ws[j], fj = fs[j];
            if (j < DIM)
                flow[j] = q(sh * (ss * wj - fj) + ss * (pr + dd * (ss - vv) * (sh - vv)) * nn[j]);
            else if (j == DIM)
                flow[j] = q(sh * (ss * wj - fj));
            else
                flow[j] = q(sh * (ss * wj - fj) + ss * (pr + dd * (ss - vv) * (sh - vv)) * sh);
        }
    } else if (s0 <= (R)0) {
        side(0, fs, ws);
#pragma unroll
        for (int j = 0; j < DIM + 2; ++j) flow[j] = fs[j];
    } else {
        return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// face pass
// ---------------------------------------------------------------------------

// One thread per face: reconstruction + Riemann flux (or the ghost's physical
// flux on boundary faces, psstConvectiveFlow.cpp:123-202), written as
// flux * area, plus the face's local-time-step terms so that the cell pass
// needs neither face geometry nor neighbour states:
//  LocalAccTime1 (psstLocalTimeCalculation.cpp:117-127): u0.n and u1.n per
//   component, the mean sound speed (sqrt(g R T1) + sqrt(g R T0)) / 2 (the
//   reference adds the two sound speeds in the opposite order on the other
//   side; IEEE addition is commutative) and S;
//  LocalAccTime2 (:189-193): S |n_k|.
// Register cap PSST_FACE_MAXNREG on the FP32 path (48: ten 128-thread blocks per SM;
// PSST_FACE_MAXNREG_DM = 56 for the DM reconstruction, which spills at 48 and
// measured 7% faster at 56).
template <typename R, int DIM, int FLUX, int REC, int LIM, int LC>
__global__ void __maxnreg__(PSST_BUDGET(R, REC == 1 ? PSST_FACE_MAXNREG_DM : PSST_FACE_MAXNREG, 128)) k_face(DevGrid g, DevState<R> st, DevWork<R> wk, Gas gas) {
    using FO = FaceOut<R, DIM>;
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= g.nface) return;
    if (g.face_case && !g.case_active[g.face_case[f]]) return;  // stopped case (merged grids)
    const FaceRec<R, DIM> fr = ldg(reinterpret_cast<const FaceRec<R, DIM> *>(g.frec) + f);
    R nn[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) nn[k] = (R)fr.n[k];
    const R S = (R)fr.S;
    const Prim<R, DIM> p0 = unpack<R, DIM>(ldg(st.rec + fr.c0));
    const Prim<R, DIM> p1 = unpack<R, DIM>(ldg(st.rec + fr.c1));
    R flow[DIM + 2];
    if (f < g.nfi) {
        const GradRec<R, DIM> *grec = reinterpret_cast<const GradRec<R, DIM> *>(wk.grec);
        GradRec<R, DIM> g0, g1;
        if (REC) {
            g0 = ldg(grec + fr.c0);
            g1 = ldg(grec + fr.c1);
        }
        Prim<R, DIM> r[2] = {p0, p1};
        if (!interior_flux<R, DIM, FLUX, REC, LIM>(r, &g0, &g1, fr, nn, gas, flow)) {
            flag_error(wk.err, FLUX == 2 ? ERR_HLL : ERR_HLLC, f);
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = (R)0;
        }
    } else {
        boundary_flux<R, DIM>(fr.c0 >= g.nint ? p0 : p1, nn, gas, flow);
    }
    FO o;
#pragma unroll
    for (int i = 0; i < (int)(sizeof(o.v) / sizeof(R)); ++i) o.v[i] = (R)0;
#pragma unroll
    for (int j = 0; j < DIM + 2; ++j) o.v[j] = flow[j] * S;
    if (LC == 1) {
        const R gr = (R)gas.gamma * (R)gas.rm;
        if (FO::NQ == DIM) {
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                o.v[FO::Q0 + k] = p0.u[k] * nn[k];
                o.v[FO::Q1 + k] = p1.u[k] * nn[k];
            }
        } else {
            R a = (R)0, b = (R)0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                a += p0.u[k] * nn[k];
                b += p1.u[k] * nn[k];
            }
            o.v[FO::Q0] = a;
            o.v[FO::Q1] = b;
        }
        o.v[FO::CN] = (sqrt(gr * p1.T) + sqrt(gr * p0.T)) * (R)0.5;
    } else if (LC == 2) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) o.v[FO::Q0 + k] = S * fabs(nn[k]);
    }
    st16(reinterpret_cast<FO *>(wk.fout) + f, o);
}

// ---------------------------------------------------------------------------
// gradients
// ---------------------------------------------------------------------------

// Thread per cell. psstGreenGauss::calculate (psstGradCalculation.cpp:80-177)
// as a per-cell gather: grad_c += sign * (beta*phi0 + (1-beta)*phi1) * S/V_c * n,
// sign -1 on side 0, +1 on side 1, faces in the reference's loop order; or the
// least squares of psstLeastSquare::calculate (:268-368) in the cell's own
// face order: 2D as the reference; 3D as a corrected restatement (the
// reference's 3D branch leaves alpha_1, alpha_2 at zero and writes alpha[3]
// out of bounds, :338): alpha_3 = (dz - r23/r22 dy + beta dx) / r33^2
// (Anderson & Bonhaus 1994), then the reference's theta corrections. Then, for limiters 4/5, the Barth-Jespersen (AIAA 89-0366) /
// Venkatakrishnan (AIAA 93-0880) cell limiter:
// psi = min over faces of phi(Delta+, Delta-), Delta- = grad . (x_f - x_c).
// Gradient (and cell limiter) of one interior cell c from the state records
// `rec`, written to out[c]. CG: state loads through L2 only (the persistent
// wavefront kernel, where other CTAs write the states between its steps).
// FP32 Green-Gauss gradient (and cell limiter) of interior cell c of a mesh
// with 4 faces per cell, from the per-entry table g.gcoef: the cell's 4
// values of each component are one 16-byte load (a warp's load covers whole
// lines), so only the 4 neighbour states are gathered. Face value
// own + w (oth - own), w the neighbour's weight; the sum runs over the faces
// in the cell's CSR order as the general path does.
template <int DIM, int CELLLIM>
__device__ __forceinline__ void gradient_cell_table(const DevGrid &g, const CellRec<float> *rec,
                                                    GradRec<float, DIM> *gout, int32_t c) {
    constexpr int NVAR = DIM + 2;
    const int4 nb = *reinterpret_cast<const int4 *>(g.csr_nb + 4 * c);
    const CellRec<float> r4[4] = {ldg(rec + nb.x), ldg(rec + nb.y), ldg(rec + nb.z), ldg(rec + nb.w)};
    const Prim<float, DIM> own = unpack<float, DIM>(ldg(rec + c));
    const float4 *tab = reinterpret_cast<const float4 *>(g.gcoef) + c;  // component j at tab[j * nint]
    float4 sn[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) sn[k] = tab[(int64_t)k * g.nint];
    const float4 wn = tab[(int64_t)DIM * g.nint];
    auto at = [](const float4 &v, int q) { return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w; };
    float gr[NVAR][DIM], mx[NVAR], mn[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) {
        mx[i] = mn[i] = pvar<float, DIM>(own, i);
#pragma unroll
        for (int k = 0; k < DIM; ++k) gr[i][k] = 0.0f;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const Prim<float, DIM> oth = unpack<float, DIM>(r4[q]);
        const float w = at(wn, q);
#pragma unroll
        for (int i = 0; i < NVAR; ++i) {
            const float a = pvar<float, DIM>(own, i), o = pvar<float, DIM>(oth, i);
            if (CELLLIM) {
                mx[i] = fmaxf(mx[i], o);
                mn[i] = fminf(mn[i], o);
            }
            const float tv = fmaf(w, o - a, a);
#pragma unroll
            for (int k = 0; k < DIM; ++k) gr[i][k] = fmaf(tv, at(sn[k], q), gr[i][k]);
        }
    }
    float lim[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) lim[i] = 1.0f;
    if (CELLLIM) {
        float4 off[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) off[k] = tab[(int64_t)(DIM + 1 + k) * g.nint];
        const float eps2 = CELLLIM == 5 ? (float)g.vk_eps2[c] : 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
#pragma unroll
            for (int i = 0; i < NVAR; ++i) {
                const float phic = pvar<float, DIM>(own, i);
                float dm = 0.0f;
#pragma unroll
                for (int k = 0; k < DIM; ++k) dm += gr[i][k] * at(off[k], q);
                float pf = 1.0f;
                if (dm != 0.0f) {
                    const float dp = dm > 0.0f ? mx[i] - phic : mn[i] - phic;
                    if (CELLLIM == 4) {
                        const float y = __fdividef(dp, dm);
                        pf = y < 1.0f ? y : 1.0f;
                    } else {
                        const float num = (dp * dp + eps2) + 2.0f * dm * dp;
                        const float den = dp * dp + 2.0f * dm * dm + dm * dp + eps2;
                        pf = __fdividef(num, den);
                    }
                }
                if (pf < lim[i]) lim[i] = pf;
            }
        }
    }
    GradRec<float, DIM> out;
#pragma unroll
    for (int i = 0; i < NVAR; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) out.g[i * DIM + k] = CELLLIM ? gr[i][k] * lim[i] : gr[i][k];
    st16(gout + c, out);
}

// FP64 (parity) form of the same: the table holds sign * (S/V), n, beta and
// the offsets exactly as the face records and the general path have them,
// and the operations below are the general path's in its order
// (psstGradCalculation.cpp:80-177): tv = beta phi0 + (1 - beta) phi1, then
// ((sign tv) (S/V)) n_k, where sign tv (S/V) = tv (sign S/V) exactly.
template <int DIM, int CELLLIM>
__device__ __forceinline__ void gradient_cell_table64(const DevGrid &g, const CellRec<double> *rec,
                                                      GradRec<double, DIM> *gout, int32_t c) {
    constexpr int NVAR = DIM + 2;
    const int4 nb = *reinterpret_cast<const int4 *>(g.csr_nb + 4 * c);
    const CellRec<double> r4[4] = {ldg(rec + nb.x), ldg(rec + nb.y), ldg(rec + nb.z), ldg(rec + nb.w)};
    const Prim<double, DIM> own = unpack<double, DIM>(ldg(rec + c));
    // entry q of component j; read per face (the cell's 32 bytes of a component
    // share one line, so the later faces' reads hit L1), which keeps few of the
    // table's values live at once
    const double *tab = reinterpret_cast<const double *>(g.gcoef) + 4 * (int64_t)c;
    auto at = [&](int j, int q) { return __ldg(tab + (int64_t)4 * j * g.nint + q); };
    double gr[NVAR][DIM], mx[NVAR], mn[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) {
        mx[i] = mn[i] = pvar<double, DIM>(own, i);
#pragma unroll
        for (int k = 0; k < DIM; ++k) gr[i][k] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const Prim<double, DIM> oth = unpack<double, DIM>(r4[q]);
        const double gps = at(0, q), beta = at(DIM + 1, q), rbeta = 1.0 - beta;
        double nrm[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) nrm[k] = at(1 + k, q);
        const bool side = gps > 0.0;
#pragma unroll
        for (int i = 0; i < NVAR; ++i) {
            const double a = pvar<double, DIM>(own, i), o = pvar<double, DIM>(oth, i);
            if (CELLLIM) {
                if (o > mx[i]) mx[i] = o;
                if (o < mn[i]) mn[i] = o;
            }
            const double phi0 = side ? o : a, phi1 = side ? a : o;
            const double tv = beta * phi0 + rbeta * phi1;
#pragma unroll
            for (int k = 0; k < DIM; ++k) gr[i][k] += tv * gps * nrm[k];
        }
    }
    double lim[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) lim[i] = 1.0;
    if (CELLLIM) {
        const double eps2 = CELLLIM == 5 ? g.vk_eps2[c] : 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double off[DIM];
#pragma unroll
            for (int k = 0; k < DIM; ++k) off[k] = at(DIM + 2 + k, q);
#pragma unroll
            for (int i = 0; i < NVAR; ++i) {
                const double phic = pvar<double, DIM>(own, i);
                double dm = 0.0;
#pragma unroll
                for (int k = 0; k < DIM; ++k) dm += gr[i][k] * off[k];
                double pf = 1.0;
                if (dm != 0.0) {
                    const double dp = dm > 0.0 ? mx[i] - phic : mn[i] - phic;
                    if (CELLLIM == 4) {
                        const double y = dp / dm;
                        pf = y < 1.0 ? y : 1.0;
                    } else {
                        const double num = (dp * dp + eps2) + 2.0 * dm * dp;
                        const double den = dp * dp + 2.0 * dm * dm + dm * dp + eps2;
                        pf = num / den;
                    }
                }
                if (pf < lim[i]) lim[i] = pf;
            }
        }
    }
    GradRec<double, DIM> out;
#pragma unroll
    for (int i = 0; i < NVAR; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) out.g[i * DIM + k] = CELLLIM ? gr[i][k] * lim[i] : gr[i][k];
    st16(gout + c, out);
}

template <typename R, int DIM, int GRAD, int CELLLIM, bool CG>
__device__ __forceinline__ void gradient_cell(const DevGrid &g, const CellRec<R> *rec, GradRec<R, DIM> *gout,
                                              int32_t c) {
    if constexpr (GRAD == 1 && !CG) {
        if (g.gcoef) {
            if constexpr (sizeof(R) == 4)
                gradient_cell_table<DIM, CELLLIM>(g, rec, gout, c);
            else
                gradient_cell_table64<DIM, CELLLIM>(g, rec, gout, c);
            return;
        }
    }
    constexpr int NVAR = DIM + 2;
    const FaceRec<R, DIM> *frec = reinterpret_cast<const FaceRec<R, DIM> *>(g.frec);
    // uniform meshes (all tets, all hexes): the CSR range follows from c, one
    // dependent load less
    const int32_t b = g.kuni ? c * g.kuni : g.csr_ptr[c], K = g.kuni ? g.kuni : g.csr_ptr[c + 1] - b;
    const Prim<R, DIM> own = unpack<R, DIM>(ldst<CG>(rec + c));
    R gr[NVAR][DIM];
#pragma unroll
    for (int i = 0; i < NVAR; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) gr[i][k] = (R)0;
    const uint64_t perm = g.wperm[c];
    // min/max of each variable over the face neighbours for limiters 4/5
    // (order-free), gathered in the same pass as the gradient
    R mx[NVAR], mn[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) mx[i] = mn[i] = pvar<R, DIM>(own, i);
    // FP64 (parity) path: the reference's arithmetic; FP32 path: one
    // reciprocal of V per cell and fast divisions in the limiter
    constexpr bool EXACT = sizeof(R) == 8;
    // all-tet meshes: the four CSR entries and neighbours of the cell as two
    // 16-byte loads up front (b = 4c), so each face costs one dependent load
    // round trip instead of two
    const bool u4 = g.kuni == 4;
    int4 e4 = make_int4(0, 0, 0, 0), n4 = make_int4(0, 0, 0, 0);
    if (u4) {
        e4 = *reinterpret_cast<const int4 *>(g.csr_ent + b);
        if (GRAD == 1) n4 = *reinterpret_cast<const int4 *>(g.csr_nb + b);
    }
    auto pick = [](const int4 &v, int32_t q) { return q == 0 ? v.x : q == 1 ? v.y : q == 2 ? v.z : v.w; };
    if (GRAD == 1) {
        const double V = g.V[c];
        const double rV = EXACT ? 0.0 : 1.0 / V;
        auto face = [&](int32_t ent, const FaceRec<R, DIM> &fr, const Prim<R, DIM> &oth, R beta) {
            const int32_t side = ent & 1;
            if (CELLLIM)
#pragma unroll
                for (int i = 0; i < NVAR; ++i) {
                    const R v = pvar<R, DIM>(oth, i);
                    if (v > mx[i]) mx[i] = v;
                    if (v < mn[i]) mn[i] = v;
                }
            const R rbeta = (R)1 - beta;
            const R gp = EXACT ? (R)(fr.S / V) : (R)(fr.S * rV);
            const R sgn = side ? (R)1 : (R)-1;
#pragma unroll
            for (int i = 0; i < NVAR; ++i) {
                const R a = pvar<R, DIM>(own, i), o = pvar<R, DIM>(oth, i);
                const R phi0 = side ? o : a, phi1 = side ? a : o;  // neighbour 0 / 1 values
                const R tv = beta * phi0 + rbeta * phi1;
#pragma unroll
                for (int k = 0; k < DIM; ++k) gr[i][k] += sgn * tv * gp * (R)fr.n[k];
            }
        };
#if PSST_GRAD_PIPE
        if (u4) {  // software pipeline: the next face's records load while this face is summed
            int32_t en = e4.x;
            FaceRec<R, DIM> frn = ldg(frec + (en >> 1));
            CellRec<R> recn = ldst<CG>(rec + n4.x);
            R betan = (R)g.beta[en >> 1];
            for (int32_t q = 0; q < 4; ++q) {
                const int32_t ent = en;
                const FaceRec<R, DIM> fr = frn;
                const Prim<R, DIM> oth = unpack<R, DIM>(recn);
                const R beta = betan;
                if (q < 3) {
                    en = pick(e4, q + 1);
                    frn = ldg(frec + (en >> 1));
                    recn = ldst<CG>(rec + pick(n4, q + 1));
                    betan = (R)g.beta[en >> 1];
                }
                face(ent, fr, oth, beta);
            }
        } else
#endif
        for (int32_t q = 0; q < K; ++q) {  // not unrolled: fewer registers, more blocks (measured faster)
            const int32_t ent = u4 ? pick(e4, q) : g.csr_ent[b + q];
            face(ent, ldg(frec + (ent >> 1)), unpack<R, DIM>(ldst<CG>(rec + (u4 ? pick(n4, q) : g.csr_nb[b + q]))),
                 (R)g.beta[ent >> 1]);
        }
    } else {
        constexpr int NR = DIM == 2 ? 3 : 7;  // r11 r12 r22 (r13 r23 r33 beta)
        R r[NR], xo[DIM];
#pragma unroll
        for (int q = 0; q < NR; ++q) r[q] = (R)g.lsq_r[(int64_t)q * g.nint + c];
#pragma unroll
        for (int k = 0; k < DIM; ++k) xo[k] = (R)g.xc[(int64_t)k * g.nall + c];
        for (int32_t j = 0; j < K; ++j) {
            const int32_t slot = b + (int32_t)((perm >> (4 * j)) & 15);
            const int32_t nb = g.csr_nb[slot];
            const Prim<R, DIM> oth = unpack<R, DIM>(ldst<CG>(rec + nb));
            if (CELLLIM)
#pragma unroll
                for (int i = 0; i < NVAR; ++i) {
                    const R v = pvar<R, DIM>(oth, i);
                    if (v > mx[i]) mx[i] = v;
                    if (v < mn[i]) mn[i] = v;
                }
            R diff[DIM];
            R w = (R)0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                diff[k] = (R)g.xc[(int64_t)k * g.nall + nb] - xo[k];
                w += diff[k] * diff[k];
            }
            const R ws = (R)1 / w;
            const R al0 = diff[0] / (r[0] * r[0]);
            const R al1 = (diff[1] - r[1] / r[0] * diff[0]) / (r[2] * r[2]);
            R th[DIM];
            th[0] = al0 - r[1] / r[0] * al1;
            th[1] = al1;
            if constexpr (DIM == 3) {  // corrected 3D restatement (see above)
                const R al2 = (diff[2] - r[4] / r[2] * diff[1] + r[6] * diff[0]) / (r[5] * r[5]);
                th[0] += al2 * r[6];
                th[1] -= r[4] / r[2] * al2;
                th[2] = al2;
            }
#pragma unroll
            for (int i = 0; i < NVAR; ++i) {
                const R phi = (pvar<R, DIM>(oth, i) - pvar<R, DIM>(own, i));
#pragma unroll
                for (int k = 0; k < DIM; ++k) gr[i][k] += ws * th[k] * phi;
            }
        }
    }
    R lim[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; ++i) lim[i] = (R)1;
    if (CELLLIM) {
        const R eps2 = CELLLIM == 5 ? (R)g.vk_eps2[c] : (R)0;
        for (int32_t q = 0; q < K; ++q) {
            const int32_t ent = u4 ? pick(e4, q) : g.csr_ent[b + q];
            R off[DIM];  // x_f - x_c of this cell
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
                        const R y = EXACT ? dp / dm : (R)__fdividef((float)dp, (float)dm);
                        pf = y < (R)1 ? y : (R)1;
                    } else {
                        const R num = (dp * dp + eps2) + (R)2 * dm * dp;
                        const R den = dp * dp + (R)2 * dm * dm + dm * dp + eps2;
                        pf = EXACT ? num / den : (R)__fdividef((float)num, (float)den);
                    }
                }
                if (pf < lim[i]) lim[i] = pf;
            }
        }
    }
    GradRec<R, DIM> out;
#pragma unroll
    for (int i = 0; i < NVAR; ++i)
#pragma unroll
        for (int k = 0; k < DIM; ++k) out.g[i * DIM + k] = CELLLIM ? gr[i][k] * lim[i] : gr[i][k];
    st16(gout + c, out);
}

template <typename R, int DIM, int GRAD, int CELLLIM>
__global__ void __launch_bounds__(256, PSST_BUDGET(R, PSST_GRAD_MINB, 1)) k_gradient(DevGrid g, DevState<R> st, DevWork<R> wk) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nint) return;
    if (g.cell_case && !g.case_active[g.cell_case[c]]) return;  // stopped case
    gradient_cell<R, DIM, GRAD, CELLLIM, false>(g, st.rec, reinterpret_cast<GradRec<R, DIM> *>(wk.grec), c);
}

// cell update
// ---------------------------------------------------------------------------

// Local time step of one cell (psstLocalTimeCalculation.cpp:90-131, 175-213),
// faces in the cell's own order. In the sequential mode, neighbours updated
// earlier in the reference's order are read from `nxt`. CG: neighbour states
// through L2 only (the persistent wavefront kernel).
template <typename R, int DIM, int LC, bool SEQ, bool CG = false>
__device__ __forceinline__ double local_time(const DevGrid &g, const CellRec<R> *cur, const CellRec<R> *nxt,
                                             const Gas &gas, double cfl, double dt_uniform, int32_t c,
                                             const Prim<R, DIM> &own) {
    if (LC == 0) return dt_uniform;
    const FaceRec<R, DIM> *frec = reinterpret_cast<const FaceRec<R, DIM> *>(g.frec);
    const int32_t b = g.csr_ptr[c], e = g.csr_ptr[c + 1];
    const uint64_t perm = g.wperm[c];
    const R gr = (R)gas.gamma * (R)gas.rm;
    const R cc = sqrt(gr * own.T);
    R den = (R)0;
    if (LC == 1) {
        R nnb = (R)0;
        int32_t myrank = 0;
        if (SEQ) myrank = g.rank[c];
        for (int32_t j = 0; j < e - b; ++j) {
            const int32_t ent = g.csr_ent[b + (int32_t)((perm >> (4 * j)) & 15)];
            const FaceRec<R, DIM> fr = ld16(frec + (ent >> 1));
            const int32_t nb = (ent & 1) ? fr.c0 : fr.c1;
            const CellRec<R> *src = (SEQ && nb < g.nint && g.rank[nb] < myrank) ? nxt : cur;
            const Prim<R, DIM> o = unpack<R, DIM>(CG ? ldcg(src + nb) : ld16(src + nb));
            const R cn = (sqrt(gr * o.T) + cc) * (R)0.5;
            R nv = (R)0;
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                const R t = (R)fr.n[k];
                nv += own.u[k] * t;
                nnb += o.u[k] * t;
            }
            nnb = (nnb + nv) * (R)0.5;
            den += (fabs(nnb) + cn) * (R)fr.S;
        }
    } else {
        R s[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) s[k] = (R)0;
        for (int32_t j = 0; j < e - b; ++j) {
            const int32_t ent = g.csr_ent[b + (int32_t)((perm >> (4 * j)) & 15)];
            const FaceRec<R, DIM> fr = ld16(frec + (ent >> 1));
            const R S = (R)fr.S;
#pragma unroll
            for (int k = 0; k < DIM; ++k) s[k] += S * fabs((R)fr.n[k]);
        }
#pragma unroll
        for (int k = 0; k < DIM; ++k) den += (fabs(own.u[k]) + cc) * s[k] * (R)0.5;
    }
    return (double)((R)cfl * (R)g.V[c] / den);
}

// Inputs of a cell's RK update: the previous-stage state (w on stage 0) and
// the volume. Loaded by rk_load before the cell stores anything, so that the
// loads issue together (stores to w/pw/dt could alias them).
template <int NV>
struct RkIn {
    double pw[NV];
    double vol;
};

template <typename R, int NV>
__device__ __forceinline__ RkIn<NV> rk_load(const DevGrid &g, const DevWork<R> &wk, int first_stage, int32_t c) {
    RkIn<NV> in;
    const double *src = first_stage ? wk.w : wk.pw;
#pragma unroll
    for (int v = 0; v < NV; ++v) in.pw[v] = src[(int64_t)v * g.nint + c];
    in.vol = g.V[c];
    return in;
}

// RK stage update of one cell given its residual (psstFiniteVolumeGrid.cpp:324-346):
// w = prev_w - dt*a*res/V in FP64, primitives, norms; returns the new record.
// w and dt are stored only when `keep` is set: inside a whole iteration only
// the last stage's values are ever read (the next iteration's first stage
// loads w; stages 2.. load the stage-start copy pw).
template <typename R, int DIM>
__device__ __forceinline__ CellRec<R> rk_update(const DevGrid &g, const DevWork<R> &wk, const Gas &gas,
                                                const RkIn<DIM + 2> &in, double dt, double alpha, int first_stage,
                                                bool keep, int32_t c, const R res[DIM + 2], double sq[DIM + 2],
                                                double mx[DIM + 2]) {
    constexpr int NV = DIM + 2;
    // FP64 (parity) path: the reference's operation order, one division per
    // component; FP32 path: one reciprocal per cell (its own rounding)
    constexpr bool EXACT = sizeof(R) == 8;
    const double vol = in.vol;
    const double step = EXACT ? 0.0 : dt * alpha / vol;
    double w[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const int64_t idx = (int64_t)v * g.nint + c;
        const double pw = in.pw[v];
        if (first_stage) wk.pw[idx] = pw;
        w[v] = EXACT ? pw - dt * alpha * (double)res[v] / vol : pw - step * (double)res[v];
        if (keep) wk.w[idx] = w[v];
        const double rv = (double)res[v];
        const double ar = fabs(rv);
        if (mx[v] < ar) mx[v] = ar;  // NaN never replaces the max, as in `if (res < |r|)` (:331)
        sq[v] += rv * rv;
        if (!(rv - rv == 0.0)) flag_error(wk.err, ERR_NONFINITE_RES, c);
    }
    const double rho = w[DIM];
    const double irho = EXACT ? 0.0 : 1.0 / rho;
    double vs = 0.0;
    R u[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const double uk = EXACT ? w[k] / rho : w[k] * irho;
        u[k] = (R)uk;
        vs += uk * uk;
    }
    const double T = EXACT ? ((w[DIM + 1] / rho) - (vs * 0.5)) / gas.cv
                           : ((w[DIM + 1] * irho) - (vs * 0.5)) * (1.0 / gas.cv);
    const double p = rho * gas.rm * T;
    if (!(rho > 0.0 && T > 0.0)) flag_error(wk.err, ERR_BAD_STATE, c);
    if (keep) wk.dt[c] = dt;
    return pack<R, DIM>((R)p, (R)T, (R)rho, u);
}

// Ghost cell after its interior neighbour's update (psstFiniteVolumeGrid.cpp:
// 351-366): dynamic condition (psstBoundaryCondition.cpp:26-37, 72-80, 108-127,
// 212-219), thermal condition (:285-288, 354-357), rho = p/(T*rm).
template <typename R, int DIM>
__device__ __forceinline__ CellRec<R> ghost_state(const DevGrid &g, const CellRec<R> &gcur, const Prim<R, DIM> &nb,
                                                  int32_t i, const Gas &gas) {
    Prim<R, DIM> s = unpack<R, DIM>(gcur);
    const int32_t z = g.g_zone[i];
    const int dyn = g.z_dyn[z], th = g.z_therm[z];
    if (dyn == 26) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) s.u[k] = nb.u[k];
        s.p = nb.p;
    } else if (dyn == 15) {
        const FaceRec<R, DIM> fr = ldg(reinterpret_cast<const FaceRec<R, DIM> *>(g.frec) + g.g_face[i]);
        R vn = (R)0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) vn += nb.u[k] * (R)fr.n[k];
#pragma unroll
        for (int k = 0; k < DIM; ++k) s.u[k] = nb.u[k] - vn * (R)fr.n[k];
        s.p = nb.p;
    } else if (dyn == 25) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) s.u[k] = nb.u[k];
    }
    if (th == 25 || th == 18) s.T = nb.T;
    return pack<R, DIM>(s.p, s.T, s.p / (s.T * (R)gas.rm), s.u);
}

// Block partials of the residual norms: part[block][v] = sum res^2,
// part[block][NV + v] = max |res|; fixed reduction pattern (reproducible).
// FMAX: the maxima are FP32 values (FP32 residuals), reduced as floats
// (exact: a max selects one of its inputs).
template <int NV, bool FMAX = false>
__device__ __forceinline__ void block_norm_partials(double sq[NV], double mx[NV], double *part) {
    __shared__ double red[2 * NV][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double x = sq[v], m = mx[v];
        float mf = (float)m;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_down_sync(FULL, x, o);
            if (FMAX)
                mf = fmaxf(mf, __shfl_down_sync(FULL, mf, o));
            else
                m = fmax(m, __shfl_down_sync(FULL, m, o));
        }
        if (FMAX) m = (double)mf;
        if (lane == 0) {
            red[v][wid] = x;
            red[NV + v][wid] = m;
        }
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0, m = 0.0;
        const int nw = (blockDim.x + 31) >> 5;
        for (int i = 0; i < nw; ++i) {
            s += red[threadIdx.x][i];
            m = fmax(m, red[NV + threadIdx.x][i]);
        }
        part[(int64_t)blockIdx.x * 2 * NV + threadIdx.x] = s;
        part[(int64_t)blockIdx.x * 2 * NV + NV + threadIdx.x] = m;
    }
}

// Stage norms from the block partials (fixed-order strided sums, warp shuffle
// trees, then the warps in order: reproducible for a given block size), folded
// into the iteration's max over stages: the reference's residual column is max
// over stages and cells of |res| (psstFiniteVolumeGrid.cpp:331-332); the RMS
// column is this project's. Executed by one whole block (a multiple of 32
// threads).
template <int NV>
__device__ __forceinline__ void finish_norms(const double *part, int nblocks, int32_t nint, double *linf, double *l2,
                                             int it_slot) {
    __shared__ double red[2 * NV][32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    double s[NV], m[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = m[v] = 0.0;
#pragma unroll 4
    for (int b = t; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            s[v] += part[(int64_t)b * 2 * NV + v];
            m[v] = fmax(m[v], part[(int64_t)b * 2 * NV + NV + v]);
        }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s[v] += __shfl_down_sync(FULL, s[v], o);
            m[v] = fmax(m[v], __shfl_down_sync(FULL, m[v], o));
        }
        if (lane == 0) {
            red[v][wid] = s[v];
            red[NV + v][wid] = m[v];
        }
    }
    __syncthreads();
    if (t < NV) {
        double a = 0.0, x = 0.0;
        const int nw = (blockDim.x + 31) >> 5;
        for (int i = 0; i < nw; ++i) {
            a += red[t][i];
            x = fmax(x, red[NV + t][i]);
        }
        const double r = sqrt(a / (double)(nint > 0 ? nint : 1));
        if (r > l2[it_slot * NV + t]) l2[it_slot * NV + t] = r;
        if (linf[it_slot * NV + t] < x) linf[it_slot * NV + t] = x;
    }
}

template <int NV>
__global__ void __launch_bounds__(256) k_norm_finish(const double *part, int nblocks, int32_t nint, double *linf,
                                                     double *l2, int it_slot) {
    finish_norms<NV>(part, nblocks, nint, linf, l2, it_slot);
}

// Per-case max |res| on merged grids: cl[case][v] holds the bits of a
// non-negative double, so an integer atomicMax is the numeric max (order-free,
// hence deterministic). Lanes of one case (the usual warp: cases are
// contiguous in device order) reduce first; cs < 0 contributes nothing. NaN
// never enters (mx skips it, as the reference's `if (res < |r|)` does).
// Called by all 32 lanes of every warp.
template <int NV>
__device__ __forceinline__ void case_max(unsigned long long *cl, int32_t cs, const double mx[NV]) {
    const int32_t c0 = __shfl_sync(FULL, cs, 0);
    if (__all_sync(FULL, cs == c0)) {
        if (c0 < 0) return;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            double m = mx[v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(FULL, m, o));
            if ((threadIdx.x & 31) == 0 && m > 0.0)
                atomicMax(cl + (int64_t)c0 * NV + v, (unsigned long long)__double_as_longlong(m));
        }
    } else if (cs >= 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v)
            if (mx[v] > 0.0) atomicMax(cl + (int64_t)cs * NV + v, (unsigned long long)__double_as_longlong(mx[v]));
    }
}

// Stop rule of merged grids (CaseStop) after one iteration; cl = that
// iteration's per-case residual columns (bits of non-negative doubles). One
// thread per case; stopped cases are left as they are.
template <int NV>
__global__ void __launch_bounds__(256) k_case_stop(CaseStop cs, const unsigned long long *cl, int32_t ncase) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncase || !cs.active[c]) return;
    const int32_t rows = ++cs.rows[c];
    double row[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) row[v] = __longlong_as_double((long long)cl[(int64_t)c * NV + v]);
    double *sc = cs.scale + (int64_t)c * NV;
    if (rows <= cs.scale_iters)
#pragma unroll
        for (int v = 0; v < NV; ++v) sc[v] = rows == 1 ? row[v] : fmax(sc[v], row[v]);
    if (rows >= cs.scale_iters) {
        bool done = true;
#pragma unroll
        for (int v = 0; v < NV; ++v) done = done && row[v] / (sc[v] > 0.0 ? sc[v] : 1.0) <= cs.drop;
        if (done) {
            cs.conv_at[c] = rows;
            cs.active[c] = 0;
        }
    }
    if (cs.active[c] && rows >= cs.cap[c]) cs.active[c] = 0;
}

// Last kernel of a run-to-stop block of `chunk` iterations (one block):
// appends the block's residual columns to the history, counts the
// iterations, and sets the while-loop condition: another block while a case
// still runs, no kernel has raised an error and fewer than max_iter
// iterations have run. The loop therefore ends after at most
// ceil(max_iter / chunk) blocks whatever the cases do.
template <int NV>
__global__ void __launch_bounds__(256) k_loop_control(CaseStop cs, int32_t ncase, const int32_t *err, LoopCtl *ctl,
                                                      const double *linf, const double *l2, int32_t chunk,
                                                      cudaGraphConditionalHandle h) {
    int any = 0;
    for (int32_t c = threadIdx.x; c < ncase; c += blockDim.x) any |= cs.active[c] != 0;
    any = __syncthreads_or(any);
    const int64_t done = ctl->done, cap = ctl->cap_rows;
    for (int64_t i = threadIdx.x; i < (int64_t)chunk * NV; i += blockDim.x) {
        if (done + i / NV >= cap) break;
        ctl->hist_linf[done * NV + i] = linf[i];
        ctl->hist_l2[done * NV + i] = l2[i];
    }
    __syncthreads();  // every thread has read ctl->done
    if (threadIdx.x == 0) {
        const int64_t now = done + chunk;
        ctl->done = now;
        cudaGraphSetConditional(h, any && err[0] == 0 && now < ctl->max_iter ? 1u : 0u);
    }
}

// Block partials of the residual norms without a block barrier: each warp
// reduces its lanes (shuffle trees) into a shared slot, and the last warp of
// the block to arrive sums the slots in warp order and writes out[2 NV] (sum
// res^2, max |res|); the other warps leave at once. `count` must be zero at
// the block's start. FMAX: the maxima are FP32 values, reduced as floats.
template <int NV, bool FMAX = false>
__device__ __forceinline__ void lastwarp_partials(double sq[NV], double mx[NV], double *out, unsigned *count) {
    __shared__ double red[2 * NV][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        double x = sq[v], m = mx[v];
        float mf = (float)m;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_down_sync(FULL, x, o);
            if (FMAX)
                mf = fmaxf(mf, __shfl_down_sync(FULL, mf, o));
            else
                m = fmax(m, __shfl_down_sync(FULL, m, o));
        }
        if (FMAX) m = (double)mf;
        if (lane == 0) {
            red[v][wid] = x;
            red[NV + v][wid] = m;
        }
    }
    unsigned last = 0;
    if (lane == 0) {
        __threadfence_block();
        last = atomicAdd(count, 1u) == (unsigned)(nw - 1);
    }
    if (!__shfl_sync(FULL, last, 0)) return;
    __threadfence_block();
    if (lane < 2 * NV) {
        const volatile double *r = red[lane];
        double a = 0.0;
        for (int i = 0; i < nw; ++i) a = lane < NV ? a + r[i] : fmax(a, r[i]);
        out[lane] = a;
    }
}

// Residual columns of one iteration from the cell pass's block partials of
// its nstage stages (part[stage][nblk][2 NV]): per stage the RMS over the
// interior cells and the max |res|, then the max over stages (the reference's
// column is max over stages and cells, psstFiniteVolumeGrid.cpp:331-332; the
// RMS column is this project's). Block (g, stage) takes a fixed range of that
// stage's partials; with 64 NV threads, thread t always reads component
// t % (2 NV) (consecutive threads read consecutive doubles), and the 32
// threads of a component are folded in thread order into mid[g][stage][2 NV].
// The last block to finish folds, per (stage, component), eight fixed
// sub-ranges of the blocks in parallel and then the eight in order
// (reproducible for a given nblk and grid).
template <int NV>
__global__ void __launch_bounds__(64 * NV) k_norm_reduce(const double *part, int nblk, int nstage, int32_t nint,
                                                         double *mid, unsigned *ticket, double *linf, double *l2,
                                                         int it_slot) {
    constexpr int W = 2 * NV, T = 32 * W, kSplit = 8, kMaxStage = 16;
    __shared__ double red[T];
    __shared__ double fin8[kMaxStage * W * kSplit];
    __shared__ bool is_last;
    const int t = threadIdx.x, comp = t % W, st = (int)blockIdx.y, G = (int)gridDim.x;
    const int chunk = (nblk + G - 1) / G;
    const int b0 = (int)blockIdx.x * chunk, b1 = min(nblk, b0 + chunk);
    const double *p = part + (int64_t)st * nblk * W;
    double a = 0.0;  // sums of res^2 and maxima of |res| are both >= 0
#pragma unroll 4
    for (int64_t e = (int64_t)b0 * W + t; e < (int64_t)b1 * W; e += T) a = comp < NV ? a + p[e] : fmax(a, p[e]);
    red[t] = a;
    __syncthreads();
    if (t < W) {
        double v = 0.0;
        for (int j = 0; j < 32; ++j) v = t < NV ? v + red[t + W * j] : fmax(v, red[t + W * j]);
        mid[((int64_t)blockIdx.x * nstage + st) * W + t] = v;
        __threadfence();
    }
    __syncthreads();
    if (t == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x * gridDim.y - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    const int npair = nstage * W, per = (G + kSplit - 1) / kSplit;
    for (int q = t; q < npair * kSplit; q += T) {
        const int pair = q / kSplit, j = q % kSplit, c = pair % W;
        const int g0 = j * per, g1 = min(G, g0 + per);
        double v = 0.0;
#pragma unroll 8
        for (int g = g0; g < g1; ++g) {
            const double x = mid[(int64_t)g * npair + pair];  // mid[g][stage][comp]
            v = c < NV ? v + x : fmax(v, x);
        }
        fin8[q] = v;
    }
    __syncthreads();
    if (t < npair) {
        double v = 0.0;
        for (int j = 0; j < kSplit; ++j) v = t % W < NV ? v + fin8[t * kSplit + j] : fmax(v, fin8[t * kSplit + j]);
        red[t] = v;  // npair <= 16 W <= T
    }
    __syncthreads();
    if (t < NV) {
        double rms = 0.0, mx = 0.0;
        for (int k = 0; k < nstage; ++k) {
            const double r = sqrt(red[k * W + t] / (double)(nint > 0 ? nint : 1));
            if (r > rms) rms = r;
            mx = fmax(mx, red[k * W + NV + t]);
        }
        l2[it_slot * NV + t] = rms;
        linf[it_slot * NV + t] = mx;
    }
    if (t == 0) *ticket = 0u;
}


template <typename R, int DIM>
__device__ __forceinline__ void gather_residual(const DevGrid &g, const FaceOut<R, DIM> *fo, int32_t c,
                                                R res[DIM + 2]) {
#pragma unroll
    for (int v = 0; v < DIM + 2; ++v) res[v] = (R)0;
    for (int32_t q = g.csr_ptr[c]; q < g.csr_ptr[c + 1]; ++q) {
        const int32_t ent = g.csr_ent[q];
        const FaceOut<R, DIM> o = ldg(fo + (ent >> 1));
        if (ent & 1) {
#pragma unroll
            for (int v = 0; v < DIM + 2; ++v) res[v] += o.v[v];
        } else {
#pragma unroll
            for (int v = 0; v < DIM + 2; ++v) res[v] -= o.v[v];
        }
    }
}

// Cell pass of one RK stage (parallel modes), thread per interior cell:
// residual = in-order sum of the face outputs (psstFiniteVolumeGrid.cpp:311 and
// the scatter at psstConvectiveFlow.cpp:289-299), local time step from the
// faces' terms in the cell's own face order (the reference's accumulation
// order, psstLocalTimeCalculation.cpp:117-127, 189-203), RK update, the cell's
// ghost cells, and the block's norm partials for this stage (formed by the
// block's last warp to finish, so no warp waits at a block barrier;
// k_norm_reduce turns the stages' partials into the iteration's columns).
// At least 4 blocks of 256 per SM (64 registers): the pass is bound by the
// latency of its gathers, and the occupancy gained outweighs a 24-byte spill
// (0.61 -> 0.56 ms per launch on 6M tets, FP32).
// LocalAccTime1 face terms seen from one side: returns the cell's own u . n
// and adds the neighbour's u . n onto the running value nnb, component by
// component where the record keeps components (the reference's order,
// psstLocalTimeCalculation.cpp:117-124).
template <typename R, int DIM>
__device__ __forceinline__ R lc1_normal_velocities(const FaceOut<R, DIM> &o, int side, R &nnb) {
    using FO = FaceOut<R, DIM>;
    if (FO::NQ == DIM) {
        R nv = (R)0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) {
            nv += side ? o.v[FO::Q1 + k] : o.v[FO::Q0 + k];
            nnb += side ? o.v[FO::Q0 + k] : o.v[FO::Q1 + k];
        }
        return nv;
    }
    nnb += side ? o.v[FO::Q0] : o.v[FO::Q1];
    return side ? o.v[FO::Q1] : o.v[FO::Q0];
}

template <typename R, int DIM, int LC, bool BATCH>
__global__ void __launch_bounds__(256, PSST_BUDGET(R, PSST_CELL_MINB, 2)) k_cell(DevGrid g, DevState<R> cur, DevState<R> nxt, DevWork<R> wk, Gas gas,
                                              double cfl, double dt_uniform, double alpha, int stage,
                                              int kstage, int it_slot) {
    // stage: bit 0 first stage of the iteration, bit 1 last stage; kstage: its index
    using FO = FaceOut<R, DIM>;
    const int first_stage = stage & 1;
    constexpr int NV = DIM + 2;
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    __shared__ unsigned warps_done;  // lastwarp_partials
    if (threadIdx.x == 0) warps_done = 0u;
    __syncthreads();
    double sq[NV], mx[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) sq[v] = mx[v] = 0.0;
    bool run = c < g.nint;
    if (BATCH && run && !g.case_active[g.cell_case[c]]) {  // stopped case: carry the state over
        run = false;
        st16(nxt.rec + c, ldg(cur.rec + c));
        for (int32_t i = g.gptr[c]; i < g.gptr[c + 1]; ++i) st16(nxt.rec + g.nint + i, ldg(cur.rec + g.nint + i));
    }
    if (run) {
        const FO *fo = reinterpret_cast<const FO *>(wk.fout);
        const R *csr_s = reinterpret_cast<const R *>(g.csr_s);
        const RkIn<NV> rin = rk_load<R, NV>(g, wk, first_stage, c);
        const int32_t b = g.kuni ? c * g.kuni : g.csr_ptr[c], K = g.kuni ? g.kuni : g.csr_ptr[c + 1] - b;
        const uint64_t perm = g.wperm[c];
        // When the cell's own face order is the face-loop order (the usual
        // case: faces are wired zone by zone in file order, and files list
        // zones in ascending id), residual and time step share one pass.
        const bool one_pass = LC != 0 && perm == (0xFEDCBA9876543210ull & ((K >= 16) ? ~0ull : ((1ull << (4 * K)) - 1)));
        R res[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) res[v] = (R)0;
        R den = (R)0, nnb = (R)0, s[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) s[k] = (R)0;
        // one CSR entry (face output o of entry ent, face area sa), in face-loop order
        auto entry = [&](int32_t ent, const FO &o, R sa) {
            const int side = ent & 1;
            if (side) {
#pragma unroll
                for (int v = 0; v < NV; ++v) res[v] += o.v[v];
            } else {
#pragma unroll
                for (int v = 0; v < NV; ++v) res[v] -= o.v[v];
            }
            if (one_pass) {
                if (LC == 1) {
                    const R nv = lc1_normal_velocities<R, DIM>(o, side, nnb);
                    nnb = (nnb + nv) * (R)0.5;
                    den += (fabs(nnb) + o.v[FO::CN]) * sa;
                } else if (LC == 2) {
#pragma unroll
                    for (int k = 0; k < DIM; ++k) s[k] += o.v[FO::Q0 + k];
                }
            }
        };
        if (g.kuni == 4) {  // all-tet meshes: the four entries (b = 4c) as one 16-byte load each
            const int4 e4 = *reinterpret_cast<const int4 *>(g.csr_ent + b);
            R sa[4];
            if constexpr (sizeof(R) == 4) {
                const float4 t = *reinterpret_cast<const float4 *>(csr_s + b);
                sa[0] = (R)t.x, sa[1] = (R)t.y, sa[2] = (R)t.z, sa[3] = (R)t.w;
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) sa[q] = csr_s[b + q];
            }
            const FO o0 = ldg(fo + (e4.x >> 1)), o1 = ldg(fo + (e4.y >> 1)), o2 = ldg(fo + (e4.z >> 1)),
                     o3 = ldg(fo + (e4.w >> 1));
            entry(e4.x, o0, sa[0]);
            entry(e4.y, o1, sa[1]);
            entry(e4.z, o2, sa[2]);
            entry(e4.w, o3, sa[3]);
        } else {
#pragma unroll 4
            for (int32_t q = 0; q < K; ++q) {
                const int32_t ent = g.csr_ent[b + q];
                entry(ent, ldg(fo + (ent >> 1)), csr_s[b + q]);
            }
        }
        double dt = dt_uniform;
        if (LC != 0) {
            if (LC == 1 && !one_pass) {  // the cell's own face order differs: second pass
                for (int32_t j = 0; j < K; ++j) {
                    const int32_t slot = b + (int32_t)((perm >> (4 * j)) & 15);
                    const int32_t ent = g.csr_ent[slot];
                    const FO o = ldg(fo + (ent >> 1));
                    const int side = ent & 1;
                    const R nv = lc1_normal_velocities<R, DIM>(o, side, nnb);
                    nnb = (nnb + nv) * (R)0.5;
                    den += (fabs(nnb) + o.v[FO::CN]) * csr_s[slot];
                }
            } else if (LC == 2) {
                if (!one_pass)
                    for (int32_t j = 0; j < K; ++j) {
                        const int32_t ent = g.csr_ent[b + (int32_t)((perm >> (4 * j)) & 15)];
                        const FO o = ldg(fo + (ent >> 1));
#pragma unroll
                        for (int k = 0; k < DIM; ++k) s[k] += o.v[FO::Q0 + k];
                    }
                const Prim<R, DIM> own = unpack<R, DIM>(ldg(cur.rec + c));
                const R cc = sqrt((R)gas.gamma * (R)gas.rm * own.T);
#pragma unroll
                for (int k = 0; k < DIM; ++k) den += (fabs(own.u[k]) + cc) * s[k] * (R)0.5;
            }
            dt = (double)((R)cfl * (R)g.V[c] / den);
        }
        const CellRec<R> nrec = rk_update<R, DIM>(g, wk, gas, rin, dt, alpha, first_stage, (stage & 2) != 0, c, res,
                                                  sq, mx);
        st16(nxt.rec + c, nrec);
        const int32_t g0 = g.gptr[c], g1 = g.gptr[c + 1];
        if (g1 > g0) {
            const Prim<R, DIM> np = unpack<R, DIM>(nrec);
            for (int32_t i = g0; i < g1; ++i) {
                const int32_t gc = g.nint + i;
                st16(nxt.rec + gc, ghost_state<R, DIM>(g, ldg(cur.rec + gc), np, i, gas));
            }
        }
    }
    if (BATCH) case_max<NV>(wk.case_linf + (int64_t)it_slot * g.ncase * NV, run ? g.cell_case[c] : -1, mx);
    lastwarp_partials<NV, sizeof(R) == 4>(sq, mx, wk.l2part + ((int64_t)kstage * gridDim.x + blockIdx.x) * 2 * NV,
                                          &warps_done);
}

// Thread-per-cell update reading the face outputs (GATHER) or the residual of
// the stage-by-stage API; local time step from states (sequential mode: the
// reference's in-loop order); ghosts by k_ghost_update.
template <typename R, int DIM, int LC, bool GATHER>
__device__ __forceinline__ void update_from_buffers(const DevGrid &g, const DevState<R> &cur, const DevState<R> &nxt,
                                                    const DevWork<R> &wk, const Gas &gas, double cfl,
                                                    double dt_uniform, double alpha, int first_stage, int32_t c,
                                                    double sq[DIM + 2], double mx[DIM + 2], bool seq) {
    constexpr int NV = DIM + 2;
    const RkIn<NV> rin = rk_load<R, NV>(g, wk, first_stage, c);
    R res[NV];
    if (GATHER) {
        gather_residual<R, DIM>(g, reinterpret_cast<const FaceOut<R, DIM> *>(wk.fout), c, res);
    } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) res[v] = wk.res[(int64_t)v * g.nint + c];
    }
    const Prim<R, DIM> own = unpack<R, DIM>(ldg(cur.rec + c));
    double dt;
    if (seq)
        dt = local_time<R, DIM, 1, true>(g, cur.rec, nxt.rec, gas, cfl, dt_uniform, c, own);
    else
        dt = local_time<R, DIM, LC, false>(g, cur.rec, nxt.rec, gas, cfl, dt_uniform, c, own);
    st16(nxt.rec + c, rk_update<R, DIM>(g, wk, gas, rin, dt, alpha, first_stage, true, c, res, sq, mx));
}

template <typename R, int DIM, int LC, bool GATHER>
__global__ void __launch_bounds__(256) k_cell_update(DevGrid g, DevState<R> cur, DevState<R> nxt, DevWork<R> wk, Gas gas,
                                                     double cfl, double dt_uniform, double alpha, int first_stage) {
    constexpr int NV = DIM + 2;
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    double sq[NV], mx[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) sq[v] = mx[v] = 0.0;
    if (c < g.nint)
        update_from_buffers<R, DIM, LC, GATHER>(g, cur, nxt, wk, gas, cfl, dt_uniform, alpha, first_stage, c, sq, mx,
                                                false);
    block_norm_partials<NV>(sq, mx, wk.l2part);
}

// Sequential LocalAccTime1 (the reference's in-loop evaluation order,
// psstFiniteVolumeGrid.cpp:317-323): cells grouped into levels so that every
// cell's earlier-ranked neighbours sit in lower levels; one block walks the
// levels with a barrier between them, and each cell reads earlier-ranked
// neighbours from the next buffer and the others from the current one.
template <typename R, int DIM, bool GATHER>
__global__ void __launch_bounds__(1024) k_cell_update_seq(DevGrid g, DevState<R> cur, DevState<R> nxt, DevWork<R> wk,
                                                          Gas gas, double cfl, double alpha, int first_stage) {
    constexpr int NV = DIM + 2;
    double sq[NV], mx[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) sq[v] = mx[v] = 0.0;
    for (int32_t l = 0; l < g.nlevels; ++l) {
        const int32_t b = g.lvl_ptr[l], e = g.lvl_ptr[l + 1];
        for (int32_t i = b + threadIdx.x; i < e; i += blockDim.x)
            update_from_buffers<R, DIM, 1, GATHER>(g, cur, nxt, wk, gas, cfl, 0.0, alpha, first_stage, g.lvl_cells[i],
                                                   sq, mx, true);
        __threadfence_block();
        __syncthreads();
    }
    block_norm_partials<NV>(sq, mx, wk.l2part);
}

// Ghost cells after the interior update (face-pass path of the sequential
// mode and of the stage-by-stage API).
template <typename R, int DIM>
__global__ void __launch_bounds__(256) k_ghost_update(DevGrid g, DevState<R> cur, DevState<R> nxt, Gas gas) {
    const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.nghost) return;
    const int32_t c = g.nint + i;
    const Prim<R, DIM> nb = unpack<R, DIM>(ld16(nxt.rec + g.g_nb[i]));
    st16(nxt.rec + c, ghost_state<R, DIM>(g, ld16(cur.rec + c), nb, i, gas));
}

// residual gather into wk.res (stage-by-stage API)
template <typename R, int DIM>
__global__ void __launch_bounds__(256) k_residual(DevGrid g, DevWork<R> wk) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nint) return;
    R res[DIM + 2];
    gather_residual<R, DIM>(g, reinterpret_cast<const FaceOut<R, DIM> *>(wk.fout), c, res);
#pragma unroll
    for (int v = 0; v < DIM + 2; ++v) wk.res[(int64_t)v * g.nint + c] = res[v];
}

// Device cell records from / to the reference's volume-ordered SoA state
// (p, T, u0.. per volume), so that host buffers move in one contiguous copy.
template <typename R, int DIM>
__global__ void k_gather_prim(int32_t nall, DevState<R> st, const double *prim, const int32_t *vol, int64_t nvol) {
    const int32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nall) return;
    const int64_t v = vol[d];
    R u[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) u[k] = (R)prim[(2 + k) * nvol + v];
    CellRec<R> r = pack<R, DIM>((R)prim[v], (R)prim[nvol + v], (R)0, u);
    st16(st.rec + d, r);
}

// Exact state from a checkpoint: records (p, T, rho, u..) of every volume and
// the FP64 conservative state w of interior cells, as stored (no prologue:
// rho and w are not recomputed, so a resumed run continues bit for bit).
template <typename R, int DIM>
__global__ void k_set_exact(int32_t nall, int32_t nint, DevState<R> st, double *wdev, const double *prim,
                            const double *rho, const double *w, const int32_t *vol, int64_t nvol) {
    const int32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nall) return;
    const int64_t v = vol[d];
    R u[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) u[k] = (R)prim[(2 + k) * nvol + v];
    st16(st.rec + d, pack<R, DIM>((R)prim[v], (R)prim[nvol + v], (R)rho[v], u));
    if (d < nint)
#pragma unroll
        for (int q = 0; q < DIM + 2; ++q) wdev[(int64_t)q * nint + d] = w[v * (DIM + 2) + q];
}

template <typename R, int DIM>
__global__ void k_scatter_prim(int32_t nall, DevState<R> st, double *prim, const int32_t *vol, int64_t nvol) {
    const int32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nall) return;
    const int64_t v = vol[d];
    const CellRec<R> r = ld16(st.rec + d);
    prim[v] = (double)r.v[RP];
    prim[nvol + v] = (double)r.v[RT];
#pragma unroll
    for (int k = 0; k < DIM; ++k) prim[(2 + k) * nvol + v] = (double)r.v[RU + k];
}

template <typename R>
__global__ void k_scatter_w(int32_t nint, int nv, const double *w, double *out, const int32_t *vol) {
    const int32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if (d >= nint) return;
    const int64_t v = vol[d];
    for (int q = 0; q < nv; ++q) out[v * nv + q] = w[(int64_t)q * nint + d];
}

// explicit_solve prologue (psstFiniteVolumeGrid.cpp:279-300): rho = p/(rm*T)
// for every volume (initialize_field and load_boundary form it so), and w for
// interior cells.
template <typename R, int DIM>
__global__ void k_prologue(DevGrid g, DevState<R> st, DevWork<R> wk, Gas gas) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= g.nall) return;
    CellRec<R> r = st.rec[c];
    const double p = (double)r.v[RP], T = (double)r.v[RT];
    const double rho = p / (gas.rm * T);
    r.v[RRHO] = (R)rho;
    st.rec[c] = r;
    if (c >= g.nint) return;
    double vs = 0.0;
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        const double t = (double)r.v[RU + k];
        wk.w[(int64_t)k * g.nint + c] = rho * t;
        vs += t * t;
    }
    const double E = gas.cv * T + 0.5 * vs;
    wk.w[(int64_t)DIM * g.nint + c] = rho;
    wk.w[(int64_t)(DIM + 1) * g.nint + c] = rho * E;
}

}  // namespace psst
