// psst_convective_residual_static: the first-order convective residual of
// caller-owned device arrays, computed without allocating any memory.
//
// Who needs it: callers that cannot call cudaMalloc -- code that runs inside a
// framework owning every device allocation (a memory pool or arena handed out
// by the host application), embedded solvers that must not grow their device
// footprint after start-up, or hosts that forbid allocation on a hot path.
// They own their inputs and outputs; the only extra memory this entry point
// needs is the per-face flux buffer, and that lives in a fixed array compiled
// into the library (g_face_flux below), so no call allocates.
//
// The computation is the face pass + per-cell gather of the solver's
// psst_convective_calculate for first-order reconstruction
// (psstFirstOrderReconstructor, psstValueReconstructor.cpp:28-48, with the
// HLL/HLLC/AUSM fluxes of psstConvectiveFlow.cpp), in FP64, using the same
// device functions, so the residuals are identical to the solver's.
//
// Compiled with -fmad=false like the FP64 solver kernels.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime_api.h>

#include "host.hpp"
#include "kernels.cuh"

namespace psst {
namespace {

// Flux * area per face for up to PSST_STATIC_MAX_FACES faces ([component][face],
// 5 components), followed by the error word. Every GPU that loads the library
// holds this array until the process exits (PSST_STATIC_MAX_FACES * 5 * 8 bytes
// + 16 = 5.24 MB). All calls share it, and it keeps the last call's contents.
constexpr int64_t kMaxFaces = PSST_STATIC_MAX_FACES;
static __device__ __align__(256) double g_face_flux[5 * kMaxFaces + 2];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_ptr[kMaxDevices] = {nullptr};

// Device address of g_face_flux on the current device. The host-side name
// g_face_flux is only a stand-in for the symbol, so the address is looked up
// once per device (with that device current) and cached.
double *scratch_on_current_device() {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        raise(PSST_ERR_CUDA, "psst_convective_residual_static: no current CUDA device");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_face_flux);
        if (e != cudaSuccess)
            raise(PSST_ERR_CUDA, std::string("cudaGetSymbolAddress of the static flux buffer failed: ") +
                                     cudaGetErrorString(e));
        g_ptr[dev] = (double *)p;
    }
    return g_ptr[dev];
}

template <int DIM>
__device__ __forceinline__ Prim<double, DIM> soa_prim(const double *prim, int32_t nall, int32_t c) {
    Prim<double, DIM> s;
    s.p = prim[c];
    s.T = prim[(int64_t)nall + c];
    s.rho = prim[2 * (int64_t)nall + c];
#pragma unroll
    for (int k = 0; k < DIM; ++k) s.u[k] = prim[(int64_t)(3 + k) * nall + c];
    return s;
}

template <int DIM, int FLUX>
__global__ void __launch_bounds__(256) k_static_face(int32_t nint, int32_t nall, int32_t nface, const int32_t *c0,
                                                     const int32_t *c1, const double *S, const double *n,
                                                     const double *prim, Gas gas, double *fs) {
    const int32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nface) return;
    const int32_t a = c0[f], b = c1[f];
    double nn[DIM];
#pragma unroll
    for (int k = 0; k < DIM; ++k) nn[k] = n[(int64_t)k * nface + f];
    double flow[DIM + 2];
    if (a >= nint || b >= nint) {  // boundary face: physical flux of the ghost state
        boundary_flux<double, DIM>(soa_prim<DIM>(prim, nall, a >= nint ? a : b), nn, gas, flow);
    } else {
        Prim<double, DIM> r[2] = {soa_prim<DIM>(prim, nall, a), soa_prim<DIM>(prim, nall, b)};
        FaceRec<double, DIM> unused{};
        GradRec<double, DIM> g0, g1;
        if (!interior_flux<double, DIM, FLUX, 0, 1>(r, &g0, &g1, unused, nn, gas, flow)) {
            int32_t *err = reinterpret_cast<int32_t *>(fs + 5 * kMaxFaces);
            flag_error(err, FLUX == 2 ? ERR_HLL : ERR_HLLC, f);
#pragma unroll
            for (int j = 0; j < DIM + 2; ++j) flow[j] = 0.0;
        }
    }
#pragma unroll
    for (int j = 0; j < DIM + 2; ++j) fs[(int64_t)j * kMaxFaces + f] = flow[j] * S[f];
}

template <int DIM>
__global__ void __launch_bounds__(256) k_static_gather(int32_t nint, const int32_t *csr_ptr, const int32_t *csr_ent,
                                                       const double *fs, double *res) {
    const int32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nint) return;
    constexpr int NV = DIM + 2;
    double r[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) r[v] = 0.0;
    for (int32_t q = csr_ptr[c]; q < csr_ptr[c + 1]; ++q) {
        const int32_t ent = csr_ent[q];
        const int32_t f = ent >> 1;
        if (ent & 1) {
#pragma unroll
            for (int v = 0; v < NV; ++v) r[v] += fs[(int64_t)v * kMaxFaces + f];
        } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) r[v] -= fs[(int64_t)v * kMaxFaces + f];
        }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) res[(int64_t)v * nint + c] = r[v];
}

template <int DIM>
void launch(int flux, int32_t nint, int32_t nall, int32_t nface, const int32_t *c0, const int32_t *c1,
            const double *S, const double *n, const int32_t *csr_ptr, const int32_t *csr_ent, const double *prim,
            const Gas &gas, double *fs, double *res, cudaStream_t s) {
    const int fb = (nface + 255) / 256, cb = (nint + 255) / 256;
    if (nface > 0) {
        if (flux == 1)
            k_static_face<DIM, 1><<<fb, 256, 0, s>>>(nint, nall, nface, c0, c1, S, n, prim, gas, fs);
        else if (flux == 2)
            k_static_face<DIM, 2><<<fb, 256, 0, s>>>(nint, nall, nface, c0, c1, S, n, prim, gas, fs);
        else
            k_static_face<DIM, 3><<<fb, 256, 0, s>>>(nint, nall, nface, c0, c1, S, n, prim, gas, fs);
    }
    if (nint > 0) k_static_gather<DIM><<<cb, 256, 0, s>>>(nint, csr_ptr, csr_ent, fs, res);
}

}  // namespace
}  // namespace psst

using namespace psst;

extern "C" psst_status psst_convective_residual_static(int32_t dim, int32_t flux, int32_t nint, int32_t nall,
                                                       int32_t nface, const int32_t *face_c0,
                                                       const int32_t *face_c1, const double *face_S,
                                                       const double *face_n, const int32_t *csr_ptr,
                                                       const int32_t *csr_ent, const double *prim, double rm,
                                                       double cp, double cv, double gamma, double *residual,
                                                       void *stream) {
    try {
        if (dim != 2 && dim != 3) raise(PSST_ERR_ARG, "psst_convective_residual_static: dim must be 2 or 3");
        if (flux < 1 || flux > 3) raise(PSST_ERR_ARG, "Error: Unknow convective flow scheme!");
        if (nint < 0 || nall < nint || nface < 0) raise(PSST_ERR_ARG, "psst_convective_residual_static: bad sizes");
        if (nface > PSST_STATIC_MAX_FACES)
            raise(PSST_ERR_ARG, "psst_convective_residual_static: " + std::to_string(nface) +
                                    " faces exceed the static flux buffer (PSST_STATIC_MAX_FACES = " +
                                    std::to_string((long long)PSST_STATIC_MAX_FACES) + ")");
        if ((nface && (!face_c0 || !face_c1 || !face_S || !face_n)) || (nint && (!csr_ptr || !csr_ent || !residual)) ||
            (nall && !prim))
            raise(PSST_ERR_ARG, "psst_convective_residual_static: null array");
        cudaStream_t s = (cudaStream_t)stream;
        double *fs = scratch_on_current_device();
        // the error word must start at zero; the flux entries are all rewritten
        cudaError_t e = cudaMemsetAsync(fs + 5 * kMaxFaces, 0, 2 * sizeof(double), s);
        if (e != cudaSuccess) raise(PSST_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
        const Gas gas{rm, cp, cv, gamma};
        if (dim == 2)
            launch<2>(flux, nint, nall, nface, face_c0, face_c1, face_S, face_n, csr_ptr, csr_ent, prim, gas, fs,
                      residual, s);
        else
            launch<3>(flux, nint, nall, nface, face_c0, face_c1, face_S, face_n, csr_ptr, csr_ent, prim, gas, fs,
                      residual, s);
        e = cudaGetLastError();
        if (e != cudaSuccess) raise(PSST_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
        int32_t err[2] = {0, 0};
        e = cudaMemcpyAsync(err, fs + 5 * kMaxFaces, sizeof err, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) raise(PSST_ERR_CUDA, std::string("stream: ") + cudaGetErrorString(e));
        if (err[0] == ERR_HLL) raise(PSST_ERR_FLUX, "Error: Could not calculate convective HLL flow!");
        if (err[0] == ERR_HLLC) raise(PSST_ERR_FLUX, "Error: Could not calculate convective HLLC flow!");
        return PSST_OK;
    } catch (const Error &e) {
        set_last_error(e.msg);
        return e.status;
    }
}
