// Coordinate MLP of the learned warm start: BF16 operands on the 5th-generation
// tensor cores (tcgen05.mma, FP32 accumulators in tensor memory), FP32 master
// weights and Adam state, everything else in plain CUDA.
//
// Network (width W = 256, 6 linear layers):
//   f  = Fourier features of the 4 inputs (Mach, ramp angle, x, y), each
//        normalised to [-1, 1]: sin / cos(2^j pi v), j < 15, plus v itself:
//        4 * 30 + 4 = 124 values, zero-padded to 128
//   h1 = silu(W1 f + b1), h_l = silu(W_l h_{l-1} + b_l) for l = 2..5
//   y  = W6 h5 + b6                                  (4 outputs: rho, u, v, p)
// Loss: mean over points and outputs of (y - target)^2.
//
// GEMM kernels: one CTA computes a 128 x NT tile of D = A . B^T, A [M x K],
// B [N x K] given by element strides (so transposed operands need no copy).
// K is walked in 64-wide chunks, four tcgen05.mma.kind::f16 (M = 128, N = NT,
// K = 16) per chunk, issued by one thread, FP32 accumulators in tensor memory.
//  * k_gemm_tma (operands 16-byte aligned with 16-byte row strides, contiguous
//    along K or along M/N): TMA tile loads (cp.async.bulk.tensor, no
//    multicast) into four shared-memory stages in the 128-byte swizzled
//    layout, each stage's mbarrier completed by the copy's byte count; the
//    issuing thread keeps up to four chunks in flight and refills the stage of
//    chunk c - 1 once the MMAs committed for it have completed. Operands
//    contiguous along M/N are loaded as such and read by the MMA in its
//    MN-major mode.
//  * k_gemm (anything else: unaligned strides, element strides on both axes,
//    split ranges that are not whole chunks): the CTA stages each chunk
//    through registers into the K-major no-swizzle layout (8-row x 16-byte
//    core matrices), two stages, transposing operands contiguous along M/N in
//    registers, 8 x 8 at a time.
// The epilogue reads the accumulator with tcgen05.ld (one row per thread, 32
// columns at a time), applies bias / SiLU / SiLU-derivative and writes each
// row segment with 16-byte stores. Split-K over gridDim.z writes FP32
// partials that a second kernel sums in a fixed order (deterministic). Every
// mbarrier wait is bounded; a wait that runs out drains the MMAs and copies in
// flight before the CTA frees its tensor memory and reports the timeout.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched through the runtime)
#include <cuda_bf16.h>
#include <cuda_runtime_api.h>

#include "host.hpp"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kTileM = 128;
constexpr int kChunkK = 64;
constexpr int kThreads = 128;
constexpr unsigned kWaitLimit = 1u << 26;  // mbarrier polls before giving up (~seconds)
constexpr int kStages = 2;                 // operand stages in shared memory

enum Epi { EPI_NONE = 0, EPI_SILU = 1, EPI_DSILU = 2 };
enum MlpErr { MLP_ERR_TIMEOUT = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, K-major, no swizzle: start address, leading
// byte offset (between the two 8-element K halves of one MMA), stride byte
// offset (between 8-row groups), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// The same for the 128-byte swizzled layouts written by TMA (tiles 1024-byte
// aligned, layout type 2): K-major, 8-row groups of 128-byte rows 1024 bytes
// apart (SBO), LBO unused (16); MN-major, groups of 8 K rows 1024 bytes apart
// (SBO) and 64-element M/N blocks `lbo` bytes apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr, uint32_t lbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: BF16 x BF16 -> FP32, M = 128; operand A (B) read
// K-major, or MN-major when AMN (BMN).
template <int NT, bool AMN = false, bool BMN = false>
__device__ __forceinline__ uint32_t umma_idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)AMN << 15) | ((uint32_t)BMN << 16) |
           ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(kTileM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Polls the mbarrier phase at most `limit` times; false if it never completed.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase, unsigned limit = kWaitLimit) {
    const uint32_t a = smem_u32(bar);
    for (unsigned i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int NT, bool AMN = false, bool BMN = false>
__device__ __forceinline__ void umma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t accumulate) {
    const uint32_t idesc = umma_idesc<NT, AMN, BMN>();
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One TMA tile load (no multicast) of the box at coordinates (x, y) of `map`;
// completes its bytes on `bar`.
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

struct GemmArgs {
    const bf16 *A;
    int64_t a_sm, a_sk;  // A[m][k] = A[m * a_sm + k * a_sk]
    const bf16 *B;
    int64_t b_sn, b_sk;  // B[n][k] = B[n * b_sn + k * b_sk]
    int M, N, K, k_split;
    const float *bias;   // [N] or null
    int epi;             // Epi
    const bf16 *Zin;     // EPI_DSILU: pre-activation [M][N] (row stride d_sm)
    float *D32;          // FP32 output [splits][M][d_sm] (or null)
    bf16 *D16;           // BF16 output [M][d_sm] (or null)
    bf16 *Z16;           // BF16 pre-activation output [M][d_sm] (EPI_SILU, or null)
    int64_t d_sm;
    int *err;
    unsigned wait_polls;  // bound of the first wait that runs out (kWaitLimit; 0 gives up at once)
    int vec;              // outputs and Zin 16-byte aligned, d_sm % 8 == 0: 16-byte epilogue stores
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

constexpr int kEpiWarpBytes = 8192;  // per warp: a 32 x 32 FP32 tile (4 KB) + two BF16 tiles (2 KB each)

// Swizzled 32-row tiles in shared memory: 16-byte chunk c of row r of an FP32
// tile (128-byte rows) at r * 128 + (c ^ (r & 7)) * 16, of a BF16 tile
// (64-byte rows) at r * 64 + (c ^ ((r >> 1) & 3)) * 16. A warp writing one
// row per lane, or reading 512 contiguous bytes, hits every bank 4 times.
__device__ __forceinline__ uint4 *tile32(unsigned char *t, int r, int c) {
    return reinterpret_cast<uint4 *>(t + r * 128 + ((c ^ (r & 7)) << 4));
}
__device__ __forceinline__ uint4 *tile16(unsigned char *t, int r, int c) {
    return reinterpret_cast<uint4 *>(t + r * 64 + ((c ^ ((r >> 1) & 3)) << 4));
}

// Writes the warp's BF16 tile (rows m0w.., columns nb..nb+31) to g (row
// stride ld): each store instruction covers 8 rows x 64 bytes.
__device__ __forceinline__ void tile16_store(unsigned char *t, bf16 *g, int64_t ld, int m0w, int M, int nb) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = 8 * i + (lane >> 2), c = lane & 3;
        if (m0w + r < M) *reinterpret_cast<uint4 *>(g + (int64_t)(m0w + r) * ld + nb + 8 * c) = *tile16(t, r, c);
    }
    __syncwarp();
}

// Epilogue: thread t holds accumulator row m0 + t (TMEM lane t) and handles it
// 32 columns at a time: bias and activation in registers; then, with a.vec and
// the whole segment inside N, each warp passes its 32 x 32 block through its
// shared-memory tiles so that global loads and stores cover whole rows (16
// bytes per lane); otherwise element by element. `tiles`: kEpiWarpBytes per
// warp of free shared memory.
template <int NT>
__device__ __forceinline__ void epilogue(const GemmArgs &a, uint32_t tmem, int m0, int n0, bool empty,
                                         unsigned char *tiles) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int m0w = m0 + 32 * warp, m = m0w + lane;
    const uint32_t lanes = (uint32_t)(32 * warp) << 16;  // this warp's 32 TMEM lanes
    unsigned char *tf = tiles + warp * kEpiWarpBytes, *th = tf + 4096, *tz = th + 2048;
    for (int c0 = 0; c0 < NT && n0 + c0 < a.N; c0 += 32) {
        float v[32];
        if (!empty)
            tmem_ld32(tmem + lanes + (uint32_t)c0, v);
        else
#pragma unroll
            for (int i = 0; i < 32; ++i) v[i] = 0.0f;
        const int nb = n0 + c0, nn = min(32, a.N - nb);
        if (a.bias)
#pragma unroll
            for (int i = 0; i < 32; ++i)
                if (i < nn) v[i] += a.bias[nb + i];
        if (a.vec && nn == 32) {  // warp-uniform
            if (a.D32) {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    *tile32(tf, lane, j) = make_uint4(__float_as_uint(v[4 * j]), __float_as_uint(v[4 * j + 1]),
                                                      __float_as_uint(v[4 * j + 2]), __float_as_uint(v[4 * j + 3]));
                __syncwarp();
                float *d32 = a.D32 + (int64_t)blockIdx.z * a.M * a.d_sm;
#pragma unroll
                for (int i = 0; i < 8; ++i) {  // 4 rows x 128 bytes per instruction
                    const int r = 4 * i + (lane >> 3), c = lane & 7;
                    if (m0w + r < a.M)
                        *reinterpret_cast<uint4 *>(d32 + (int64_t)(m0w + r) * a.d_sm + nb + 4 * c) = *tile32(tf, r, c);
                }
                __syncwarp();
            }
            if (a.epi == EPI_SILU && a.Z16) {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    *tile16(tz, lane, j) =
                        make_uint4(pack_bf16(v[8 * j], v[8 * j + 1]), pack_bf16(v[8 * j + 2], v[8 * j + 3]),
                                   pack_bf16(v[8 * j + 4], v[8 * j + 5]), pack_bf16(v[8 * j + 6], v[8 * j + 7]));
                tile16_store(tz, a.Z16, a.d_sm, m0w, a.M, nb);
            }
            if (a.D16) {
                if (a.epi == EPI_SILU) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) v[i] = silu(v[i]);
                } else if (a.epi == EPI_DSILU) {
                    // the pre-activations of the warp's rows, loaded whole rows at a time
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        const int r = 8 * i + (lane >> 2), c = lane & 3;
                        if (m0w + r < a.M)
                            *tile16(tz, r, c) =
                                *reinterpret_cast<const uint4 *>(a.Zin + (int64_t)(m0w + r) * a.d_sm + nb + 8 * c);
                    }
                    __syncwarp();
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const uint4 zq = *tile16(tz, lane, j);
                        const uint32_t zw[4] = {zq.x, zq.y, zq.z, zq.w};
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const __nv_bfloat162 z2 = *reinterpret_cast<const __nv_bfloat162 *>(&zw[q]);
                            v[8 * j + 2 * q] *= dsilu(__low2float(z2));
                            v[8 * j + 2 * q + 1] *= dsilu(__high2float(z2));
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    *tile16(th, lane, j) =
                        make_uint4(pack_bf16(v[8 * j], v[8 * j + 1]), pack_bf16(v[8 * j + 2], v[8 * j + 3]),
                                   pack_bf16(v[8 * j + 4], v[8 * j + 5]), pack_bf16(v[8 * j + 6], v[8 * j + 7]));
                tile16_store(th, a.D16, a.d_sm, m0w, a.M, nb);
            }
        } else if (m < a.M) {
            const int64_t o = (int64_t)m * a.d_sm + nb;
            float *d32 = a.D32 ? a.D32 + (int64_t)blockIdx.z * a.M * a.d_sm + o : nullptr;
#pragma unroll
            for (int i = 0; i < 32; ++i) {  // unrolled: v stays in registers
                if (i >= nn) break;
                const float z = v[i];
                if (d32) d32[i] = z;
                if (a.epi == EPI_SILU && a.Z16) a.Z16[o + i] = __float2bfloat16(z);
                if (a.D16) {
                    float h = z;
                    if (a.epi == EPI_SILU) h = silu(z);
                    else if (a.epi == EPI_DSILU) h = z * dsilu(__bfloat162float(a.Zin[o + i]));
                    a.D16[o + i] = __float2bfloat16(h);
                }
            }
        }
    }
}

// Stages rows [r0, r0+ROWS) x K columns [k0, k0+64) of a strided BF16 matrix
// (element (r, k) at g[r * sr + k * sk]) into the K-major no-swizzle layout:
// element (r, k) at ((k/8) * ROWS + r) * 16 + (k%8) * 2 bytes. Out-of-range
// elements (r >= nrows, k >= kend) are zero.
//  * contiguous along K (sk == 1): one 16-byte load per (row, 8 k);
//  * contiguous along the rows (sr == 1): one 16-byte load per (8 rows, k),
//    eight of them (8 k) transposed in registers into eight (row, 8 k) units;
//  * otherwise element by element.
template <int ROWS>
__device__ __forceinline__ void stage(bf16 *s, const bf16 *g, int64_t sr, int64_t sk, int r0, int nrows, int k0,
                                      int kend) {
    if (sk == 1 && (sr % 8) == 0 && ((uintptr_t)g & 15) == 0 && r0 + ROWS <= nrows && k0 + kChunkK <= kend) {
        // whole tile in range: every load of the thread issued before any store
        constexpr int IT = ROWS * 8 / kThreads;
        int4 v[IT];
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int i = threadIdx.x + it * kThreads;
            v[it] = *reinterpret_cast<const int4 *>(g + (int64_t)(r0 + i / 8) * sr + k0 + (i % 8) * 8);
        }
#pragma unroll
        for (int it = 0; it < IT; ++it) {
            const int i = threadIdx.x + it * kThreads;
            *reinterpret_cast<int4 *>(s + ((size_t)(i % 8) * ROWS + i / 8) * 8) = v[it];
        }
    } else if (sk == 1 && (sr % 8) == 0 && ((uintptr_t)g & 15) == 0) {
        for (int i = threadIdx.x; i < ROWS * 8; i += kThreads) {
            const int r = i / 8, kc = i % 8;  // eight lanes read one row's 128 bytes
            const int k = k0 + kc * 8;
            int4 v = make_int4(0, 0, 0, 0);
            if (r0 + r < nrows && k < kend) {
                if (k + 8 <= kend) {
                    v = *reinterpret_cast<const int4 *>(g + (int64_t)(r0 + r) * sr + k);
                } else {
                    bf16 t[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        t[j] = k + j < kend ? g[(int64_t)(r0 + r) * sr + k + j] : __float2bfloat16(0.0f);
                    memcpy(&v, t, 16);
                }
            }
            *reinterpret_cast<int4 *>(s + ((size_t)kc * ROWS + r) * 8) = v;
        }
    } else if (sr == 1 && (sk % 8) == 0 && ((uintptr_t)g & 15) == 0) {
        for (int i = threadIdx.x; i < ROWS; i += kThreads) {  // (8-row block, 8-k group) per i
            const int rb = (i % (ROWS / 8)) * 8, kc = i / (ROWS / 8);
            uint32_t v[8][4];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int k = k0 + kc * 8 + j;
                int4 t = make_int4(0, 0, 0, 0);
                if (k < kend) {
                    const bf16 *src = g + (int64_t)k * sk + r0 + rb;
                    if (r0 + rb + 8 <= nrows) {
                        t = *reinterpret_cast<const int4 *>(src);
                    } else {
                        bf16 e[8];
#pragma unroll
                        for (int q = 0; q < 8; ++q) e[q] = r0 + rb + q < nrows ? src[q] : __float2bfloat16(0.0f);
                        memcpy(&t, e, 16);
                    }
                }
                v[j][0] = (uint32_t)t.x, v[j][1] = (uint32_t)t.y, v[j][2] = (uint32_t)t.z, v[j][3] = (uint32_t)t.w;
            }
            // v[j] holds rows rb..rb+7 of column j (two rows per word); row r of
            // the unit takes the half r%2 of word r/2 from columns 2q, 2q+1
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const uint32_t sel = (r & 1) ? 0x7632u : 0x5410u;
                int4 o;
                o.x = (int)__byte_perm(v[0][r >> 1], v[1][r >> 1], sel);
                o.y = (int)__byte_perm(v[2][r >> 1], v[3][r >> 1], sel);
                o.z = (int)__byte_perm(v[4][r >> 1], v[5][r >> 1], sel);
                o.w = (int)__byte_perm(v[6][r >> 1], v[7][r >> 1], sel);
                *reinterpret_cast<int4 *>(s + ((size_t)kc * ROWS + rb + r) * 8) = o;
            }
        }
    } else {
        for (int i = threadIdx.x; i < ROWS * kChunkK; i += kThreads) {
            const int r = i % ROWS, kk = i / ROWS;
            const int k = k0 + kk;
            bf16 v = __float2bfloat16(0.0f);
            if (r0 + r < nrows && k < kend) v = g[(int64_t)(r0 + r) * sr + (int64_t)k * sk];
            s[((size_t)(kk / 8) * ROWS + r) * 8 + (kk % 8)] = v;
        }
    }
}

template <int NT>
__global__ void __launch_bounds__(kThreads, 2) k_gemm(GemmArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    constexpr int kStageBytes = (kTileM + NT) * kChunkK * 2;
    __shared__ __align__(8) uint64_t bar[kStages];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * NT;
    const int kb = blockIdx.z * a.k_split, ke = min(a.K, kb + a.k_split);
    const int warp = threadIdx.x >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(NT < 32 ? 32 : NT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int b = 0; b < kStages; ++b) mbar_init(&bar[b], 1);
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    unsigned phase = 0u;  // bit b: the phase of stage b's mbarrier to wait for
    unsigned polls = a.wait_polls;  // the first wait that runs out uses this bound, the drain kWaitLimit
    // thread 0: waits (bounded) for the MMAs committed to stage b; on a wait
    // that runs out it marks the launch failed and waits (bounded again) for
    // the latest commit, stage `newest`, which covers every MMA issued, so no
    // MMA is in flight when the accumulator is freed
    auto wait_stage = [&](int b, int newest) {
        if (threadIdx.x == 0 && !failed) {
            if (polls == 0 || !mbar_wait(&bar[b], (phase >> b) & 1u, polls)) {
                failed = 1;
                mbar_wait(&bar[newest], (phase >> newest) & 1u);
            }
        }
        phase ^= 1u << b;
    };
    const int nchunks = ke > kb ? (ke - kb + kChunkK - 1) / kChunkK : 0;
    for (int c = 0; c < nchunks; ++c) {
        const int b = c % kStages;
        if (c >= kStages) wait_stage(b, (c - 1) % kStages);  // the MMAs of chunk c - 2 read this stage
        __syncthreads();
        if (failed) break;
        bf16 *sA = reinterpret_cast<bf16 *>(smem + b * kStageBytes);
        bf16 *sB = reinterpret_cast<bf16 *>(smem + b * kStageBytes + kTileM * kChunkK * 2);
        const int k0 = kb + c * kChunkK;
        stage<kTileM>(sA, a.A, a.a_sm, a.a_sk, m0, a.M, k0, ke);
        stage<NT>(sB, a.B, a.b_sn, a.b_sk, n0, a.N, k0, ke);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t abase = smem_u32(sA), bbase = smem_u32(sB);
#pragma unroll
            for (int q = 0; q < kChunkK / 16; ++q) {
                const uint64_t da = umma_desc(abase + 2 * q * kTileM * 16, kTileM * 16, 128);
                const uint64_t db = umma_desc(bbase + 2 * q * NT * 16, NT * 16, 128);
                umma_bf16<NT>(tmem, da, db, (c > 0 || q > 0) ? 1u : 0u);
            }
            umma_commit(&bar[b]);
        }
    }
    // the last commit covers every MMA issued before it
    if (nchunks > 0 && !failed) wait_stage((nchunks - 1) % kStages, (nchunks - 1) % kStages);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (failed) {
        if (threadIdx.x == 0) atomicExch(a.err, MLP_ERR_TIMEOUT);
    } else {
        epilogue<NT>(a, tmem, m0, n0, nchunks == 0, smem);  // the operand stages are free now
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NT < 32 ? 32 : NT));
}

constexpr int kTmaStages = 4;  // chunks in flight: K = 256 (the network's widths) loads in one go

// TMA-fed variant. Stage s holds the A tile then the B tile of one 64-wide K
// chunk in the 128-byte swizzled layout: K-major operands as one box of
// (64 k) x rows, rows 128 bytes apart; MN-major operands as boxes of
// (64 rows) x (64 k), one per 64 rows, K rows 128 bytes apart. Thread 0
// issues the copies and the MMAs: the first kTmaStages chunks are loaded at
// once; after the MMAs of chunk c are issued, the stage of chunk c - 1 is
// refilled (with chunk c - 1 + kTmaStages) as soon as its MMAs have completed.
template <int NT, bool AMN, bool BMN>
__global__ void __launch_bounds__(kThreads, 1)
    k_gemm_tma(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs a) {
    constexpr uint32_t kABytes = kTileM * kChunkK * 2, kBBytes = NT * kChunkK * 2, kStage = kABytes + kBBytes;
    extern __shared__ unsigned char smem_raw[];
    // the swizzle pattern repeats every 1024 bytes: tiles start on that boundary
    unsigned char *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    __shared__ __align__(8) uint64_t full[kTmaStages], empty[kTmaStages];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;
    const int m0 = blockIdx.x * kTileM, n0 = blockIdx.y * NT;
    const int kb = blockIdx.z * a.k_split, ke = min(a.K, kb + a.k_split);
    const int nchunks = ke > kb ? (ke - kb + kChunkK - 1) / kChunkK : 0;
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(NT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        for (int b = 0; b < kTmaStages; ++b) {
            mbar_init(&full[b], 1);
            mbar_init(&empty[b], 1);
        }
        failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;
    if (threadIdx.x == 0) {
        const unsigned polls = a.wait_polls;  // 0: the first wait gives up at once
        int issued = 0, consumed = 0, committed = 0;
        auto load = [&](int c) {
            const int b = c % kTmaStages, k0 = kb + c * kChunkK;
            unsigned char *sa = smem + b * kStage, *sb = sa + kABytes;
            mbar_expect_tx(&full[b], kStage);  // out-of-range box elements arrive as zeros and count
            if (AMN) {
#pragma unroll
                for (int j = 0; j < kTileM / 64; ++j) tma_load(sa + j * 8192, &ta, m0 + 64 * j, k0, &full[b]);
            } else {
                tma_load(sa, &ta, k0, m0, &full[b]);
            }
            if (BMN) {
#pragma unroll
                for (int j = 0; j < NT / 64; ++j) tma_load(sb + j * 8192, &tb, n0 + 64 * j, k0, &full[b]);
            } else {
                tma_load(sb, &tb, k0, n0, &full[b]);
            }
            ++issued;
        };
        // use: how many earlier chunks went through this stage (the phase parity to wait for)
        auto wait = [&](uint64_t *bar, int use) { return polls != 0 && mbar_wait(bar, (unsigned)use & 1u, polls); };
        bool ok = true;
        for (int c = 0; c < min(kTmaStages, nchunks); ++c) load(c);
        for (int c = 0; c < nchunks; ++c) {
            const int b = c % kTmaStages;
            if (!(ok = wait(&full[b], c / kTmaStages))) break;
            ++consumed;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_u32(smem + b * kStage), sb = sa + kABytes;
#pragma unroll
            for (int q = 0; q < kChunkK / 16; ++q) {  // K = 16 per MMA: 32 bytes along a row, or 16 K rows
                const uint64_t da = AMN ? umma_desc_sw128(sa + q * 2048, 8192) : umma_desc_sw128(sa + q * 32, 16);
                const uint64_t db = BMN ? umma_desc_sw128(sb + q * 2048, 8192) : umma_desc_sw128(sb + q * 32, 16);
                umma_bf16<NT, AMN, BMN>(tmem, da, db, (c > 0 || q > 0) ? 1u : 0u);
            }
            umma_commit(&empty[b]);
            ++committed;
            const int next = c - 1 + kTmaStages;
            if (c >= 1 && next < nchunks) {
                if (!(ok = wait(&empty[(c - 1) % kTmaStages], (c - 1) / kTmaStages))) break;
                load(next);
            }
        }
        // the last commit covers every MMA issued before it
        if (ok && committed > 0) ok = wait(&empty[(committed - 1) % kTmaStages], (committed - 1) / kTmaStages);
        if (!ok) {
            // a wait ran out: let the MMAs and the copies in flight finish (bounded) before the
            // accumulator and the stages are given up
            failed = 1;
            if (committed > 0)
                mbar_wait(&empty[(committed - 1) % kTmaStages], (unsigned)((committed - 1) / kTmaStages) & 1u);
            for (int c = consumed; c < issued; ++c) mbar_wait(&full[c % kTmaStages], (unsigned)(c / kTmaStages) & 1u);
        }
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (failed) {
        if (threadIdx.x == 0) atomicExch(a.err, MLP_ERR_TIMEOUT);
    } else {
        epilogue<NT>(a, tmem, m0, n0, nchunks == 0, smem);  // the stages are free now
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NT));
}

// out[i] = sum over z of part[z][i] (fixed order), optional BF16 copy.
__global__ void k_sum_splits(const float *part, int splits, int64_t n, float *out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(int64_t)z * n + i];
    out[i] = s;
}

}  // namespace

namespace {

constexpr int kWidth = 256;
constexpr int kFeat = 128;       // Fourier features, padded
constexpr int kFreq = 15;
constexpr int kIn = 4, kOut = 4;
constexpr int kHidden = 5;       // layers with SiLU
constexpr int kSplitRows = 256;  // batch rows per split of a weight-gradient GEMM (16384 rows: 128 CTAs)

// Fourier features of x[b][4] (inputs normalised to [-1, 1]).
__global__ void k_features(const float *x, int B, bf16 *f) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    bf16 *o = f + (int64_t)b * kFeat;
    int q = 0;
    for (int i = 0; i < kIn; ++i) {
        const float v = x[(int64_t)b * kIn + i];
        o[q++] = __float2bfloat16(v);
        float w = 3.14159265358979f;
        for (int j = 0; j < kFreq; ++j, w *= 2.0f) {
            o[q++] = __float2bfloat16(sinf(w * v));
            o[q++] = __float2bfloat16(cosf(w * v));
        }
    }
    for (; q < kFeat; ++q) o[q] = __float2bfloat16(0.0f);
}

// Output layer y = W6 h5 + b6 on CUDA cores (4 outputs), and for training
// dy = 2 (y - t) / (4 B) plus per-block partial sums of (y - t)^2.
__global__ void k_output(const bf16 *h, const float *W6, const float *b6, int B, float *y, const float *t,
                         float *dy, float *loss_part) {
    __shared__ float red[8];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (b < B) {
        float acc[kOut];
        for (int o = 0; o < kOut; ++o) acc[o] = b6[o];
        const bf16 *hr = h + (int64_t)b * kWidth;
        for (int j = 0; j < kWidth; ++j) {
            const float hv = __bfloat162float(hr[j]);
            for (int o = 0; o < kOut; ++o) acc[o] += W6[o * kWidth + j] * hv;
        }
        for (int o = 0; o < kOut; ++o) {
            if (y) y[(int64_t)b * kOut + o] = acc[o];
            if (t) {
                const float d = acc[o] - t[(int64_t)b * kOut + o];
                l += d * d;
                dy[(int64_t)b * kOut + o] = 2.0f * d / (float)(kOut * B);
            }
        }
    }
    if (!loss_part) return;
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        loss_part[blockIdx.x] = s;
    }
}

// dz5 = (dy W6) * silu'(z5), BF16.
__global__ void k_output_back(const float *dy, const float *W6, const bf16 *z5, int B, bf16 *dz) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * kWidth) return;
    const int b = (int)(i / kWidth), j = (int)(i % kWidth);
    float s = 0.0f;
    for (int o = 0; o < kOut; ++o) s += dy[(int64_t)b * kOut + o] * W6[o * kWidth + j];
    dz[i] = __float2bfloat16(s * dsilu(__bfloat162float(z5[i])));
}

// Gradient of the output layer: part[chunk][o * 256 + j] = sum over the chunk's
// rows of dy[b][o] h5[b][j]; part[chunk][1024 + o] = sum of dy[b][o].
__global__ void k_output_wgrad(const float *dy, const bf16 *h, int B, int rows, float *part) {
    const int chunk = blockIdx.x, idx = blockIdx.y * blockDim.x + threadIdx.x;
    if (idx >= kOut * kWidth + kOut) return;
    const int b0 = chunk * rows, b1 = min(B, b0 + rows);
    float s = 0.0f;
    if (idx < kOut * kWidth) {
        const int o = idx / kWidth, j = idx % kWidth;
        for (int b = b0; b < b1; ++b) s += dy[(int64_t)b * kOut + o] * __bfloat162float(h[(int64_t)b * kWidth + j]);
    } else {
        const int o = idx - kOut * kWidth;
        for (int b = b0; b < b1; ++b) s += dy[(int64_t)b * kOut + o];
    }
    part[(int64_t)chunk * (kOut * kWidth + kOut) + idx] = s;
}

// Column sums of dz [B][256] over row chunks: part[chunk][j].
__global__ void k_colsum(const bf16 *dz, int B, int rows, float *part) {
    const int chunk = blockIdx.x, j = threadIdx.x;
    const int b0 = chunk * rows, b1 = min(B, b0 + rows);
    float s = 0.0f;
    for (int b = b0; b < b1; ++b) s += __bfloat162float(dz[(int64_t)b * kWidth + j]);
    part[(int64_t)chunk * kWidth + j] = s;
}

// Adam (Kingma & Ba, 2015) on the FP32 master parameters; refreshes the BF16
// copies of the tensor-core weights (entries with wmap[i] >= 0).
__global__ void k_adam(float *p, const float *g, float *m, float *v, int64_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2, const int64_t *wmap, bf16 *wbf) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    p[i] = pi;
    if (wmap[i] >= 0) wbf[wmap[i]] = __float2bfloat16(pi);
}

__global__ void k_to_bf16(const float *p, int64_t n, const int64_t *wmap, bf16 *wbf) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && wmap[i] >= 0) wbf[wmap[i]] = __float2bfloat16(p[i]);
}

}  // namespace

using namespace psst;

struct psst_mlp {
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    int64_t nparam = 0, nwbf = 0;
    int64_t offW[6] = {}, offb[6] = {}, offWbf[5] = {};
    int din[6] = {kFeat, kWidth, kWidth, kWidth, kWidth, kWidth}, dout[6] = {kWidth, kWidth, kWidth, kWidth, kWidth, kOut};
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    int64_t *wmap = nullptr;
    bf16 *wbf = nullptr;
    int64_t step = 0;
    int cap = 0;
    bf16 *F = nullptr, *Z[kHidden] = {}, *H[kHidden] = {}, *dZ[2] = {};
    float *y = nullptr, *dy = nullptr, *lpart = nullptr, *part = nullptr;
    int64_t part_n = 0;
    int *err = nullptr;
    std::vector<void *> allocs, ws;
    ~psst_mlp() {
        cudaSetDevice(device);
        for (void *q : ws) cudaFree(q);
        for (void *q : allocs) cudaFree(q);
        if (own) cudaStreamDestroy(own);
    }
};

namespace {

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) raise(PSST_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <class T>
T *dmalloc(std::vector<void *> &list, size_t n) {
    void *q = nullptr;
    ck(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    list.push_back(q);
    return (T *)q;
}

constexpr size_t kGemmSmem = 100 * 1024;  // at most two CTAs per SM, so two 256-column TMEM allocations fit
template <int NT>
constexpr size_t tma_smem() {
    return (size_t)kTmaStages * (kTileM + NT) * kChunkK * 2 + 1024;  // + the 1024-byte alignment of the tiles
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_tiled() {
    static const EncodeTiled fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    if (!fn) raise(PSST_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the CUDA driver");
    return fn;
}

// An operand (element (r, k) at g[r * sr + k * sk]) that TMA can load:
// 16-byte aligned, contiguous along K or along the rows, 16-byte row stride.
bool tma_operand(const bf16 *g, int64_t sr, int64_t sk) {
    if (((uintptr_t)g & 15) != 0) return false;
    if (sk == 1) return sr > 0 && sr % 8 == 0;
    if (sr == 1) return sk > 0 && sk % 8 == 0;
    return false;
}

// Its tensor map, boxes landing in the 128-byte swizzled layout: contiguous
// along K, box (64 k) x box_rows; contiguous along the rows, (64 rows) x (64 k).
CUtensorMap operand_map(const bf16 *g, int64_t sr, int64_t sk, int nrows, int K, int box_rows) {
    CUtensorMap map;
    const bool kmajor = sk == 1;
    const cuuint64_t dim[2] = {(cuuint64_t)(kmajor ? K : nrows), (cuuint64_t)(kmajor ? nrows : K)};
    const cuuint64_t stride[1] = {(cuuint64_t)(kmajor ? sr : sk) * 2};
    const cuuint32_t box[2] = {64, (cuuint32_t)(kmajor ? box_rows : 64)};
    const cuuint32_t estride[2] = {1, 1};
    const CUresult r = encode_tiled()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16 *>(g), dim, stride,
                                      box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) raise(PSST_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return map;
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15) == 0; }

// once per device and kernel (a per-launch call costs host time between back-to-back GEMMs)
template <class F>
void smem_attribute(F *kernel, size_t bytes, unsigned long long &done_devices) {
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 64 || !(done_devices >> dev & 1ull)) {
        ck(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), "attribute");
        if (dev < 64) done_devices |= 1ull << dev;
    }
}

template <int NT, bool AMN, bool BMN>
void launch_tma(const CUtensorMap &ta, const CUtensorMap &tb, const GemmArgs &a, dim3 grid, cudaStream_t s) {
    static thread_local unsigned long long done_devices = 0;
    smem_attribute(k_gemm_tma<NT, AMN, BMN>, tma_smem<NT>(), done_devices);
    k_gemm_tma<NT, AMN, BMN><<<grid, kThreads, tma_smem<NT>(), s>>>(ta, tb, a);
}

// One GEMM launch worked out once (kernel, grid, tensor maps), launched any
// number of times.
struct GemmPlan {
    GemmArgs a;
    dim3 grid;
    int nt = 256;
    int kind = 0;  // 0: register-staged; 1 + 2 AMN + BMN: TMA-fed
    CUtensorMap ta, tb;
};

template <int NT>
GemmPlan plan(const GemmArgs &a0, int splits) {
    GemmPlan p;
    p.a = a0;
    GemmArgs &a = p.a;
    a.vec = a.d_sm % 8 == 0 && aligned16(a.D32) && aligned16(a.D16) && aligned16(a.Z16) && aligned16(a.Zin);
    p.nt = NT;
    p.grid = dim3((a.M + kTileM - 1) / kTileM, (a.N + NT - 1) / NT, splits);
    // TMA boxes are whole 64-wide chunks: a split range must be whole chunks unless it is the only one
    if (a.K > 0 && (splits == 1 || a.k_split % kChunkK == 0) && tma_operand(a.A, a.a_sm, a.a_sk) &&
        tma_operand(a.B, a.b_sn, a.b_sk)) {
        p.ta = operand_map(a.A, a.a_sm, a.a_sk, a.M, a.K, kTileM);
        p.tb = operand_map(a.B, a.b_sn, a.b_sk, a.N, a.K, NT);
        p.kind = 1 + 2 * (a.a_sk != 1) + (a.b_sk != 1);
    }
    return p;
}

template <int NT>
void launch_nt(const GemmPlan &p, cudaStream_t s) {
    switch (p.kind) {
        case 1: launch_tma<NT, false, false>(p.ta, p.tb, p.a, p.grid, s); return;
        case 2: launch_tma<NT, false, true>(p.ta, p.tb, p.a, p.grid, s); return;
        case 3: launch_tma<NT, true, false>(p.ta, p.tb, p.a, p.grid, s); return;
        case 4: launch_tma<NT, true, true>(p.ta, p.tb, p.a, p.grid, s); return;
        default: {
            static thread_local unsigned long long done_devices = 0;
            smem_attribute(k_gemm<NT>, kGemmSmem, done_devices);
            k_gemm<NT><<<p.grid, kThreads, kGemmSmem, s>>>(p.a);
        }
    }
}

void launch(const GemmPlan &p, cudaStream_t s) {
    if (p.nt == 128)
        launch_nt<128>(p, s);
    else
        launch_nt<256>(p, s);
}

template <int NT>
void gemm(const GemmArgs &a, int splits, cudaStream_t s) {
    launch(plan<NT>(a, splits), s);
}

GemmArgs gargs(const bf16 *A, int64_t a_sm, int64_t a_sk, const bf16 *B, int64_t b_sn, int64_t b_sk, int M, int N,
               int K, int *err) {
    GemmArgs a{};
    a.A = A;
    a.a_sm = a_sm;
    a.a_sk = a_sk;
    a.B = B;
    a.b_sn = b_sn;
    a.b_sk = b_sk;
    a.M = M;
    a.N = N;
    a.K = K;
    a.k_split = K;
    a.err = err;
    a.wait_polls = kWaitLimit;
    return a;
}

unsigned nb(int64_t n, int b = 256) { return (unsigned)((n + b - 1) / b); }

void ensure_ws(psst_mlp *m, int B) {
    if (B <= m->cap) return;
    for (void *q : m->ws) cudaFree(q);
    m->ws.clear();
    const int cap = std::max(B, 2 * m->cap);
    m->F = dmalloc<bf16>(m->ws, (size_t)cap * kFeat);
    for (int l = 0; l < kHidden; ++l) {
        m->Z[l] = dmalloc<bf16>(m->ws, (size_t)cap * kWidth);
        m->H[l] = dmalloc<bf16>(m->ws, (size_t)cap * kWidth);
    }
    m->dZ[0] = dmalloc<bf16>(m->ws, (size_t)cap * kWidth);
    m->dZ[1] = dmalloc<bf16>(m->ws, (size_t)cap * kWidth);
    m->y = dmalloc<float>(m->ws, (size_t)cap * kOut);
    m->dy = dmalloc<float>(m->ws, (size_t)cap * kOut);
    m->lpart = dmalloc<float>(m->ws, nb(cap));
    const int64_t splits = (cap + kSplitRows - 1) / kSplitRows;
    m->part_n = splits * (int64_t)kWidth * kWidth;
    m->part = dmalloc<float>(m->ws, m->part_n);
    m->cap = cap;
}

void check_err(psst_mlp *m) {
    int e = 0;
    ck(cudaMemcpyAsync(&e, m->err, sizeof e, cudaMemcpyDeviceToHost, m->stream), "error word");
    ck(cudaStreamSynchronize(m->stream), "stream sync");
    if (e) {
        ck(cudaMemsetAsync(m->err, 0, sizeof(int), m->stream), "memset");
        raise(PSST_ERR_TIMEOUT, "tensor-core GEMM: an mbarrier wait ran out");
    }
}

// Forward pass; with t != null also the loss terms (returns the loss).
float forward(psst_mlp *m, const float *x, int B, const float *t, float *yout) {
    cudaStream_t s = m->stream;
    k_features<<<nb(B), 256, 0, s>>>(x, B, m->F);
    const bf16 *in = m->F;
    int64_t ld = kFeat;
    for (int l = 0; l < kHidden; ++l) {
        GemmArgs a = gargs(in, ld, 1, m->wbf + m->offWbf[l], ld, 1, B, kWidth, (int)ld, m->err);
        a.bias = m->p + m->offb[l];
        a.epi = EPI_SILU;
        a.Z16 = m->Z[l];
        a.D16 = m->H[l];
        a.d_sm = kWidth;
        gemm<256>(a, 1, s);
        in = m->H[l];
        ld = kWidth;
    }
    k_output<<<nb(B), 256, 0, s>>>(m->H[kHidden - 1], m->p + m->offW[5], m->p + m->offb[5], B, yout ? yout : m->y, t,
                                   m->dy, t ? m->lpart : nullptr);
    ck(cudaGetLastError(), "forward");
    if (!t) return 0.0f;
    std::vector<float> lp(nb(B));
    ck(cudaMemcpyAsync(lp.data(), m->lpart, lp.size() * sizeof(float), cudaMemcpyDeviceToHost, s), "loss copy");
    check_err(m);
    double sum = 0.0;
    for (float v : lp) sum += v;
    return (float)(sum / ((double)kOut * B));
}

// Gradients of the loss of the last forward pass into m->g.
void backward(psst_mlp *m, int B) {
    cudaStream_t s = m->stream;
    const int splits = (B + kSplitRows - 1) / kSplitRows;
    // output layer (CUDA cores)
    k_output_back<<<nb((int64_t)B * kWidth), 256, 0, s>>>(m->dy, m->p + m->offW[5], m->Z[kHidden - 1], B, m->dZ[0]);
    const int nout = kOut * kWidth + kOut;
    k_output_wgrad<<<dim3(splits, nb(nout)), 256, 0, s>>>(m->dy, m->H[kHidden - 1], B, kSplitRows, m->part);
    k_sum_splits<<<nb(nout), 256, 0, s>>>(m->part, splits, nout, m->g + m->offW[5]);
    int cur = 0;
    for (int l = kHidden - 1; l >= 0; --l) {
        const bf16 *prev = l == 0 ? m->F : m->H[l - 1];
        const int din = m->din[l];
        // dW_l = dZ_l^T . H_{l-1}: split over batch rows, fixed-order sum
        GemmArgs a = gargs(m->dZ[cur], 1, kWidth, prev, 1, din, kWidth, din, B, m->err);
        a.k_split = kSplitRows;
        a.D32 = m->part;
        a.d_sm = din;
        if (din == 256)
            gemm<256>(a, splits, s);
        else
            gemm<128>(a, splits, s);
        k_sum_splits<<<nb((int64_t)kWidth * din), 256, 0, s>>>(m->part, splits, (int64_t)kWidth * din,
                                                               m->g + m->offW[l]);
        k_colsum<<<splits, kWidth, 0, s>>>(m->dZ[cur], B, kSplitRows, m->part);
        k_sum_splits<<<1, kWidth, 0, s>>>(m->part, splits, kWidth, m->g + m->offb[l]);
        if (l > 0) {  // dZ_{l-1} = (dZ_l . W_l) * silu'(Z_{l-1})
            GemmArgs d = gargs(m->dZ[cur], kWidth, 1, m->wbf + m->offWbf[l], 1, din, B, kWidth, kWidth, m->err);
            d.epi = EPI_DSILU;
            d.Zin = m->Z[l - 1];
            d.D16 = m->dZ[cur ^ 1];
            d.d_sm = kWidth;
            gemm<256>(d, 1, s);
            cur ^= 1;
        }
    }
    ck(cudaGetLastError(), "backward");
}

}  // namespace

#define MLP_BEGIN try {
#define MLP_END                                \
    return PSST_OK;                            \
    }                                          \
    catch (const Error &e) {                   \
        set_last_error(e.msg);                 \
        return e.status;                       \
    }                                          \
    catch (const std::bad_alloc &) {           \
        set_last_error("out of host memory");  \
        return PSST_ERR_ARG;                   \
    }

extern "C" psst_status psst_mlp_create(int device, uint64_t seed, psst_mlp **out) {
    MLP_BEGIN
    if (!out) raise(PSST_ERR_ARG, "psst_mlp_create: null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) raise(PSST_ERR_CUDA, "no CUDA device available");
    if (device < 0 || device >= ndev) raise(PSST_ERR_ARG, "invalid device index");
    std::unique_ptr<psst_mlp> m(new psst_mlp);
    m->device = device;
    ck(cudaSetDevice(device), "cudaSetDevice");
    ck(cudaStreamCreateWithFlags(&m->own, cudaStreamNonBlocking), "stream");
    m->stream = m->own;
    int64_t off = 0, wo = 0;
    for (int l = 0; l < 6; ++l) {
        m->offW[l] = off;
        off += (int64_t)m->dout[l] * m->din[l];
        m->offb[l] = off;
        off += m->dout[l];
        if (l < kHidden) {
            m->offWbf[l] = wo;
            wo += (int64_t)m->dout[l] * m->din[l];
        }
    }
    m->nparam = off;
    m->nwbf = wo;
    // PyTorch's default Linear initialisation: U(-1/sqrt(in), 1/sqrt(in)) for weights and biases
    std::vector<float> h(off);
    std::vector<int64_t> map(off, -1);
    uint64_t st = seed * 0x9E3779B97F4A7C15ull + 0x2545F4914F6CDD1Dull;
    auto uni = [&]() {  // splitmix64 -> [0, 1)
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    for (int l = 0; l < 6; ++l) {
        const double bound = 1.0 / std::sqrt((double)(l == 0 ? 4 * (2 * kFreq + 1) : m->din[l]));
        for (int64_t i = m->offW[l]; i < m->offb[l] + m->dout[l]; ++i) h[i] = (float)((2.0 * uni() - 1.0) * bound);
        if (l < kHidden)
            for (int64_t i = 0; i < (int64_t)m->dout[l] * m->din[l]; ++i) map[m->offW[l] + i] = m->offWbf[l] + i;
    }
    m->p = dmalloc<float>(m->allocs, off);
    m->g = dmalloc<float>(m->allocs, off);
    m->m1 = dmalloc<float>(m->allocs, off);
    m->m2 = dmalloc<float>(m->allocs, off);
    m->wmap = dmalloc<int64_t>(m->allocs, off);
    m->wbf = dmalloc<bf16>(m->allocs, wo);
    m->err = dmalloc<int>(m->allocs, 1);
    ck(cudaMemcpy(m->p, h.data(), off * sizeof(float), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemcpy(m->wmap, map.data(), off * sizeof(int64_t), cudaMemcpyHostToDevice), "upload");
    ck(cudaMemset(m->m1, 0, off * sizeof(float)), "memset");
    ck(cudaMemset(m->m2, 0, off * sizeof(float)), "memset");
    ck(cudaMemset(m->g, 0, off * sizeof(float)), "memset");
    ck(cudaMemset(m->err, 0, sizeof(int)), "memset");
    k_to_bf16<<<nb(off), 256, 0, m->stream>>>(m->p, off, m->wmap, m->wbf);
    ck(cudaStreamSynchronize(m->stream), "init");
    *out = m.release();
    MLP_END
}

extern "C" int64_t psst_mlp_param_count(const psst_mlp *m) { return m ? m->nparam : -1; }

extern "C" psst_status psst_mlp_get_params(psst_mlp *m, float *out, int64_t n) {
    MLP_BEGIN
    if (!m || !out || n != m->nparam) raise(PSST_ERR_ARG, "psst_mlp_get_params: bad argument");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    ck(cudaMemcpyAsync(out, m->p, n * sizeof(float), cudaMemcpyDeviceToHost, m->stream), "copy");
    ck(cudaStreamSynchronize(m->stream), "sync");
    MLP_END
}

extern "C" psst_status psst_mlp_set_params(psst_mlp *m, const float *in, int64_t n) {
    MLP_BEGIN
    if (!m || !in || n != m->nparam) raise(PSST_ERR_ARG, "psst_mlp_set_params: bad argument");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    ck(cudaMemcpyAsync(m->p, in, n * sizeof(float), cudaMemcpyHostToDevice, m->stream), "copy");
    k_to_bf16<<<nb(n), 256, 0, m->stream>>>(m->p, n, m->wmap, m->wbf);
    ck(cudaStreamSynchronize(m->stream), "sync");
    m->step = 0;
    ck(cudaMemset(m->m1, 0, n * sizeof(float)), "memset");
    ck(cudaMemset(m->m2, 0, n * sizeof(float)), "memset");
    MLP_END
}

extern "C" psst_status psst_mlp_forward(psst_mlp *m, const float *x, int B, float *y) {
    MLP_BEGIN
    if (!m || !x || !y || B <= 0) raise(PSST_ERR_ARG, "psst_mlp_forward: bad argument");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    ensure_ws(m, B);
    forward(m, x, B, nullptr, y);
    check_err(m);
    MLP_END
}

extern "C" psst_status psst_mlp_gradients(psst_mlp *m, const float *x, const float *t, int B, float *grads,
                                          float *loss) {
    MLP_BEGIN
    if (!m || !x || !t || B <= 0) raise(PSST_ERR_ARG, "psst_mlp_gradients: bad argument");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    ensure_ws(m, B);
    const float l = forward(m, x, B, t, nullptr);
    backward(m, B);
    if (grads) ck(cudaMemcpyAsync(grads, m->g, m->nparam * sizeof(float), cudaMemcpyDeviceToHost, m->stream), "copy");
    check_err(m);
    if (loss) *loss = l;
    MLP_END
}

extern "C" psst_status psst_mlp_train_step(psst_mlp *m, const float *x, const float *t, int B, float lr,
                                           float *loss) {
    MLP_BEGIN
    if (!m || !x || !t || B <= 0) raise(PSST_ERR_ARG, "psst_mlp_train_step: bad argument");
    ck(cudaSetDevice(m->device), "cudaSetDevice");
    ensure_ws(m, B);
    const float l = forward(m, x, B, t, nullptr);
    backward(m, B);
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = (float)(1.0 - std::pow((double)b1, (double)m->step));
    const float c2 = (float)(1.0 - std::pow((double)b2, (double)m->step));
    k_adam<<<nb(m->nparam), 256, 0, m->stream>>>(m->p, m->g, m->m1, m->m2, m->nparam, lr, b1, b2, 1e-8f, c1, c2,
                                                  m->wmap, m->wbf);
    ck(cudaGetLastError(), "adam");
    check_err(m);
    if (loss) *loss = l;
    MLP_END
}

extern "C" psst_status psst_mlp_set_stream(psst_mlp *m, void *stream) {
    MLP_BEGIN
    if (!m) raise(PSST_ERR_ARG, "null network");
    m->stream = stream ? (cudaStream_t)stream : m->own;
    MLP_END
}

extern "C" void psst_mlp_destroy(psst_mlp *m) { delete m; }

namespace {

// ms != null (timing): *ms receives the mean device time of one launch over
// reps launches replayed back to back.
void tc_gemm(const void *A, int64_t a_sm, int64_t a_sk, const void *B, int64_t b_sn, int64_t b_sk, int M, int N,
             int K, int k_split, float *D, int64_t d_sm, void *stream, unsigned wait_polls, int reps = 1,
             double *ms = nullptr) {
    if (!A || !B || !D || M <= 0 || N <= 0 || K < 0 || k_split <= 0 || d_sm < N)
        raise(PSST_ERR_ARG, "psst_tc_gemm_bf16: bad argument");
    static thread_local int *err = nullptr;
    static thread_local int err_dev = -1;
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    if (!err || err_dev != dev) {
        ck(cudaMalloc(&err, sizeof(int)), "cudaMalloc");
        ck(cudaMemset(err, 0, sizeof(int)), "memset");
        err_dev = dev;
    }
    cudaStream_t s = (cudaStream_t)stream;
    GemmArgs a = gargs((const bf16 *)A, a_sm, a_sk, (const bf16 *)B, b_sn, b_sk, M, N, K, err);
    a.k_split = k_split;
    a.D32 = D;
    a.d_sm = d_sm;
    a.wait_polls = wait_polls;
    const int splits = K == 0 ? 1 : (K + k_split - 1) / k_split;
    const GemmPlan p = N <= 128 ? plan<128>(a, splits) : plan<256>(a, splits);
    if (!ms) {
        launch(p, s);
        ck(cudaGetLastError(), "gemm launch");
    } else {
        // timing: the reps launches captured once as a CUDA graph on a private
        // stream (ordered after the caller's stream) and replayed between two
        // events, so the figure is device time with no host time between launches
        launch(p, s);  // first launch of this kernel (module load, attributes) outside the graph
        ck(cudaGetLastError(), "gemm launch");
        cudaStream_t ts = nullptr;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        auto release = [&] {
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            if (ts) cudaStreamDestroy(ts);
        };
        try {
            ck(cudaStreamCreateWithFlags(&ts, cudaStreamNonBlocking), "stream");
            ck(cudaEventCreate(&e0), "event");
            ck(cudaEventCreate(&e1), "event");
            ck(cudaEventRecord(e0, s), "event");
            ck(cudaStreamWaitEvent(ts, e0, 0), "stream wait");
            ck(cudaStreamBeginCapture(ts, cudaStreamCaptureModeThreadLocal), "capture");
            for (int r = 0; r < reps; ++r) launch(p, ts);
            ck(cudaStreamEndCapture(ts, &graph), "capture");
            ck(cudaGraphInstantiate(&exec, graph, 0), "graph");
            ck(cudaGraphLaunch(exec, ts), "graph");  // warm replay
            ck(cudaEventRecord(e0, ts), "event");
            ck(cudaGraphLaunch(exec, ts), "graph");
            ck(cudaEventRecord(e1, ts), "event");
            ck(cudaEventSynchronize(e1), "event");
            float t = 0.0f;
            ck(cudaEventElapsedTime(&t, e0, e1), "event");
            *ms = t / reps;
            ck(cudaEventRecord(e1, ts), "event");
            ck(cudaStreamWaitEvent(s, e1, 0), "stream wait");
        } catch (...) {
            release();
            throw;
        }
        release();
    }
    int e = 0;
    ck(cudaMemcpyAsync(&e, err, sizeof e, cudaMemcpyDeviceToHost, s), "error word");
    ck(cudaStreamSynchronize(s), "stream sync");
    if (e) {
        cudaMemset(err, 0, sizeof(int));
        raise(PSST_ERR_TIMEOUT, "tensor-core GEMM: an mbarrier wait ran out");
    }
}

}  // namespace

// D[z][m][n] = sum over k in split z of A[m][k] B[n][k] (BF16 in, FP32 out).
extern "C" psst_status psst_tc_gemm_bf16(const void *A, int64_t a_sm, int64_t a_sk, const void *B, int64_t b_sn,
                                         int64_t b_sk, int M, int N, int K, int k_split, float *D, int64_t d_sm,
                                         void *stream) {
    MLP_BEGIN
    tc_gemm(A, a_sm, a_sk, B, b_sn, b_sk, M, N, K, k_split, D, d_sm, stream, kWaitLimit);
    MLP_END
}

// Device time of one launch, the mean over reps back-to-back launches.
extern "C" psst_status psst_tc_gemm_bf16_time(const void *A, int64_t a_sm, int64_t a_sk, const void *B,
                                              int64_t b_sn, int64_t b_sk, int M, int N, int K, int k_split,
                                              float *D, int64_t d_sm, void *stream, int reps, double *ms) {
    MLP_BEGIN
    if (reps <= 0 || !ms) raise(PSST_ERR_ARG, "psst_tc_gemm_bf16_time: reps > 0 and ms needed");
    tc_gemm(A, a_sm, a_sk, B, b_sn, b_sk, M, N, K, k_split, D, d_sm, stream, kWaitLimit, reps, ms);
    MLP_END
}

// The same with the bound of the first mbarrier wait given (in polls).
extern "C" psst_status psst_tc_gemm_bf16_wait(const void *A, int64_t a_sm, int64_t a_sk, const void *B,
                                              int64_t b_sn, int64_t b_sk, int M, int N, int K, int k_split,
                                              float *D, int64_t d_sm, void *stream, int64_t wait_polls) {
    MLP_BEGIN
    tc_gemm(A, a_sm, a_sk, B, b_sn, b_sk, M, N, K, k_split, D, d_sm, stream,
            wait_polls < 0 || wait_polls > (int64_t)kWaitLimit ? kWaitLimit : (unsigned)wait_polls);
    MLP_END
}
