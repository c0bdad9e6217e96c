// MLP column emulator: hand-written BF16 training and inference kernels on tcgen05.
//
// Stands in for the column parameterizations large-scale condensation and convection
// of the primitive-equation wet model (SpeedyWeather/src/parameterizations/
// large_scale_condensation.jl:55-178, convection.jl:33-253), called per column through
// the parameterization interface parameterization!(ij, vars, p, model)
// (SpeedyWeather/src/parameterizations/tendencies.jl:3-90). The plain parameterizations
// (column_physics.cu) label the training columns, evaluate the emulator, and replace it
// for columns outside the range of its training inputs.
//
// Network: 33 inputs (T, q, u, v on 8 layers and log surface pressure, normalised)
// -> 256 -> 256 -> 256 (GELU) -> 16 outputs (dT/dt and dq/dt on 8 layers, normalised).
// Weights in BF16 (FP32 master copies and Adam moments for training), FP32 accumulate.
//
// Training and sht_mlp_infer: every matrix product is one launch of a tcgen05 GEMM,
// C[M x N] = A[M x K] B[K x N], A and B row-major BF16 in global memory, each either
// K-major (K contiguous) or MN-major (M or N contiguous), loaded by 2-D TMA boxes of
// 64 x 64 with 128-byte swizzle into a ring of shared-memory stages; one elected thread
// issues tcgen05.mma kind::f16 (M = 128, N <= 256) into a TMEM accumulator; eight warps
// read it (tcgen05.ld), transpose 32 x 32 blocks through shared memory for coalesced
// stores and apply a fused epilogue:
//   forward hidden layer   Z = A W^T + b, A' = bf16(GELU(Z)) (Z kept for the backward)
//   forward output layer   Y = A W^T + b
//   backward data          dZ = bf16((dZ' W) * GELU'(Z))
//   backward weights       dW = dZ^T A (FP32; the batch split over the grid, partial
//                          products reduced in a fixed order)
// The emulator as a parameterization (sht_column_emulate) is one fused kernel instead:
// gather, the four layers with the activations kept in shared memory, output and plain
// physics fallback (mlp_fused_kernel below).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <vector>

#include "column_physics.cuh"
#include "sht_internal.h"
#include "tc_ptx.cuh"

namespace sht {
int set_error(int code, const char* msg);
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();
}  // namespace sht

using namespace sht;
using namespace sht::tcx;

namespace {

constexpr int G_THREADS = 320;                 // producer warp, MMA warp, 8 epilogue warps
constexpr int G_BOX = 64;                       // TMA box edge (elements) = K block
constexpr int G_BOX_BYTES = G_BOX * G_BOX * 2;  // 8 KB
constexpr int G_STAGES = 3;

enum Epi { EPI_F32 = 0, EPI_BIAS_F32 = 1, EPI_BIAS_GELU = 2, EPI_GELU_BWD = 3 };

struct GemmArgs {
    int M, N, K;
    int a_mn, b_mn;                 // operand major-ness: 1 = M (N) contiguous, 0 = K contiguous
    int epi;
    float* out_f32;                 // EPI_F32 / EPI_BIAS_F32 output, or EPI_BIAS_GELU pre-activation copy
    int64_t ld_f32;
    __nv_bfloat16* out_bf16;        // EPI_BIAS_GELU / EPI_GELU_BWD output
    int64_t ld_bf16;
    const float* bias;              // [N]
    const float* zin;               // EPI_GELU_BWD: pre-activation [M][ld_z]
    int64_t ld_z;
    int32_t* err;
    int kb_per_split;               // K blocks of 64 per CTA along grid z (split K; EPI_F32 only)
    int64_t split_stride;           // elements between the partial products of consecutive splits
};
constexpr int G_EPI_LD = 33;        // epilogue transpose tile [32 rows][33]
constexpr int G_EPI_BYTES = 8 * 32 * G_EPI_LD * 4;

// GELU in its tanh form (Hendrycks & Gimpel 2016): gelu(x) = x (1 + tanh(u)) / 2,
// u = sqrt(2 / pi) (x + 0.044715 x^3), with tanh on the special-function unit
// (tanh.approx.f32: one instruction, relative error about 2^-11, saturating to +-1; the
// activations are rounded to BF16, 2^-9, right after).
constexpr float GELU_C = 0.7978845608028654f;    // sqrt(2 / pi)
constexpr float GELU_A = 0.044715f;
__device__ __forceinline__ float tanh_sfu(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float gelu_tanh(float x) { return tanh_sfu(GELU_C * x * fmaf(GELU_A * x, x, 1.f)); }
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + gelu_tanh(x)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float t = gelu_tanh(x);
    const float du = GELU_C * fmaf(3.f * GELU_A * x, x, 1.f);
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * du;
}

// One 128 x nt output tile per CTA (nt a multiple of 16, <= 256; tile y covers columns
// [nt y, nt y + nt)) over the K blocks [z kb_per_split, (z + 1) kb_per_split) of grid
// slice z. The epilogue transposes each 32 x 32 block of the accumulator through shared
// memory (the stage buffers, free once the accumulator is complete) so that a warp's
// stores cover consecutive columns of one row (coalesced), then applies the fused
// operation to 32 independent rows at a time.
__global__ void __launch_bounds__(G_THREADS, 2)
    bf16_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     const GemmArgs g, int nt, uint32_t tmem_cols) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int m0 = blockIdx.x * 128, n0 = blockIdx.y * nt;
    const int kb0 = blockIdx.z * g.kb_per_split;
    const int nbox_b = (nt + G_BOX - 1) / G_BOX;
    const int a_bytes = 2 * G_BOX_BYTES;
    const int stage_bytes = a_bytes + nbox_b * G_BOX_BYTES;
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + (size_t)G_STAGES * stage_bytes);
    uint64_t* empty_bar = full_bar + G_STAGES;
    uint64_t* acc_bar = empty_bar + G_STAGES;      // accumulator complete: the epilogue may start
    uint64_t* mma_bar = acc_bar + 1;               // every issued MMA complete (also after an abort)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    float* epi_tile = reinterpret_cast<float*>(smem);
    const int nk = min((g.K + G_BOX - 1) / G_BOX - kb0, g.kb_per_split);   // >= 1 by construction

    if (threadIdx.x == 0) {
        for (int s = 0; s < G_STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(acc_bar, 1);
        mbar_init(mma_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---- producer: A tile (128 x 64 K) and B tile (nt x 64 K) per K block
        int issued = 0;
        for (int kb = 0; kb < nk && !*abort_flag; ++kb, ++issued) {
            const int s = kb % G_STAGES;
            if (kb >= G_STAGES && !mbar_wait(&empty_bar[s], ((kb / G_STAGES) - 1) & 1)) {
                *abort_flag = 1;
                atomicExch(g.err, 11);
                break;
            }
            uint8_t* st = smem + (size_t)s * stage_bytes;
            mbar_expect_tx(&full_bar[s], (uint32_t)stage_bytes);
            const int kx = (kb0 + kb) * G_BOX;
            for (int h = 0; h < 2; ++h) {   // A: rows (K-major) or columns (MN-major) m0 + 64 h
                if (g.a_mn)
                    tma_load_2d(st + h * G_BOX_BYTES, &map_a, m0 + h * G_BOX, kx, &full_bar[s]);
                else
                    tma_load_2d(st + h * G_BOX_BYTES, &map_a, kx, m0 + h * G_BOX, &full_bar[s]);
            }
            for (int h = 0; h < nbox_b; ++h) {
                if (g.b_mn)
                    tma_load_2d(st + a_bytes + h * G_BOX_BYTES, &map_b, n0 + h * G_BOX, kx, &full_bar[s]);
                else
                    tma_load_2d(st + a_bytes + h * G_BOX_BYTES, &map_b, kx, n0 + h * G_BOX, &full_bar[s]);
            }
        }
        // no copy may still land after the CTA exits
        for (int u = issued - 1; u >= 0 && u >= issued - G_STAGES; --u)
            if (!mbar_wait(&full_bar[u % G_STAGES], (u / G_STAGES) & 1)) atomicExch(g.err, 12);
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer
        const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)g.a_mn << 15) |
                               ((uint32_t)g.b_mn << 16) | (((uint32_t)nt >> 3) << 17) | ((128u >> 4) << 24);
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % G_STAGES;
            if (!mbar_wait(&full_bar[s], (kb / G_STAGES) & 1)) {
                *abort_flag = 1;
                atomicExch(g.err, 13);
                break;
            }
            tc_fence_after();
            const uint32_t st = smem_u32(smem + (size_t)s * stage_bytes);
            for (int kk = 0; kk < G_BOX / 16; ++kk) {
                const uint64_t da = g.a_mn ? sdesc(st + kk * 2048, G_BOX_BYTES, 1024) : sdesc(st + kk * 32, 16, 1024);
                const uint64_t db = g.b_mn ? sdesc(st + a_bytes + kk * 2048, G_BOX_BYTES, 1024)
                                           : sdesc(st + a_bytes + kk * 32, 16, 1024);
                umma_f16(tmem, da, db, idesc, (kb | kk) ? 1u : 0u);
            }
            umma_commit(&empty_bar[s]);
        }
        // after an abort the epilogue is not released (its bounded wait expires): copies may
        // still land in the stage buffers it would reuse
        if (!*abort_flag) umma_commit(acc_bar);
        umma_commit(mma_bar);
        if (!mbar_wait(mma_bar, 0)) atomicExch(g.err, 14);     // all MMAs done before the dealloc
    } else if (warp >= 2) {
        // ---- epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows); each 32 x 32
        // block goes through a padded shared tile so that lane = column for the stores
        const int quarter = warp % 4, half = (warp - 2) / 4;   // TMEM lanes 32 quarter.., column chunks half, half + 2, ..
        const int rbase = m0 + quarter * 32;
        float* tile = epi_tile + (warp - 2) * 32 * G_EPI_LD;
        const bool ok = __all_sync(0xffffffffu, mbar_wait(acc_bar, 0));
        if (!ok) {
            *abort_flag = 1;
            atomicExch(g.err, 15);
        }
        tc_fence_after();
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16);
        float* out_f32 = g.out_f32 ? g.out_f32 + (int64_t)blockIdx.z * g.split_stride : nullptr;
        const int rows = min(32, g.M - rbase);
        for (int c0 = 32 * half; c0 < nt; c0 += 64) {
            float v[32];
            tmem_ld32(taddr + c0, v);
            if (!ok || rows <= 0) continue;
#pragma unroll
            for (int q = 0; q < 32; ++q) tile[lane * G_EPI_LD + q] = v[q];
            __syncwarp();
#pragma unroll
            for (int r = 0; r < 32; ++r) v[r] = tile[r * G_EPI_LD + lane];   // v[r] = (row rbase + r, column lane)
            __syncwarp();
            const int n = n0 + c0 + lane;
            if (c0 + lane >= nt || n >= g.N) continue;
            const float bias = g.bias ? g.bias[n] : 0.f;
            const int64_t base = (int64_t)rbase;
            if (g.epi == EPI_F32 || g.epi == EPI_BIAS_F32) {
#pragma unroll
                for (int r = 0; r < 32; ++r)
                    if (r < rows) out_f32[(base + r) * g.ld_f32 + n] = v[r] + bias;
            } else if (g.epi == EPI_BIAS_GELU) {
                if (out_f32) {
#pragma unroll
                    for (int r = 0; r < 32; ++r)
                        if (r < rows) out_f32[(base + r) * g.ld_f32 + n] = v[r] + bias;
                }
#pragma unroll
                for (int r = 0; r < 32; ++r)
                    if (r < rows) g.out_bf16[(base + r) * g.ld_bf16 + n] = __float2bfloat16_rn(gelu(v[r] + bias));
            } else {   // EPI_GELU_BWD
                float z[32];
#pragma unroll
                for (int r = 0; r < 32; ++r) z[r] = r < rows ? g.zin[(base + r) * g.ld_z + n] : 0.f;
#pragma unroll
                for (int r = 0; r < 32; ++r)
                    if (r < rows) g.out_bf16[(base + r) * g.ld_bf16 + n] = __float2bfloat16_rn(v[r] * gelu_grad(z[r]));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
    }
}

// 2-D tensor map of a row-major BF16 matrix [rows][cols] (row pitch ld elements),
// box 64 x 64, 128-byte swizzle, zero fill outside.
bool make_map(CUtensorMap* map, const void* base, int64_t rows, int64_t cols, int64_t ld) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    std::memset(map, 0, sizeof *map);
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {G_BOX, G_BOX};
    cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Dynamic shared memory of a launch with an N tile of nt columns; the kernel's limit is
// raised once per device to the largest (nt = 256).
int gemm_smem(int nt) {
    const int stage_bytes = 2 * G_BOX_BYTES + ((nt + G_BOX - 1) / G_BOX) * G_BOX_BYTES;
    static_assert(G_EPI_BYTES <= G_STAGES * 3 * G_BOX_BYTES, "the epilogue tiles live in the stage buffers");
    return 1024 + G_STAGES * stage_bytes + 256;
}
cudaError_t gemm_attributes() {
    static std::mutex mu;
    static std::vector<bool> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= dev) done.resize(dev + 1, false);
    if (done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(bf16_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_smem(256));
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

// Tensor maps of one network's buffers, reused across steps (encoding them costs host
// time on every product otherwise); keyed by base, rows, columns and pitch
struct MapCache {
    struct Entry {
        const void* base;
        int64_t rows, cols, ld;
        CUtensorMap map;
    };
    std::vector<Entry> e;
};
bool cached_map(MapCache* c, CUtensorMap* out, const void* base, int64_t rows, int64_t cols, int64_t ld) {
    if (!c) return make_map(out, base, rows, cols, ld);
    for (const auto& x : c->e)
        if (x.base == base && x.rows == rows && x.cols == cols && x.ld == ld) {
            *out = x.map;
            return true;
        }
    if (c->e.size() >= 64) c->e.clear();
    MapCache::Entry x{base, rows, cols, ld, {}};
    if (!make_map(&x.map, base, rows, cols, ld)) return false;
    c->e.push_back(x);
    *out = x.map;
    return true;
}

// C = A B with A [M][K] (a_mn = 0: stored [M][lda], K contiguous; 1: stored [K][lda],
// M contiguous) and B [K][N] (b_mn = 0: stored [N][ldb]; 1: stored [K][ldb]).
// ksplit > 1 (EPI_F32 only) splits K over grid z; slice z writes its partial product to
// g.out_f32 + z g.split_stride, which the caller reduces.
cudaError_t gemm(const __nv_bfloat16* A, int64_t lda, int a_mn, const __nv_bfloat16* B, int64_t ldb, int b_mn,
                 GemmArgs g, cudaStream_t s, int ksplit = 1, int* nz_out = nullptr, MapCache* cache = nullptr) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0) return cudaSuccess;
    if ((lda * 2) % 16 || (ldb * 2) % 16) return cudaErrorInvalidValue;   // TMA row pitch
    CUtensorMap ma, mb;
    const bool ok_a = a_mn ? cached_map(cache, &ma, A, g.K, g.M, lda) : cached_map(cache, &ma, A, g.M, g.K, lda);
    const bool ok_b = b_mn ? cached_map(cache, &mb, B, g.K, g.N, ldb) : cached_map(cache, &mb, B, g.N, g.K, ldb);
    if (!ok_a || !ok_b) return cudaErrorInvalidValue;
    const cudaError_t ea = gemm_attributes();
    if (ea != cudaSuccess) return ea;
    g.a_mn = a_mn;
    g.b_mn = b_mn;
    const int nkb = (g.K + G_BOX - 1) / G_BOX;
    g.kb_per_split = ksplit > 1 ? (nkb + ksplit - 1) / ksplit : nkb;
    const int nz = (nkb + g.kb_per_split - 1) / g.kb_per_split;     // every slice has >= 1 block
    if (nz > 1 && g.epi != EPI_F32) return cudaErrorInvalidValue;
    if (nz_out) *nz_out = nz;
    // N tile: up to 256 columns; 128 when that still fits two CTAs per SM in one wave
    // (more SMs share a small product's epilogue)
    int nt = std::min(256, (g.N + 15) / 16 * 16);
    const int64_t mtiles = (g.M + 127) / 128;
    if (nt > 128 && mtiles * ((g.N + 127) / 128) * nz <= 2 * 148) nt = 128;
    uint32_t cols = 32;
    while ((int)cols < nt) cols <<= 1;
    dim3 grid((unsigned)mtiles, (g.N + nt - 1) / nt, nz);
    bf16_gemm_kernel<<<grid, G_THREADS, gemm_smem(nt), s>>>(ma, mb, g, nt, cols);
    return cudaGetLastError();
}

// out[m][n] (row pitch ldo) = sum over z of partial[z][m][n] (pitch N), in order of z
__global__ void split_reduce_kernel(const float* __restrict__ partial, int nz, int64_t M, int N, float* __restrict__ out,
                                    int64_t ldo) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= M * N) return;
    float acc = 0.f;
    for (int z = 0; z < nz; ++z) acc += partial[z * M * N + i];
    out[(i / N) * ldo + i % N] = acc;
}

// ---- elementwise kernels ----
// X0[b][0..63] = bf16((x[b][i] - mean[i]) / std[i]) for i < nin, 0 beyond
__global__ void normalize_in_kernel(const float* __restrict__ x, int64_t ldx, int B, int nin, const float* __restrict__ mean,
                                    const float* __restrict__ stdv, __nv_bfloat16* __restrict__ X0, int ld0) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * ld0) return;
    const int b = (int)(i / ld0), c = (int)(i % ld0);
    const float v = c < nin ? (x[(int64_t)b * ldx + c] - mean[c]) / stdv[c] : 0.f;
    X0[i] = __float2bfloat16_rn(v);
}
// dY = bf16(2 (Y - yn) / (B nout)), yn = (y - mean) / std; loss += sum (Y - yn)^2 / (B nout)
__global__ void output_grad_kernel(const float* __restrict__ Y, const float* __restrict__ y, int B, int nout,
                                   const float* __restrict__ mean, const float* __restrict__ stdv,
                                   __nv_bfloat16* __restrict__ dY, float* __restrict__ loss) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    float l = 0.f;
    if (i < (int64_t)B * nout) {
        const int c = (int)(i % nout);
        const float d = Y[i] - (y[i] - mean[c]) / stdv[c];
        const float inv = 1.f / ((float)B * nout);
        dY[i] = __float2bfloat16_rn(2.f * d * inv);
        l = d * d * inv;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}
// db[n] = sum_b dZ[b][n], deterministic in one pass: a block sums 32 columns, warp w the
// rows w, w + 8, ... (lanes over consecutive columns: coalesced), then warp 0 adds the 8
// partial sums in order
__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ dZ, int B, int N, int64_t ld,
                                 float* __restrict__ db) {
    __shared__ float part[8][32];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int n = blockIdx.x * 32 + lane;
    float acc = 0.f;
    if (n < N)
        for (int b = warp; b < B; b += 8) acc += __bfloat162float(dZ[(int64_t)b * ld + n]);
    part[warp][lane] = acc;
    __syncthreads();
    if (warp == 0 && n < N) {
        float t = 0.f;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += part[w][lane];
        db[n] = t;
    }
}
// Adam over all parameter tensors in one launch (per tensor: master, gradient, moments,
// optional BF16 copy, length); thread i updates element i of the concatenation
struct AdamSet {
    float* w[8];
    const float* g[8];
    float* m[8];
    float* v[8];
    __nv_bfloat16* wb[8];
    int64_t end[8];      // cumulative lengths
    int count;
};
__global__ void adam_multi_kernel(const AdamSet set, float lr, float b1, float b2, float c1, float c2, float eps) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= set.end[set.count - 1]) return;
    int t = 0;
    while (i >= set.end[t]) ++t;
    const int64_t j = i - (t ? set.end[t - 1] : 0);
    const float g = set.g[t][j];
    const float mi = b1 * set.m[t][j] + (1.f - b1) * g;
    const float vi = b2 * set.v[t][j] + (1.f - b2) * g * g;
    set.m[t][j] = mi;
    set.v[t][j] = vi;
    const float wi = set.w[t][j] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    set.w[t][j] = wi;
    if (set.wb[t]) set.wb[t][j] = __float2bfloat16_rn(wi);
}
// y[b][c] = Y[b][c] std[c] + mean[c]
__global__ void denormalize_kernel(const float* __restrict__ Y, int B, int nout, const float* __restrict__ mean,
                                   const float* __restrict__ stdv, float* __restrict__ y, int64_t ldy) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= (int64_t)B * nout) return;
    const int b = (int)(i / nout), c = (int)(i % nout);
    y[(int64_t)b * ldy + c] = Y[i] * stdv[c] + mean[c];
}
__global__ void to_bf16_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int64_t n) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// ---- the emulator as one kernel ----------------------------------------------------
// One CTA per 128 columns: the inputs are gathered from the layer-major fields,
// normalised and written as BF16 straight into the K-major 128-byte-swizzled activation
// tile in shared memory; the four layers run on tcgen05 with the weights streamed by TMA
// (three 32 KB stages, 13 blocks of 64 input features in all) and the accumulator in
// TMEM; after each hidden layer 8 epilogue warps add the bias, apply GELU and write the
// BF16 activations back into the tile in place (the layer's MMAs have completed), so no
// activation leaves the SM. The output layer is de-normalised and written into the
// tendency fields; columns outside the training range get the plain physics instead.
constexpr int NLC = SHT_COLUMN_LAYERS;
constexpr int F_THREADS = 576;                       // producer warp, MMA warp, 16 epilogue warps
constexpr int F_EPI = F_THREADS - 64;                // epilogue threads
constexpr int F_STAGES = 3;
constexpr int F_W_STAGE = 4 * G_BOX_BYTES;           // 256 rows x 64 features
constexpr int F_ACT_BYTES = 4 * 2 * G_BOX_BYTES;     // 128 rows x 256 features (4 blocks of 16 KB)
constexpr int F_TAIL = 128 + 512;                    // barriers, inside flags [4][128]
// the network's constants, staged once per CTA: input mean / std [33] [33], output mean /
// std [16] [16], biases [256] [256] [256] [16]
constexpr int F_C_XM = 0, F_C_XS = 33, F_C_YM = 66, F_C_YS = 82, F_C_B0 = 98, F_C_B1 = 354, F_C_B2 = 610,
              F_C_B3 = 866, F_C_N = 882;
constexpr int F_CONST = 4096;
static_assert(F_C_N * 4 <= F_CONST, "constants exceed their shared-memory area");
constexpr int F_SMEM = 1024 + F_ACT_BYTES + F_STAGES * F_W_STAGE + F_TAIL + F_CONST;

struct FusedArgs {
    const float *T, *q, *u, *v, *ps;
    int64_t ld;
    int ncol;
    int cpb;                 // columns per CTA (<= 128: the MMA tile's rows)
    const float *xm, *xs, *ym, *ys;
    const float* bias[4];
    float zmax, dt;
    colphys::Levels L;
    float *dT, *dq;
    int add;
    int32_t* nfallback;
    int32_t* err;
};

// byte offset of feature k (< 256) of row r (< 128) in the K-major SWIZZLE_128B tile
__device__ __forceinline__ uint32_t act_off(int r, int k) {
    return (uint32_t)((k >> 6) * (2 * G_BOX_BYTES) + r * 128 + ((((k & 63) >> 3) ^ (r & 7)) << 4) + ((k & 7) << 1));
}
// two reals rounded to bf16 (each to nearest, as two separate roundings) by one paired
// conversion instruction
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__global__ void __launch_bounds__(F_THREADS, 1)
    mlp_fused_kernel(const __grid_constant__ CUtensorMap w0, const __grid_constant__ CUtensorMap w1,
                     const __grid_constant__ CUtensorMap w2, const __grid_constant__ CUtensorMap w3,
                     const FusedArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* act = smem;
    uint8_t* wst = smem + F_ACT_BYTES;
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(wst + F_STAGES * F_W_STAGE);
    uint64_t* empty_bar = full_bar + F_STAGES;
    uint64_t* acc_bar = empty_bar + F_STAGES;         // layer l accumulated (phase l)
    uint64_t* act_bar = acc_bar + 1;                  // input of layer l in the tile (phase l)
    uint64_t* mma_bar = act_bar + 1;                  // every issued MMA complete
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_bar + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    uint8_t* inside = reinterpret_cast<uint8_t*>(full_bar) + 128;
    float* cst = reinterpret_cast<float*>(inside + 512);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int col0 = blockIdx.x * a.cpb;
    const int nrow = min(a.cpb, a.ncol - col0);
    // per layer: K blocks of 64 inputs, 64-row boxes of weights, outputs (no arrays: no stack)
    auto nkb = [](int l) { return l == 0 ? 1 : 4; };
    auto nbox = [](int l) { return l == 3 ? 1 : 4; };
    auto nout = [](int l) { return l == 3 ? 16 : 256; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < F_STAGES; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(acc_bar, 1);
        mbar_init(act_bar, F_EPI);
        mbar_init(mma_bar, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(256u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    // the epilogue warps' raw inputs, loaded before the barrier that publishes the
    // constants (both loads in flight at once): row r, features [16 kh, 16 kh + 16)
    float raw[16];
    if (warp >= 2) {
        const int et = threadIdx.x - 64, r = et & 127, kh = et >> 7;
        const int64_t ij = col0 + r;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int c = 16 * kh + i;
            float x = 0.f;
            if (c < 4 * NLC + 1 && r < nrow) {
                if (c < 4 * NLC) {
                    const float* f = c < NLC ? a.T : c < 2 * NLC ? a.q : c < 3 * NLC ? a.u : a.v;
                    x = __ldg(f + (int64_t)(c % NLC) * a.ld + ij);
                } else {
                    x = __ldg(a.ps + ij);
                }
            }
            raw[i] = x;
        }
    }
    for (int i = threadIdx.x; i < F_C_N; i += blockDim.x) {   // the constants, read once
        float c;
        if (i < F_C_XS) c = a.xm[i];
        else if (i < F_C_YM) c = a.xs[i - F_C_XS];
        else if (i < F_C_YS) c = a.ym[i - F_C_YM];
        else if (i < F_C_B0) c = a.ys[i - F_C_YS];
        else if (i < F_C_B1) c = a.bias[0][i - F_C_B0];
        else if (i < F_C_B2) c = a.bias[1][i - F_C_B1];
        else if (i < F_C_B3) c = a.bias[2][i - F_C_B2];
        else c = a.bias[3][i - F_C_B3];
        cst[i] = c;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ---- producer: the weight blocks of the four layers in order
        int g = 0;
        for (int l = 0; l < 4 && !*abort_flag; ++l) {
            const CUtensorMap* map = l == 0 ? &w0 : l == 1 ? &w1 : l == 2 ? &w2 : &w3;
            for (int kb = 0; kb < nkb(l) && !*abort_flag; ++kb, ++g) {
                const int s = g % F_STAGES;
                if (g >= F_STAGES && !mbar_wait(&empty_bar[s], ((g / F_STAGES) - 1) & 1)) {
                    *abort_flag = 1;
                    atomicExch(a.err, 21);
                    break;
                }
                uint8_t* st = wst + s * F_W_STAGE;
                mbar_expect_tx(&full_bar[s], (uint32_t)(nbox(l) * G_BOX_BYTES));
                for (int h = 0; h < nbox(l); ++h) tma_load_2d(st + h * G_BOX_BYTES, map, kb * G_BOX, h * G_BOX, &full_bar[s]);
            }
        }
        for (int u = g - 1; u >= 0 && u >= g - F_STAGES; --u)   // no copy lands after the exit
            if (!mbar_wait(&full_bar[u % F_STAGES], (u / F_STAGES) & 1)) atomicExch(a.err, 22);
    } else if (warp == 1 && lane == 0) {
        // ---- MMA issuer: layer l once its input is in the tile
        int g = 0;
        bool ok = true;
        for (int l = 0; l < 4 && ok; ++l) {
            if (!mbar_wait(act_bar, l & 1)) {
                *abort_flag = 1;
                atomicExch(a.err, 23);
                break;
            }
            tc_fence_after();
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (((uint32_t)nout(l) >> 3) << 17) | ((128u >> 4) << 24);
            for (int kb = 0; kb < nkb(l); ++kb, ++g) {
                const int s = g % F_STAGES;
                if (!mbar_wait(&full_bar[s], (g / F_STAGES) & 1)) {
                    *abort_flag = 1;
                    atomicExch(a.err, 24);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t sa = smem_u32(act + kb * 2 * G_BOX_BYTES), sb = smem_u32(wst + s * F_W_STAGE);
                for (int kk = 0; kk < G_BOX / 16; ++kk)
                    umma_f16(tmem, sdesc(sa + kk * 32, 16, 1024), sdesc(sb + kk * 32, 16, 1024), idesc,
                             (kb | kk) ? 1u : 0u);
                umma_commit(&empty_bar[s]);
            }
            if (ok) umma_commit(acc_bar);
        }
        umma_commit(mma_bar);
        if (!mbar_wait(mma_bar, 0)) atomicExch(a.err, 25);
    } else if (warp >= 2) {
        const int et = threadIdx.x - 64;
        {   // ---- gather: row r, features [16 kh, 16 kh + 16), normalised, BF16 into the tile
            const int r = et & 127, kh = et >> 7;
            bool in = true;
            uint32_t pk[8];
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
                float z2[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int c = 16 * kh + i + e;
                    float z = 0.f;
                    if (c < 4 * NLC + 1 && r < nrow) {
                        const float x = c < 4 * NLC ? raw[i + e] : logf(raw[i + e]);
                        z = (x - cst[F_C_XM + c]) / cst[F_C_XS + c];
                        in = in && fabsf(z) <= a.zmax;
                    }
                    z2[e] = z;
                }
                pk[i / 2] = pack_bf16x2(z2[0], z2[1]);
            }
#pragma unroll
            for (int c8 = 0; c8 < 2; ++c8)
                *reinterpret_cast<uint4*>(act + act_off(r, 16 * kh + 8 * c8)) =
                    make_uint4(pk[4 * c8], pk[4 * c8 + 1], pk[4 * c8 + 2], pk[4 * c8 + 3]);
            // features 64 .. 255 of layer 1 stay unread (its K is 64)
            inside[kh * 128 + r] = in ? 1 : 0;
            fence_proxy_async();
            mbar_arrive(act_bar);
            asm volatile("bar.sync 1, %0;" ::"n"(F_EPI) : "memory");   // the flags, among the epilogue warps
        }
        // warp w reads TMEM lanes 32 (w % 4) .. + 31; the four warps of a lane quarter take
        // every fourth 32-column chunk
        const int quarter = warp % 4, half = (warp - 2) / 4;
        const int r = quarter * 32 + lane;
        const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16);
        bool ok = true;
        const bool rows_used = quarter * 32 < nrow;   // lane quarters past the CTA's columns skip the work
        for (int l = 0; l < 3 && ok; ++l) {   // ---- hidden layers: bias, GELU, BF16 in place
            ok = __all_sync(0xffffffffu, mbar_wait(acc_bar, l & 1));
            if (!ok) {
                *abort_flag = 1;
                atomicExch(a.err, 26);
                break;
            }
            tc_fence_after();
            const float* bias = cst + (l == 0 ? F_C_B0 : l == 1 ? F_C_B1 : F_C_B2);
            for (int c0 = 32 * half; c0 < (rows_used ? 256 : 0); c0 += 128) {
                float v[32];
                tmem_ld32(taddr + c0, v);
                uint32_t pk[16];
#pragma unroll
                for (int q2 = 0; q2 < 16; ++q2)
                    pk[q2] = pack_bf16x2(gelu(v[2 * q2] + bias[c0 + 2 * q2]), gelu(v[2 * q2 + 1] + bias[c0 + 2 * q2 + 1]));
#pragma unroll
                for (int c8 = 0; c8 < 4; ++c8)
                    *reinterpret_cast<uint4*>(act + act_off(r, c0 + 8 * c8)) =
                        make_uint4(pk[4 * c8], pk[4 * c8 + 1], pk[4 * c8 + 2], pk[4 * c8 + 3]);
            }
            fence_proxy_async();
            tc_fence_before();
            mbar_arrive(act_bar);
        }
        if (ok) {   // ---- output layer (16 columns): de-normalise, or the plain physics outside the range
            ok = __all_sync(0xffffffffu, mbar_wait(acc_bar, 1));
            if (!ok) {
                *abort_flag = 1;
                atomicExch(a.err, 27);
            }
        }
        if (ok && half == 0) {
            tc_fence_after();
            float v[32];
            tmem_ld32(taddr, v);
            if (r < nrow) {
                const int64_t ij = col0 + r;
                float dT[NLC], dq[NLC];
                if (inside[r] && inside[128 + r] && inside[256 + r] && inside[384 + r]) {
#pragma unroll
                    for (int k = 0; k < NLC; ++k) {
                        const float y0 = v[k] + cst[F_C_B3 + k], y1 = v[NLC + k] + cst[F_C_B3 + NLC + k];
                        dT[k] = y0 * cst[F_C_YS + k] + cst[F_C_YM + k];
                        dq[k] = y1 * cst[F_C_YS + NLC + k] + cst[F_C_YM + NLC + k];
                    }
                } else {
                    float T[NLC], q[NLC];
#pragma unroll
                    for (int k = 0; k < NLC; ++k) {
                        T[k] = a.T[(int64_t)k * a.ld + ij];
                        q[k] = a.q[(int64_t)k * a.ld + ij];
                    }
                    colphys::column_tendencies(T, q, a.ps[ij], a.dt, a.L, dT, dq);
                    if (a.nfallback) atomicAdd(a.nfallback, 1);
                }
#pragma unroll
                for (int k = 0; k < NLC; ++k) {
                    float* pa = a.dT + (int64_t)k * a.ld + ij;
                    float* pb = a.dq + (int64_t)k * a.ld + ij;
                    *pa = a.add ? *pa + dT[k] : dT[k];
                    *pb = a.add ? *pb + dq[k] : dq[k];
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u) : "memory");
    }
}

cudaError_t fused_attributes() {
    static std::mutex mu;
    static std::vector<bool> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)done.size() <= dev) done.resize(dev + 1, false);
    if (done[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(mlp_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, F_SMEM);
    if (e == cudaSuccess) done[dev] = true;
    return e;
}


}  // namespace

// ------------------------------------------------------------------------------------
struct sht_mlp {
    static constexpr int NLAYER = 4;
    int device = 0, cap = 0;
    int nin = 4 * SHT_COLUMN_LAYERS + 1, in_pad = 64, hidden = 256, nout = 2 * SHT_COLUMN_LAYERS;
    int fan_in[NLAYER], fan_out[NLAYER];          // padded input width, output width
    float *W[NLAYER] = {}, *b[NLAYER] = {};        // FP32 masters [out][in_pad], [out]
    __nv_bfloat16* Wb[NLAYER] = {};
    float *mW[NLAYER] = {}, *vW[NLAYER] = {}, *mb[NLAYER] = {}, *vb[NLAYER] = {};
    float *dW[NLAYER] = {}, *db[NLAYER] = {};
    __nv_bfloat16* X0 = nullptr;                    // [cap][in_pad]
    float* Z[3] = {};                               // pre-activations [cap][hidden]
    __nv_bfloat16* A[3] = {};                       // activations [cap][hidden]
    __nv_bfloat16* dZ[3] = {};                      // [cap][hidden]
    float* Y = nullptr;                             // [cap][nout]
    __nv_bfloat16* dY = nullptr;                    // [cap][nout]
    float *xm = nullptr, *xs = nullptr, *ym = nullptr, *ys = nullptr;   // normalisation
    float* loss = nullptr;
    CUtensorMap wmap[NLAYER];                       // TMA maps of the BF16 weights (fused emulator kernel)
    MapCache maps;                                  // TMA maps of the layer-by-layer products
    int* nfallback = nullptr;
    static constexpr int MAX_SPLIT = 32;
    float* splitbuf = nullptr;                      // [MAX_SPLIT][256][256] split-K partial weight gradients
    int32_t* err = nullptr;
    int step = 0;
};

namespace {
thread_local char g_msg[256];
int mcuda(cudaError_t e, const char* what) {
    snprintf(g_msg, sizeof g_msg, "%s: %s", what, cudaGetErrorString(e));
    return set_error(e == cudaErrorMemoryAllocation ? SHT_ENOMEM : SHT_ECUDA, g_msg);
}
struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};
template <class T>
cudaError_t alloc(T** p, size_t n) {
    return cudaMalloc((void**)p, std::max<size_t>(1, n) * sizeof(T));
}
void release(sht_mlp* m) {
    for (int l = 0; l < sht_mlp::NLAYER; ++l) {
        void* ps[] = {m->W[l], m->b[l], m->Wb[l], m->mW[l], m->vW[l], m->mb[l], m->vb[l], m->dW[l], m->db[l]};
        for (void* q : ps)
            if (q) cudaFree(q);
    }
    for (int l = 0; l < 3; ++l) {
        void* ps[] = {m->Z[l], m->A[l], m->dZ[l]};
        for (void* q : ps)
            if (q) cudaFree(q);
    }
    void* ps[] = {m->X0, m->Y, m->dY, m->xm, m->xs, m->ym, m->ys, m->loss, m->nfallback, m->splitbuf,
                  m->err};
    for (void* q : ps)
        if (q) cudaFree(q);
}

GemmArgs args(sht_mlp* m, int M, int N, int K, int epi) {
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.epi = epi;
    g.err = m->err;
    return g;
}

// forward pass over B rows of X0; keep = store the pre-activations (for the backward pass)
cudaError_t forward(sht_mlp* m, int B, bool keep, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    const __nv_bfloat16* in = m->X0;
    int64_t ld_in = m->in_pad;
    for (int l = 0; l < 3 && e == cudaSuccess; ++l) {
        GemmArgs g = args(m, B, m->hidden, m->fan_in[l], EPI_BIAS_GELU);
        g.out_f32 = keep ? m->Z[l] : nullptr;
        g.ld_f32 = m->hidden;
        g.out_bf16 = m->A[l];
        g.ld_bf16 = m->hidden;
        g.bias = m->b[l];
        e = gemm(in, ld_in, 0, m->Wb[l], m->fan_in[l], 0, g, s, 1, nullptr, &m->maps);
        in = m->A[l];
        ld_in = m->hidden;
    }
    if (e != cudaSuccess) return e;
    GemmArgs g = args(m, B, m->nout, m->hidden, EPI_BIAS_F32);
    g.out_f32 = m->Y;
    g.ld_f32 = m->nout;
    g.bias = m->b[3];
    return gemm(in, ld_in, 0, m->Wb[3], m->hidden, 0, g, s, 1, nullptr, &m->maps);
}
}  // namespace

int sht_mlp_create(int batch_capacity, uint64_t seed, int device, sht_mlp** out) {
    if (!out || batch_capacity < 1) return set_error(SHT_EINVAL, "sht_mlp_create: bad arguments");
    *out = nullptr;
    DevGuard dg(device);
    sht_mlp* m = new sht_mlp();
    m->device = device;
    m->cap = (batch_capacity + 127) / 128 * 128;
    const int fi[4] = {m->in_pad, m->hidden, m->hidden, m->hidden};
    const int fo[4] = {m->hidden, m->hidden, m->hidden, m->nout};
    cudaError_t e = cudaSuccess;
    std::mt19937_64 rng(seed);
    for (int l = 0; l < 4 && e == cudaSuccess; ++l) {
        m->fan_in[l] = fi[l];
        m->fan_out[l] = fo[l];
        const size_t nw = (size_t)fo[l] * fi[l];
        const int real_in = l == 0 ? m->nin : fi[l];
        // He initialisation for GELU layers, Xavier for the output; padded inputs get 0
        std::normal_distribution<float> nd(0.f, l < 3 ? std::sqrt(2.f / real_in) : std::sqrt(1.f / real_in));
        std::vector<float> w(nw, 0.f);
        for (int o = 0; o < fo[l]; ++o)
            for (int i = 0; i < real_in; ++i) w[(size_t)o * fi[l] + i] = nd(rng);
        std::vector<float> z(nw, 0.f);
        if ((e = alloc(&m->W[l], nw)) != cudaSuccess) break;
        if ((e = cudaMemcpy(m->W[l], w.data(), nw * 4, cudaMemcpyHostToDevice)) != cudaSuccess) break;
        if ((e = alloc(&m->Wb[l], nw)) != cudaSuccess) break;
        to_bf16_kernel<<<(unsigned)((nw + 255) / 256), 256>>>(m->W[l], m->Wb[l], (int64_t)nw);
        if ((e = alloc(&m->mW[l], nw)) == cudaSuccess) e = cudaMemset(m->mW[l], 0, nw * 4);
        if (e == cudaSuccess && (e = alloc(&m->vW[l], nw)) == cudaSuccess) e = cudaMemset(m->vW[l], 0, nw * 4);
        if (e == cudaSuccess) e = alloc(&m->dW[l], nw);
        if (e == cudaSuccess && (e = alloc(&m->b[l], fo[l])) == cudaSuccess) e = cudaMemset(m->b[l], 0, fo[l] * 4);
        if (e == cudaSuccess && (e = alloc(&m->mb[l], fo[l])) == cudaSuccess) e = cudaMemset(m->mb[l], 0, fo[l] * 4);
        if (e == cudaSuccess && (e = alloc(&m->vb[l], fo[l])) == cudaSuccess) e = cudaMemset(m->vb[l], 0, fo[l] * 4);
        if (e == cudaSuccess) e = alloc(&m->db[l], fo[l]);
    }
    const size_t cap = m->cap;
    if (e == cudaSuccess && (e = alloc(&m->X0, cap * m->in_pad)) == cudaSuccess) e = cudaMemset(m->X0, 0, cap * m->in_pad * 2);
    for (int l = 0; l < 3 && e == cudaSuccess; ++l) {
        if ((e = alloc(&m->Z[l], cap * m->hidden)) != cudaSuccess) break;
        if ((e = alloc(&m->A[l], cap * m->hidden)) != cudaSuccess) break;
        e = alloc(&m->dZ[l], cap * m->hidden);
    }
    if (e == cudaSuccess) e = alloc(&m->Y, cap * m->nout);
    if (e == cudaSuccess) e = alloc(&m->dY, cap * m->nout);
    if (e == cudaSuccess) e = alloc(&m->xm, m->nin);
    if (e == cudaSuccess) e = alloc(&m->xs, m->nin);
    if (e == cudaSuccess) e = alloc(&m->ym, m->nout);
    if (e == cudaSuccess) e = alloc(&m->ys, m->nout);
    if (e == cudaSuccess) e = alloc(&m->loss, 1);
    if (e == cudaSuccess) e = alloc(&m->nfallback, 1);
    if (e == cudaSuccess) e = alloc(&m->splitbuf, (size_t)sht_mlp::MAX_SPLIT * m->hidden * m->hidden);
    if (e == cudaSuccess && (e = alloc(&m->err, 1)) == cudaSuccess) e = cudaMemset(m->err, 0, 4);
    if (e == cudaSuccess) {          // identity normalisation until set
        std::vector<float> zero(m->nin, 0.f), one(m->nin, 1.f);
        cudaMemcpy(m->xm, zero.data(), m->nin * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(m->xs, one.data(), m->nin * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(m->ym, zero.data(), m->nout * 4, cudaMemcpyHostToDevice);
        e = cudaMemcpy(m->ys, one.data(), m->nout * 4, cudaMemcpyHostToDevice);
    }
    for (int l = 0; l < 4 && e == cudaSuccess; ++l)
        if (!make_map(&m->wmap[l], m->Wb[l], m->fan_out[l], m->fan_in[l], m->fan_in[l])) e = cudaErrorInvalidValue;
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        release(m);
        delete m;
        return mcuda(e, "sht_mlp_create");
    }
    *out = m;
    return SHT_OK;
}

int sht_mlp_set_normalization(sht_mlp* m, const float* x_mean, const float* x_std, const float* y_mean,
                              const float* y_std) {
    if (!m || !x_mean || !x_std || !y_mean || !y_std) return set_error(SHT_EINVAL, "sht_mlp_set_normalization: NULL");
    for (int i = 0; i < m->nin; ++i)
        if (!(x_std[i] > 0)) return set_error(SHT_EINVAL, "sht_mlp_set_normalization: std must be > 0");
    for (int i = 0; i < m->nout; ++i)
        if (!(y_std[i] > 0)) return set_error(SHT_EINVAL, "sht_mlp_set_normalization: std must be > 0");
    DevGuard dg(m->device);
    cudaError_t e = cudaMemcpy(m->xm, x_mean, m->nin * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->xs, x_std, m->nin * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->ym, y_mean, m->nout * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(m->ys, y_std, m->nout * 4, cudaMemcpyHostToDevice);
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_mlp_set_normalization");
}

namespace {
// loss and gradients dW, db of every layer for the batch (x [B][33], y [B][16])
cudaError_t backward(sht_mlp* m, const float* x, const float* y, int B, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(m->loss, 0, 4, s);
    const int64_t nx = (int64_t)B * m->in_pad;
    normalize_in_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, s>>>(x, m->nin, B, m->nin, m->xm, m->xs, m->X0,
                                                                     m->in_pad);
    if (e == cudaSuccess) e = forward(m, B, true, s);
    const int64_t ny = (int64_t)B * m->nout;
    if (e == cudaSuccess)
        output_grad_kernel<<<(unsigned)((ny + 255) / 256), 256, 0, s>>>(m->Y, y, B, m->nout, m->ym, m->ys, m->dY,
                                                                         m->loss);
    // backward: layer 3 (output), then the hidden layers
    const __nv_bfloat16* act[4] = {m->X0, m->A[0], m->A[1], m->A[2]};
    const int64_t ld_act[4] = {m->in_pad, m->hidden, m->hidden, m->hidden};
    const __nv_bfloat16* dz = m->dY;
    int64_t ld_dz = m->nout;
    for (int l = 3; l >= 0 && e == cudaSuccess; --l) {
        const int fo = m->fan_out[l], fi = m->fan_in[l];
        // dW[l] [fo][fi] = dz^T act[l]   (A = dz MN-major, B = act MN-major), K = B split
        // over grid z into slices of >= 2 blocks of 64 rows, about one CTA per SM in all,
        // partial products reduced in a fixed order (deterministic)
        GemmArgs gw = args(m, fo, fi, B, EPI_F32);
        const int tiles = ((fo + 127) / 128) * ((fi + 255) / 256);
        const int ksplit = std::max(1, std::min(std::min((int)sht_mlp::MAX_SPLIT, 148 / tiles), (B + 127) / 128));
        gw.out_f32 = m->splitbuf;
        gw.ld_f32 = fi;
        gw.split_stride = (int64_t)fo * fi;
        int nz = 1;
        e = gemm(dz, ld_dz, 1, act[l], ld_act[l], 1, gw, s, ksplit, &nz, &m->maps);
        if (e != cudaSuccess) break;
        split_reduce_kernel<<<(unsigned)(((int64_t)fo * fi + 255) / 256), 256, 0, s>>>(m->splitbuf, nz, fo, fi,
                                                                                        m->dW[l], fi);
        bias_grad_kernel<<<(fo + 31) / 32, 256, 0, s>>>(dz, B, fo, ld_dz, m->db[l]);
        if (l == 0) break;
        // dZ[l-1] = (dz W[l]) * GELU'(Z[l-1])   (A = dz K-major, B = W[l] [fo][fi] MN-major)
        GemmArgs gd = args(m, B, fi, fo, EPI_GELU_BWD);
        gd.out_bf16 = m->dZ[l - 1];
        gd.ld_bf16 = m->hidden;
        gd.zin = m->Z[l - 1];
        gd.ld_z = m->hidden;
        e = gemm(dz, ld_dz, 0, m->Wb[l], fi, 1, gd, s, 1, nullptr, &m->maps);
        dz = m->dZ[l - 1];
        ld_dz = m->hidden;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}
}  // namespace

int sht_mlp_backward(sht_mlp* m, const float* x, const float* y, int B, void* stream) {
    if (!m || !x || !y) return set_error(SHT_EINVAL, "sht_mlp_backward: NULL argument");
    if (B < 1 || B > m->cap) return set_error(SHT_EINVAL, "sht_mlp_backward: batch outside 1 .. capacity");
    DevGuard dg(m->device);
    const cudaError_t e = backward(m, x, y, B, (cudaStream_t)stream);
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_mlp_backward");
}

int sht_mlp_train_step(sht_mlp* m, const float* x, const float* y, int B, float lr, void* stream) {
    if (!m || !x || !y) return set_error(SHT_EINVAL, "sht_mlp_train_step: NULL argument");
    if (B < 1 || B > m->cap) return set_error(SHT_EINVAL, "sht_mlp_train_step: batch outside 1 .. capacity");
    DevGuard dg(m->device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = backward(m, x, y, B, s);
    // Adam
    ++m->step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)m->step), c2 = 1.f - std::pow(b2, (float)m->step);
    if (e == cudaSuccess) {
        AdamSet set{};
        int64_t total = 0;
        for (int l = 0; l < 4; ++l) {
            const int64_t nw = (int64_t)m->fan_out[l] * m->fan_in[l];
            set.w[2 * l] = m->W[l];
            set.g[2 * l] = m->dW[l];
            set.m[2 * l] = m->mW[l];
            set.v[2 * l] = m->vW[l];
            set.wb[2 * l] = m->Wb[l];
            set.end[2 * l] = (total += nw);
            set.w[2 * l + 1] = m->b[l];
            set.g[2 * l + 1] = m->db[l];
            set.m[2 * l + 1] = m->mb[l];
            set.v[2 * l + 1] = m->vb[l];
            set.wb[2 * l + 1] = nullptr;
            set.end[2 * l + 1] = (total += m->fan_out[l]);
        }
        set.count = 8;
        adam_multi_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(set, lr, b1, b2, c1, c2, 1e-8f);
        e = cudaGetLastError();
    }
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_mlp_train_step");
}

int sht_mlp_infer(sht_mlp* m, const float* x, float* y, int B, void* stream) {
    if (!m || !x || !y) return set_error(SHT_EINVAL, "sht_mlp_infer: NULL argument");
    if (B < 0 || B > m->cap) return set_error(SHT_EINVAL, "sht_mlp_infer: batch outside 0 .. capacity");
    if (B == 0) return SHT_OK;
    DevGuard dg(m->device);
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t nx = (int64_t)B * m->in_pad;
    normalize_in_kernel<<<(unsigned)((nx + 255) / 256), 256, 0, s>>>(x, m->nin, B, m->nin, m->xm, m->xs, m->X0,
                                                                     m->in_pad);
    cudaError_t e = forward(m, B, false, s);
    const int64_t ny = (int64_t)B * m->nout;
    if (e == cudaSuccess)
        denormalize_kernel<<<(unsigned)((ny + 255) / 256), 256, 0, s>>>(m->Y, B, m->nout, m->ym, m->ys, y, m->nout);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_mlp_infer");
}

int sht_mlp_loss(sht_mlp* m, float* loss) {
    if (!m || !loss) return set_error(SHT_EINVAL, "sht_mlp_loss: NULL argument");
    DevGuard dg(m->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(loss, m->loss, 4, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_mlp_loss");
}

int sht_mlp_params(sht_mlp* m, int layer, float* w, float* b, int set) {
    if (!m || layer < 0 || layer >= 4) return set_error(SHT_EINVAL, "sht_mlp_params: bad layer");
    if (set < 0 || set > 2) return set_error(SHT_EINVAL, "sht_mlp_params: mode must be 0 (get), 1 (set) or 2 (gradients)");
    DevGuard dg(m->device);
    const size_t nw = (size_t)m->fan_out[layer] * m->fan_in[layer];
    cudaError_t e = cudaSuccess;
    if (set == 2) {            // gradients of the last backward pass
        e = cudaDeviceSynchronize();
        if (e == cudaSuccess && w) e = cudaMemcpy(w, m->dW[layer], nw * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && b) e = cudaMemcpy(b, m->db[layer], m->fan_out[layer] * 4, cudaMemcpyDeviceToHost);
    } else if (set) {
        if (w) e = cudaMemcpy(m->W[layer], w, nw * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && b) e = cudaMemcpy(m->b[layer], b, m->fan_out[layer] * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) to_bf16_kernel<<<(unsigned)((nw + 255) / 256), 256>>>(m->W[layer], m->Wb[layer], nw);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    } else {
        if (w) e = cudaMemcpy(w, m->W[layer], nw * 4, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && b) e = cudaMemcpy(b, m->b[layer], m->fan_out[layer] * 4, cudaMemcpyDeviceToHost);
    }
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_mlp_params");
}

int sht_column_emulate(sht_mlp* m, const float* temp, const float* humid, const float* u, const float* v,
                       const float* surface_pressure, int64_t ld, int ncol, double dt, double z_max, float* dtemp,
                       float* dhumid, unsigned flags, int32_t* nfallback, void* stream) {
    if (!m || !temp || !humid || !u || !v || !surface_pressure || !dtemp || !dhumid)
        return set_error(SHT_EINVAL, "sht_column_emulate: NULL argument");
    if (ncol < 0 || ld < ncol) return set_error(SHT_EINVAL, "sht_column_emulate: DimensionMismatch: ld < ncol");
    if (ncol == 0) return SHT_OK;
    DevGuard dg(m->device);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = fused_attributes();
    // the fallback count only when asked for (it synchronises the stream)
    if (e == cudaSuccess && nfallback) e = cudaMemsetAsync(m->nfallback, 0, 4, s);
    if (e == cudaSuccess) {
        FusedArgs fa{};
        fa.T = temp;
        fa.q = humid;
        fa.u = u;
        fa.v = v;
        fa.ps = surface_pressure;
        fa.ld = ld;
        fa.ncol = ncol;
        fa.xm = m->xm;
        fa.xs = m->xs;
        fa.ym = m->ym;
        fa.ys = m->ys;
        for (int l = 0; l < 4; ++l) fa.bias[l] = m->b[l];
        fa.zmax = (float)z_max;
        fa.dt = (float)dt;
        fa.L = column_levels();
        fa.dT = dtemp;
        fa.dq = dhumid;
        fa.add = (flags & SHT_ADD) ? 1 : 0;
        fa.nfallback = nfallback ? m->nfallback : nullptr;
        fa.err = m->err;
        // one CTA per SM when the columns allow it (at most 128 per CTA: the MMA tile's rows)
        int nsm = 148;
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device) != cudaSuccess || nsm < 1) nsm = 148;
        fa.cpb = std::min(128, std::max(1, (ncol + nsm - 1) / nsm));
        mlp_fused_kernel<<<(ncol + fa.cpb - 1) / fa.cpb, F_THREADS, F_SMEM, s>>>(m->wmap[0], m->wmap[1], m->wmap[2],
                                                                               m->wmap[3], fa);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && nfallback) {
        e = cudaMemcpyAsync(nfallback, m->nfallback, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_column_emulate");
}

int sht_mlp_device_status(sht_mlp* m, int32_t* status) {
    if (!m || !status) return set_error(SHT_EINVAL, "sht_mlp_device_status: NULL argument");
    DevGuard dg(m->device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(status, m->err, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, 4);
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_mlp_device_status");
}

int sht_mlp_destroy(sht_mlp* m) {
    if (!m) return SHT_OK;
    DevGuard dg(m->device);
    release(m);
    delete m;
    return SHT_OK;
}

// A general BF16 matrix product on the tensor cores (the MLP's building block):
// C [M][ldc] FP32 = A B, A [M][K] (a_mn = 0: stored [M][lda]; 1: stored [K][lda]) and
// B [K][N] (b_mn = 0: stored [N][ldb]; 1: stored [K][ldb]); leading dimensions in elements,
// multiples of 8.
int sht_bf16_gemm(const void* A, int64_t lda, int a_mn, const void* B, int64_t ldb, int b_mn, float* C, int64_t ldc,
                  int M, int N, int K, int32_t* device_error, void* stream) {
    if (!A || !B || !C || !device_error) return set_error(SHT_EINVAL, "sht_bf16_gemm: NULL argument");
    if (M < 0 || N < 0 || K < 0 || ldc < N || (lda % 8) || (ldb % 8))
        return set_error(SHT_EINVAL, "sht_bf16_gemm: DimensionMismatch: sizes or leading dimensions");
    GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.epi = EPI_F32;
    g.out_f32 = C;
    g.ld_f32 = ldc;
    g.err = device_error;
    const cudaError_t e = gemm((const __nv_bfloat16*)A, lda, a_mn, (const __nv_bfloat16*)B, ldb, b_mn, g,
                               (cudaStream_t)stream);
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_bf16_gemm");
}
