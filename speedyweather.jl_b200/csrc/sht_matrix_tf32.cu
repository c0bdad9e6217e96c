// Dense-matrix products of the FP32 MatrixSpectralTransform on the tensor cores, as
// three TF32 products (tcgen05.mma kind::tf32) with FP32 accumulation.
//
// Replaces the Float32 mul! of SpeedyTransforms/src/matrix_transform.jl:206-258:
//   out[n][row] = sum_d A[row][d] in[n][d]     (n < K layers, row < M, d < depth)
// with A the analysis matrix (rows = real/imaginary parts of the coefficients, depth =
// grid points) or the synthesis matrix (rows = grid points, depth = the coefficients
// viewed as floats).
//
// Precision. x = hi + lo with hi = tf32(x) and lo = tf32(x - hi) (round to nearest;
// 11-bit significands each, so hi + lo carries 22 bits of x). The product is
//   A_hi B_hi + (A_hi B_lo + A_lo B_hi)
// (A_lo B_lo, 2^-22 of the product, is left out). B = [B_hi; B_lo] is stacked along N,
// so one MMA of A_hi against it writes the leading product to columns [0, NP) and
// A_hi B_lo to [NP, 2 NP); a second MMA adds A_lo B_hi to the latter. The tensor core
// truncates each update of its FP32 accumulator toward zero; the leading accumulator
// therefore only sums one 128-deep chunk (16 updates) before the drain warps read it
// and add it, with the cross accumulator, to FP32 registers with rounding to nearest.
//
// Data flow. The matrix is stored once, at creation, as FP32 tiles of 128 rows x 32
// deep (16 KB) in the SWIZZLE_128B K-major layout the MMA reads, in the order
// (row tile, k-block): a CTA's range of k-blocks is one contiguous run of bytes, read
// from HBM once by 1-D bulk copies. Four converter warps split each tile in shared
// memory: hi in place, lo into a second buffer (the MMA needs TF32 values). A small
// pre-pass per call writes the layers' pieces [B_hi; B_lo] as one swizzled tile per
// k-block in the same way.
//
// Work split (stream-K): the M / 128 row tiles times depth / 32 k-blocks are cut into
// G equal contiguous ranges, one per CTA (G <= the SM count), so every SM streams the
// same number of matrix bytes whatever the shape. A CTA writes the sums of each row tile
// it touches to a partial slot; a second kernel, one thread per output, adds a tile's
// partials in CTA order, scales the rows and writes the output. The order of every
// addition is fixed, so results are bitwise reproducible.
//
// Roles: warp 0 issues the copies, warp 1 allocates the tensor memory and issues the
// MMAs, warps 2-5 split the tiles, warps 6-9 drain the accumulators. Every wait is
// bounded (one second); on expiry the CTA records an error in the status word, stops,
// waits for its copies in flight and for its MMAs, and frees its tensor memory.
#include <algorithm>
#include <vector>

#include "sht_internal.h"
#include "tc_ptx.cuh"

namespace sht {

namespace {

using namespace tcx;

constexpr int MX_THREADS = 320;
constexpr int MX_DEPTH = 32;              // depth per k-block: 128 bytes of FP32 per row
constexpr int MX_ROWS = 128;              // matrix rows per tile (MMA M)
constexpr int MX_CHUNK = 4;               // k-blocks per accumulator fill (16 leading-sum updates)
constexpr int MX_A_BYTES = MX_ROWS * 128; // 16 KB
constexpr int MX_SMEM = 227 * 1024;
constexpr int MX_MAX_STAGES = 8;

struct MxArgs {
    const float* a_img;        // [mtiles KB][128][32] FP32, swizzled tiles
    const float* b_img;        // [ct][KB][2 NP][32] TF32 pieces, swizzled tiles
    int M, KB, mtiles, K;
    int64_t W;                 // mtiles x KB k-blocks
    int G;                     // CTAs (gridDim.x)
    int S;                     // partial slots per CTA
    int stages;
    float* part;               // [ct][G][S][NP][128]
    float* out;
    int64_t ldo;
    const float* row_scale;    // per output row, or nullptr (the reduction's arguments)
    int32_t* err;
};

__device__ __forceinline__ float tf32_rna(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
// tf32(x) rounded to nearest, ties away from zero, on the integer pipe: add half a unit
// of the 11-bit significand's last place to the magnitude bits and clear the 13 low
// bits (the carry moves into the exponent where it must); finite x.
__device__ __forceinline__ float tf32_int(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// First k-block of CTA c, and the CTA whose range holds k-block w (ranges are non-empty
// when G <= W).
__host__ __device__ __forceinline__ int64_t range_begin(int64_t c, int64_t W, int G) { return c * W / G; }
__device__ __forceinline__ int cta_of(int64_t w, int64_t W, int G) { return (int)(((w + 1) * G - 1) / W); }

// Chunks of up to MX_CHUNK k-blocks that never cross a row tile; the roles all walk the
// CTA's range [w0, w1) in the same chunks.
struct Walk {
    int64_t w0, w1;
    int KB;
    __device__ int64_t chunk_end(int64_t w) const {
        const int64_t tile_end = (w / KB + 1) * KB;
        return min(min(w + MX_CHUNK, tile_end), w1);
    }
};

template <int NP>
__global__ void __launch_bounds__(MX_THREADS, 1) matrix_tf32_kernel(const MxArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    constexpr int B_BYTES = 2 * NP * 128;
    constexpr int STAGE = 2 * MX_A_BYTES + B_BYTES;
    constexpr uint32_t SET_COLS = 2 * NP;
    constexpr int NSETS = 512 / (2 * NP);   // accumulator sets filling the 512 TMEM columns
    const int stages = a.stages;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int ct = blockIdx.y;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)stages * STAGE);   // copies landed
    uint64_t* empty = full + MX_MAX_STAGES;                                          // stage's MMAs done
    uint64_t* conv = empty + MX_MAX_STAGES;                                          // stage split
    uint64_t* setf = conv + MX_MAX_STAGES;                                           // set filled
    uint64_t* sete = setf + 16;                                                      // set drained
    uint64_t* fin = sete + 16;                                                       // all MMAs done
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

    Walk wk;
    wk.KB = a.KB;
    wk.w0 = range_begin(blockIdx.x, a.W, a.G);
    wk.w1 = range_begin(blockIdx.x + 1, a.W, a.G);

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
            mbar_init(&conv[s], 4);
        }
        for (int s = 0; s < NSETS; ++s) {
            mbar_init(&setf[s], 1);
            mbar_init(&sete[s], 4);
        }
        mbar_init(fin, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(512u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------ copies
        int g = 0;
        for (int64_t w = wk.w0; w < wk.w1 && !*abort_flag; ++w, ++g) {
            const int s = g % stages;
            if (g >= stages && !mbar_wait(&empty[s], ((g / stages) - 1) & 1)) {
                *abort_flag = 1;
                atomicExch(a.err, 11);
                break;
            }
            uint8_t* st = smem + (size_t)s * STAGE;
            const int kb = (int)(w % a.KB);
            mbar_expect_tx(&full[s], (uint32_t)(MX_A_BYTES + B_BYTES));
            bulk_load(st, a.a_img + w * (MX_A_BYTES / 4), MX_A_BYTES, &full[s]);
            bulk_load(st + 2 * MX_A_BYTES, a.b_img + ((int64_t)ct * a.KB + kb) * (B_BYTES / 4), B_BYTES, &full[s]);
        }
        // no copy may still be landing in shared memory when the CTA exits
        for (int u = g - 1; u >= 0 && u >= g - stages; --u)
            if (!mbar_wait(&full[u % stages], (u / stages) & 1)) atomicExch(a.err, 15);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------ MMAs
        const uint32_t id2 = idesc_f16(2u, 0u, 0u, 2 * NP);   // TF32: A_hi x [B_hi; B_lo]
        const uint32_t id1 = idesc_f16(2u, 0u, 0u, NP);       // TF32: A_lo x B_hi
        int g = 0, ci = 0;
        bool ok = true;
        for (int64_t w = wk.w0; w < wk.w1 && ok && !*abort_flag;) {
            const int64_t we = wk.chunk_end(w);
            const int set = ci % NSETS;
            if (ci >= NSETS && !mbar_wait(&sete[set], ((ci / NSETS) - 1) & 1)) {
                *abort_flag = 1;
                atomicExch(a.err, 14);
                break;
            }
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)set * SET_COLS;
            const int64_t wc = w;                  // the chunk's first k-block starts a fresh fill
            for (; w < we; ++w, ++g) {
                const int s = g % stages;
                if (!mbar_wait(&conv[s], (g / stages) & 1)) {
                    *abort_flag = 1;
                    atomicExch(a.err, 12);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t hi = smem_u32(smem + (size_t)s * STAGE);
                const uint32_t lo = hi + MX_A_BYTES, bb = hi + 2 * MX_A_BYTES;
                for (int kk = 0; kk < MX_DEPTH / 8; ++kk) {       // 8 deep (32 bytes) per MMA
                    const uint64_t db = sdesc(bb + kk * 32, 16, 1024);
                    umma_tf32(d, sdesc(hi + kk * 32, 16, 1024), db, id2, (w == wc && kk == 0) ? 0u : 1u);
                    umma_tf32(d + NP, sdesc(lo + kk * 32, 16, 1024), db, id1, 1u);
                }
                umma_commit(&empty[s]);
            }
            if (!ok) break;
            umma_commit(&setf[set]);
            ++ci;
        }
        // every MMA must be complete before the tensor memory is released
        umma_commit(fin);
        if (!mbar_wait(fin, 0)) atomicExch(a.err, 16);
    } else if (warp >= 2 && warp < 6) {
        // ------------------------------------------------ split into TF32 pieces
        const int c = threadIdx.x - 64;
        int g = 0;
        for (int64_t w = wk.w0; w < wk.w1; ++w, ++g) {
            const int s = g % stages;
            const bool got = __all_sync(0xffffffffu, mbar_wait(&full[s], (g / stages) & 1));
            if (!got || *abort_flag) {
                *abort_flag = 1;
                if (!got) atomicExch(a.err, 13);
                break;
            }
            float4* x = reinterpret_cast<float4*>(smem + (size_t)s * STAGE);
            float4* y = reinterpret_cast<float4*>(smem + (size_t)s * STAGE + MX_A_BYTES);
#pragma unroll
            for (int j = 0; j < MX_A_BYTES / 16 / 128; ++j) {
                const int i = c + 128 * j;
                const float4 v = x[i];
                float4 h, l;
                h.x = tf32_int(v.x); l.x = tf32_int(v.x - h.x);
                h.y = tf32_int(v.y); l.y = tf32_int(v.y - h.y);
                h.z = tf32_int(v.z); l.z = tf32_int(v.z - h.z);
                h.w = tf32_int(v.w); l.w = tf32_int(v.w - h.w);
                x[i] = h;
                y[i] = l;
            }
            fence_proxy_async();           // the MMA reads these through the async proxy
            __syncwarp();
            if (lane == 0) mbar_arrive(&conv[s]);
        }
    } else if (warp >= 6) {
        // ------------------------------------------------ drain
        const int quarter = warp % 4;
        const int r = quarter * 32 + lane;
        const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
        float acc[NP];
#pragma unroll
        for (int n = 0; n < NP; ++n) acc[n] = 0.f;
        int ci = 0;
        const int t0 = (int)(wk.w0 / a.KB);
        for (int64_t w = wk.w0; w < wk.w1; ++ci) {
            const int64_t we = wk.chunk_end(w);
            const int set = ci % NSETS;
            // warp-uniform outcome: tcgen05.ld below is a warp-collective instruction
            if (*abort_flag || !__all_sync(0xffffffffu, mbar_wait(&setf[set], (ci / NSETS) & 1))) {
                *abort_flag = 1;
                atomicExch(a.err, 17);
                break;
            }
            tc_fence_after();
            const uint32_t ta = tmem + (uint32_t)set * SET_COLS + lane_off;
            if (NP == 16) {
                float v[32];
                tmem_ld32(ta, v);
#pragma unroll
                for (int n = 0; n < 16; ++n) acc[n] = __fadd_rn(acc[n], __fadd_rn(v[n], v[16 + n]));
            } else {
#pragma unroll
                for (int h = 0; h < NP / 32; ++h) {
                    float v[32], x[32];
                    tmem_ld32(ta + h * 32, v);
                    tmem_ld32(ta + NP + h * 32, x);
#pragma unroll
                    for (int n = 0; n < 32; ++n) acc[h * 32 + n] = __fadd_rn(acc[h * 32 + n], __fadd_rn(v[n], x[n]));
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&sete[set]);
            w = we;
            if (w != wk.w1 && w % a.KB != 0) continue;
            // this CTA's part of row tile (w - 1) / KB is complete: its partial slot
            float* slot = a.part + ((((int64_t)ct * a.G + blockIdx.x) * a.S + ((w - 1) / a.KB - t0)) * NP) * 128;
#pragma unroll
            for (int n = 0; n < NP; ++n) {
                slot[n * 128 + r] = acc[n];
                acc[n] = 0.f;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u) : "memory");
    }
}

// out[n ldo + row] = row_scale[row] x the sum, in CTA order, of the partial slots of the
// CTAs whose ranges cover row tile t = blockIdx.x (layer n = blockIdx.y, row t 128 + thread).
template <int NP>
__global__ void __launch_bounds__(128) mx_reduce_kernel(const MxArgs a) {
    const int t = blockIdx.x, n = blockIdx.y, ct = n / NP, nl = n % NP;
    const int row = t * MX_ROWS + threadIdx.x;
    if (row >= a.M) return;
    const int cf = cta_of((int64_t)t * a.KB, a.W, a.G), cl = cta_of((int64_t)t * a.KB + a.KB - 1, a.W, a.G);
    auto slot = [&](int c) {
        const int tc0 = (int)(range_begin(c, a.W, a.G) / a.KB);
        return a.part[((((int64_t)ct * a.G + c) * a.S + (t - tc0)) * NP + nl) * 128 + threadIdx.x];
    };
    float s = slot(cf);
    int c = cf + 1;
    for (; c + 3 <= cl; c += 4) {          // four independent loads in flight, added in order
        const float v0 = slot(c), v1 = slot(c + 1), v2 = slot(c + 2), v3 = slot(c + 3);
        s = __fadd_rn(__fadd_rn(__fadd_rn(__fadd_rn(s, v0), v1), v2), v3);
    }
    for (; c <= cl; ++c) s = __fadd_rn(s, slot(c));
    a.out[(int64_t)n * a.ldo + row] = a.row_scale ? __fmul_rn(s, a.row_scale[row]) : s;
}

// Offset (in floats) of element (row, col) of a tile of 128-byte rows in the
// SWIZZLE_128B layout: the 16-byte chunk col / 4 of row r sits at chunk (col / 4) ^ (r % 8).
__device__ __forceinline__ int swz(int row, int col) { return row * 32 + ((((col >> 2) ^ row) & 7) << 2) + (col & 3); }

// The matrix in[d][m] (depth x M, M contiguous) as swizzled tiles out[t KB + kb][row][col]
// = in[kb 32 + col][t 128 + row] (zero outside). Block: tile (t, kb), 32 of its rows.
__global__ void matrix_tiles_kernel(const float* __restrict__ in, int depth, int M, int KB, float* __restrict__ out) {
    __shared__ float tile[32][33];
    const int kb = blockIdx.x, t = blockIdx.y / 4, r0 = (blockIdx.y % 4) * 32;
    for (int c = threadIdx.y; c < 32; c += 8) {      // coalesced along m
        const int d = kb * 32 + c, m = t * MX_ROWS + r0 + threadIdx.x;
        tile[c][threadIdx.x] = d < depth && m < M ? in[(int64_t)d * M + m] : 0.f;
    }
    __syncthreads();
    float* o = out + ((int64_t)t * KB + kb) * (MX_ROWS * 32);
    for (int r = threadIdx.y; r < 32; r += 8) o[swz(r0 + r, threadIdx.x)] = tile[threadIdx.x][r];
}

// The layers of one call as TF32 pieces in swizzled tiles: tile (ct, kb), row p NP + nl
// holds piece p (0: hi = tf32(x), 1: lo = tf32(x - hi)) of x = in[(ct NP + nl) ld + d],
// zero for layers >= K or d >= depth; layers < gridDim.y.
__global__ void layer_pieces_kernel(const float* __restrict__ in, int64_t ld, int depth, int K, int NP, int KB,
                                    float* __restrict__ img) {
    const int n = blockIdx.y, ct = n / NP, nl = n % NP;
    for (int d = blockIdx.x * blockDim.x + threadIdx.x; d < KB * 32; d += gridDim.x * blockDim.x) {
        const float x = n < K && d < depth ? __ldg(in + (int64_t)n * ld + d) : 0.f;
        const float h = tf32_rna(x);
        float* o = img + ((int64_t)ct * KB + d / 32) * (2 * NP * 32);
        o[swz(nl, d % 32)] = h;
        o[swz(NP + nl, d % 32)] = tf32_rna(x - h);
    }
}

int stages_for(int np) {
    const int stage = 2 * MX_A_BYTES + 2 * np * 128;
    return std::min(MX_MAX_STAGES, (MX_SMEM - 2048) / stage);
}
int smem_for_np(int np) { return stages_for(np) * (2 * MX_A_BYTES + 2 * np * 128) + 2048; }

}  // namespace

struct MxDir {
    int M = 0, depth = 0, KB = 0, mtiles = 0, G = 0, S = 0;
    int64_t W = 0;
    float* d_a = nullptr;            // [mtiles KB][128][32] swizzled tiles
    float* d_img = nullptr;          // [ctiles][KB][2 np][32] swizzled tiles
    float* d_part = nullptr;         // [ctiles][G][S][np][128]
};

struct MxTf32 {
    int np = 16, ctiles = 1, nlayers = 0, nsm = 148;
    MxDir dir[2];                    // 0: analysis, 1: synthesis
};

void mx_tf32_destroy(MxTf32* x) {
    if (!x) return;
    for (auto& m : x->dir) {
        void* ptrs[] = {m.d_a, m.d_img, m.d_part};
        for (void* q : ptrs)
            if (q) cudaFree(q);
    }
    delete x;
}

// a[d]: the matrix of direction d as [depth][M] (M contiguous), FP32, on the device.
cudaError_t mx_tf32_create(MxTf32** out, const float* const a[2], const int depth[2], const int M[2], int nlayers) {
    MxTf32* x = new MxTf32();
    *out = x;
    x->nlayers = nlayers;
    x->np = nlayers <= 16 ? 16 : nlayers <= 32 ? 32 : 64;
    x->ctiles = (nlayers + x->np - 1) / x->np;
    {
        int dev = 0, nsm = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && nsm > 0)
            x->nsm = nsm;
    }
    cudaError_t e;
    for (int d = 0; d < 2; ++d) {
        MxDir& m = x->dir[d];
        m.M = M[d];
        m.depth = depth[d];
        m.KB = (depth[d] + MX_DEPTH - 1) / MX_DEPTH;
        m.mtiles = (M[d] + MX_ROWS - 1) / MX_ROWS;
        m.W = (int64_t)m.mtiles * m.KB;
        m.G = (int)std::max<int64_t>(1, std::min<int64_t>(x->nsm, m.W / 4));
        for (int c = 0; c < m.G; ++c) {                   // row tiles a CTA's range touches
            const int64_t w0 = range_begin(c, m.W, m.G), w1 = range_begin(c + 1, m.W, m.G);
            m.S = std::max<int>(m.S, (int)((w1 - 1) / m.KB - w0 / m.KB + 1));
        }
        if ((e = cudaMalloc(&m.d_a, (size_t)m.W * MX_A_BYTES)) != cudaSuccess) return e;
        matrix_tiles_kernel<<<dim3(m.KB, m.mtiles * 4), dim3(32, 8)>>>(a[d], m.depth, m.M, m.KB, m.d_a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const size_t img = (size_t)x->ctiles * m.KB * 2 * x->np * 32 * sizeof(float);
        if ((e = cudaMalloc(&m.d_img, img)) != cudaSuccess) return e;
        if ((e = cudaMemset(m.d_img, 0, img)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&m.d_part, (size_t)x->ctiles * m.G * m.S * x->np * 128 * sizeof(float))) != cudaSuccess)
            return e;
    }
    const int smem = smem_for_np(x->np);
    if (x->np == 16)
        e = cudaFuncSetAttribute(matrix_tf32_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    else if (x->np == 32)
        e = cudaFuncSetAttribute(matrix_tf32_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    else
        e = cudaFuncSetAttribute(matrix_tf32_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaDeviceSynchronize();
}

// out[n ldo + row] = sum_d A[row][d] in[n ld + d] (times row_scale[row]) for n < K:
// three launches (the layers' pieces, the products, the reduction of the partials).
cudaError_t mx_tf32_apply(const MxTf32* x, int which, const float* in, int64_t ld, float* out, int64_t ldo, int K,
                          const float* row_scale, int32_t* d_err, cudaStream_t st) {
    const MxDir& m = x->dir[which];
    if (K <= 0 || K > x->nlayers) return cudaErrorInvalidValue;
    const int ct = (K + x->np - 1) / x->np;
    layer_pieces_kernel<<<dim3(std::min(64, (m.KB * MX_DEPTH + 255) / 256), ct * x->np), 256, 0, st>>>(
        in, ld, m.depth, K, x->np, m.KB, m.d_img);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    MxArgs a{};
    a.a_img = m.d_a;
    a.b_img = m.d_img;
    a.M = m.M;
    a.KB = m.KB;
    a.mtiles = m.mtiles;
    a.K = K;
    a.W = m.W;
    a.G = m.G;
    a.S = m.S;
    a.stages = stages_for(x->np);
    a.part = m.d_part;
    a.out = out;
    a.ldo = ldo;
    a.row_scale = row_scale;
    a.err = d_err;
    const dim3 grid(m.G, ct), rgrid(m.mtiles, K);
    const int smem = smem_for_np(x->np);
    if (x->np == 16) {
        matrix_tf32_kernel<16><<<grid, MX_THREADS, smem, st>>>(a);
        mx_reduce_kernel<16><<<rgrid, 128, 0, st>>>(a);
    } else if (x->np == 32) {
        matrix_tf32_kernel<32><<<grid, MX_THREADS, smem, st>>>(a);
        mx_reduce_kernel<32><<<rgrid, 128, 0, st>>>(a);
    } else {
        matrix_tf32_kernel<64><<<grid, MX_THREADS, smem, st>>>(a);
        mx_reduce_kernel<64><<<rgrid, 128, 0, st>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace sht
