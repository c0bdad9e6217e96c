// Legendre stage on the 5th-generation tensor cores (tcgen05) in split precision.
//
// Replaces SpeedyTransforms/src/legendre_ka.jl:19-200 (and the CPU loops of
// SpeedyTransforms/src/legendre.jl:2-195) for plans with SHT_PREC_BF16X3 / SHT_PREC_BF16X5.
//
// Per order m and parity p of l - m the stage is one GEMM (see sht_legendre_simt.cu):
//   synthesis  D[j, c] = sum_i Lam[m][p][i][j] B[i, c]     (M = rings, K = parity rows)
//   analysis   D[i, c] = sum_j Lam[m][p][i][j] B[j, c]     (M = parity rows, K = rings)
// FP32 operands are split into 16-bit pieces x = x_0 + x_1 (+ x_2) and the product
// is the sum of the cross products whose magnitude is above the split's residual,
// accumulated in FP32 in tensor memory:
//   SHT_PREC_BF16X3: Lam in 2 bf16 pieces, data in 2: L0 B0 + L0 B1 + L1 B0
//   SHT_PREC_BF16X5: Lam in 3 bf16 pieces (from FP64), data in 2:
//                    L0 B0 + L0 B1 + L1 B0 + L1 B1 + L2 B0
//   SHT_PREC_FP16X3: as BF16X3 with fp16 pieces (11-bit significands), Lam scaled by
//                    2^(15 - e_m) per order and the data by 2^(15 - e) with e from
//                    the max-abs of the call's input: per order and layer for the
//                    synthesis (reduced by the image kernel), per layer for the analysis
//                    (a pass over the grid), so that the largest values sit in
//                    [2^14, 2^15): both pieces stay normal fp16 numbers down to 2^-18 of
//                    the maximum, and the products stay far inside FP32's range. The
//                    epilogue multiplies by 2^(e_m + e - 30), which is exact.
//
// Operands in shared memory use the SWIZZLE_128B canonical layouts of tcgen05:
// * Lam[m][p] is stored [piece][i][j - j0(m)] in global memory; one TMA tensor map
//   per (m, p) loads 64 x 64 boxes (rows i, 128 B of j). The same box is the
//   MN-major A block of the synthesis (M = j) and the K-major A block of the
//   analysis (K = j). Out-of-range parts of a box are zero-filled by the TMA without
//   memory traffic.
// * The data operands are written by their producers (a pre-pass over the
//   coefficients for the synthesis, the FFT kernel for the analysis) directly as
//   swizzled shared-memory images in global memory and loaded with 1-D bulk copies.
//
// A persistent CTA per SM computes a sequence of 128 x N output tiles (N <= 128 real
// columns for the transforms, <= 256 for dense matrices): warp 0 issues the copies,
// warp 1 owns the tensor memory and one of its threads issues the MMAs, warps 2-9 (two
// per TMEM lane quarter) read the accumulator (tcgen05.ld) and store while the next
// tile accumulates.
//
// Accumulation. The tensor core adds each MMA's products to its FP32 accumulator with
// truncation, not rounding to nearest: every update loses on average half a unit in
// the last place of the accumulator, always toward zero. Over the long same-sign sums
// of the transforms (the l = 0 coefficient sums all rings; the synthesis of a field
// with a large mean sums the same sign over l) these losses add up to a bias (measured
// at T511: the a_00 error pointed toward zero in 98 % of layers, and made up ~70 % of
// the squared error of every split form). The transforms therefore give each tile two
// accumulators: one for the leading product (piece 0 x piece 0) and one for all the
// cross products, which are 2^-8 (bf16) or 2^-11 (fp16) smaller, so their truncation
// is negligible; the epilogue adds the two in FP32 with rounding to nearest. The large
// accumulator then takes one update per 16-deep step instead of 3 (5 for BF16X5). The CTA's items are read into shared memory once. Every wait is
// bounded by a one-second global-timer limit; on expiry the CTA records an error
// in the plan's status word, drains, frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "sht_internal.h"
#include "tc_ptx.cuh"

namespace sht {

namespace {

constexpr int TC_THREADS = 320;     // producer warp, MMA warp, 8 epilogue warps
constexpr int BLK = 64;                     // Legendre box edge (rows x rings)
constexpr int BOX_BYTES = BLK * BLK * 2;    // 8 KB
constexpr int A_PIECE_BYTES = 2 * BOX_BYTES;
// Column tile of the transforms' GEMMs: two buffers of two accumulators of up to 128
// FP32 columns fill the 512 columns of tensor memory.
constexpr int kTcTileCols = 128;

struct TcItem {
    int32_t m, par, tile, pad;
};

// Everything the kernels need, passed by value.
struct TcDev {
    const CUtensorMap* maps;       // per (m, par)
    const int32_t* nr;             // per m: rings [j0, nh)
    const int32_t* j0;             // per m
    const int32_t* rows;           // per m: parity rows
    const int64_t* lm_off;         // per m
    const int64_t* syn_tile_base;  // per m: image tile index of (m, par 0, kt 0)
    const int64_t* ana_tile_base;  // per m
    const int32_t* nkt;            // per m: ceil(rows / 64)
    const int32_t* njt;            // per m: ceil(nr / 64)
    const RingDesc* rings;
    const uint16_t* syn_img;
    const uint16_t* ana_img;
    int32_t* err;
    int nh, lmax, mmax;
    int npa, npb, nprod;
    uint32_t prod;                 // product i: A piece (prod >> 4i) & 3, B piece (prod >> (4i + 2)) & 3
    int64_t syn_tile_bytes;        // one (m, p, kt, piece) synthesis data tile at nmax columns
    int64_t ana_tile_bytes;        // one (m, p, jt, piece) analysis data tile
    int nmax;                      // columns of the data images (multiple of 64)
    int fp16;                      // 1: fp16 pieces with power-of-two scaling
    const int32_t* mexp;           // per m: e_m of the Legendre scaling
    const float2* kscale_syn;      // per layer: (2^(e_k - 15), 2^(15 - e_k)) of the dense-matrix input
    float2* mkscale_syn;           // per (m, layer), [m K + k]: the same for the synthesis input of order m
    const float2* kscale_ana;      // per layer: the same for the analysis data (E, O)
    // dense matrix transforms (MatrixSpectralTransform): one "order" m = 0 whose A operand
    // is the matrix; the epilogue writes out[n ldo + row] for the K layer columns n
    int matrix;
    int mrows;                     // rows of the matrix (output length per layer)
    float* mout;
    int64_t ldo;
    const float* row_scale;        // per output row (1 / cos lat of its ring) or nullptr
    int kchunk;                    // > 0: accumulate the depth in chunks of kchunk 64-deep blocks,
                                   // each on a fresh accumulator, summed in FP32 by the epilogue
};

struct TcState {
    int ctw = kTcTileCols;         // column tile width of the transforms' GEMMs (64 or 128; autotuned)
    int npa = 2, npb = 2, nprod = 3;
    uint32_t prod = 0;
    int nmax = 0;
    CUtensorMap* d_maps = nullptr;
    uint16_t* d_lam = nullptr;
    int32_t *d_nr = nullptr, *d_nkt = nullptr, *d_njt = nullptr;
    int64_t *d_syn_base = nullptr, *d_ana_base = nullptr;
    uint16_t* d_syn_img = nullptr;
    uint16_t* d_ana_img = nullptr;
    int64_t syn_tile_bytes = 0, ana_tile_bytes = 0;
    TcItem* d_syn_items = nullptr;
    int n_syn_items = 0;
    TcItem* d_ana_items = nullptr;
    int n_ana_items = 0;
    int max_smem = 0;
    int nsm = 148;                 // SMs of the device (persistent grid)
    int fp16 = 0;
    int32_t* d_mexp = nullptr;
    float* d_absmax = nullptr;     // [2 nlayers]: the analysis input's max-abs in [nlayers, 2 nlayers)
                                   // (the synthesis image kernel reduces its own per order and layer)
    float2* d_kscale = nullptr;    // [2 nlayers]: (2^(e_k - 15), 2^(15 - e_k)) per layer, analysis half used
    float2* d_mkscale = nullptr;   // [mmax][nlayers]: the same per order and layer (synthesis input)
    float ana_mul = 0.f;
};

using namespace tcx;

constexpr int F16_TOP = 15;        // fp16 data scaled to [2^14, 2^15) of its maximum

// Exponent e with |bound| 2^-e < 1 (0 for a zero bound).
__device__ __forceinline__ int scale_exp(float bound) {
    int e = 0;
    if (bound > 0.f) frexpf(bound, &e);
    return e;
}
// 16-bit pieces of x (bf16 or fp16), x = sum of the pieces to ~8 or ~11 bits each.
template <bool F16>
__device__ __forceinline__ uint32_t piece_bits(float& r) {
    if (F16) {
        const __half h = __float2half_rn(r);
        r -= __half2float(h);
        return __half_as_ushort(h);
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(r);
    r -= __bfloat162float(h);
    return __bfloat16_as_ushort(h);
}
// The next pieces of two reals r0 (low half) and r1 (high half) with one paired rounding
// (the same bits as piece_bits on each); the residuals are formed only when another piece
// follows.
template <bool F16, bool RESIDUAL>
__device__ __forceinline__ uint32_t piece_bits2(float& r0, float& r1) {
    if (F16) {
        const __half2 h = __floats2half2_rn(r0, r1);
        if (RESIDUAL) {
            const float2 b = __half22float2(h);
            r0 -= b.x;
            r1 -= b.y;
        }
        return *reinterpret_cast<const uint32_t*>(&h);
    }
    const __nv_bfloat162 h = __floats2bfloat162_rn(r0, r1);
    if (RESIDUAL) {
        const float2 b = __bfloat1622float2(h);
        r0 -= b.x;
        r1 -= b.y;
    }
    return *reinterpret_cast<const uint32_t*>(&h);
}

// ---------------------------------------------------------------- the GEMM kernel
// SYN: A = Lam^T (MN-major), B = synthesis image (K-major), D -> Fourier scratch.
// ANA: A = Lam (K-major), B = analysis image (MN-major), D -> coefficients.
// Persistent: CTA b of the grid's x dimension computes the items b, b + gridDim.x, ...
// of its column tile (grid y). The copy warp runs ahead through a ring of shared
// memory stages across items; the MMA thread alternates two accumulators in tensor
// memory so that the epilogue of one item overlaps the MMAs of the next.

template <bool SYN>
__device__ __forceinline__ int item_steps(const TcDev& t, const TcItem& it) {
    return SYN ? t.nkt[it.m] : t.njt[it.m];
}

// A CTA's items with their step counts and data-image tile bases, fetched by all its
// threads at once before the roles start (shared memory), so the producer does not wait
// on dependent global loads at the start of every item.
struct ItemInfo {
    TcItem it;
    int64_t tb;       // image tile index of (m, par, step 0)
    int32_t nsteps;
    int32_t pad;
};
constexpr int TC_ITEM_CACHE = 128;
constexpr int TC_ITEM_BYTES = TC_ITEM_CACHE * (int)sizeof(ItemInfo);

template <bool SYN>
__device__ __forceinline__ ItemInfo item_info(const TcDev& t, const TcItem& it) {
    ItemInfo f;
    f.it = it;
    f.nsteps = item_steps<SYN>(t, it);
    f.tb = SYN ? t.syn_tile_base[it.m] + (int64_t)it.par * t.nkt[it.m]
               : t.ana_tile_base[it.m] + (int64_t)it.par * t.njt[it.m];
    f.pad = 0;
    return f;
}

// 32 columns of the tile at TMEM address taddr: the leading-product accumulator plus,
// with xoff > 0, the cross-product accumulator xoff columns further (rounded FP32 sum)
__device__ __forceinline__ void acc_ld32(uint32_t taddr, uint32_t xoff, float (&v)[32]) {
    tmem_ld32(taddr, v);
    if (xoff) {
        float w[32];
        tmem_ld32(taddr + xoff, w);
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] = __fadd_rn(v[i], w[i]);
    }
}

template <bool SYN>
__device__ void epilogue_store(const TcDev& t, const TcItem& it, int ct, int ctw, int nt_cols, int K, uint32_t taddr,
                               uint32_t xoff, int r, int cb, float2* four, float2* coeffs, int64_t ldc, int add,
                               bool good, bool accumulate) {
    // this warp's column chunks: cb, cb + 64, ... (the other warp of its lane quarter takes the rest)
    const int m = it.m, par = it.par, tile = it.tile;
    const float mscale = t.fp16 ? ldexpf(1.f, t.mexp[m] - F16_TOP) : 1.f;
    if (SYN && t.matrix) {
        const int row = tile * 128 + r;
        const bool valid = good && row < t.mrows;
        const float rs = (valid && t.row_scale) ? t.row_scale[row] : 1.f;
        for (int c0 = cb; c0 < nt_cols; c0 += 64) {
            float v[32];
            acc_ld32(taddr + c0, xoff, v);
            if (!valid) continue;
#pragma unroll
            for (int q = 0; q < 32; ++q) {
                const int n = ct * ctw + c0 + q;
                if (n >= K) break;
                float x = v[q];
                if (t.fp16) x = x * mscale * t.kscale_syn[n].x;
                x = x * rs;
                float* o = t.mout + (int64_t)n * t.ldo + row;
                *o = accumulate ? *o + x : x;      // later depth chunks: this thread wrote *o before
            }
        }
        return;
    }
    if (SYN) {
        // Lane r holds ring r's 32 columns (16 complex k) of a chunk. A warp transposes the
        // chunk at float4 granularity with three shfl_xor stages so that one store instruction
        // writes 4 rings x 128 contiguous bytes (whole 128-byte lines when K is a multiple of
        // 16) instead of 16 bytes of each of 32 rings: after the exchange, float4 slot s of
        // lane x is ring 4 s + (x & 3), complex pair x >> 2.
        const int j = t.j0[m] + tile * 128 + r;
        const bool valid = good && j < t.nh && m <= t.rings[j].mt;
        float2* dst = valid ? four + ((t.rings[j].gofs + m) * 2 + par) * K : nullptr;
        const unsigned vm = __ballot_sync(0xffffffffu, valid);
        const int lane = r % 32;
        float2* rowp[8];
#pragma unroll
        for (int s = 0; s < 8; ++s)
            rowp[s] = reinterpret_cast<float2*>(
                __shfl_sync(0xffffffffu, reinterpret_cast<uintptr_t>(dst), 4 * s + (lane & 3)));
        for (int c0 = cb; c0 < nt_cols; c0 += 64) {
            float v[32];
            acc_ld32(taddr + c0, xoff, v);
            if (vm == 0) continue;
            const int k0 = (ct * ctw + c0) / 2;
            if (t.fp16) {
                const float2* mk = t.mkscale_syn + (int64_t)m * K;
#pragma unroll
                for (int q = 0; q < 16; ++q) {
                    const float f = mk[min(k0 + q, K - 1)].x;
                    v[2 * q] = v[2 * q] * mscale * f;
                    v[2 * q + 1] = v[2 * q + 1] * mscale * f;
                }
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {        // swap register bit i of the float4 index with lane bit 2 + i
                const bool upper = (lane >> (2 + i)) & 1;
#pragma unroll
                for (int f = 0; f < 8; ++f) {
                    if ((f >> i) & 1) continue;
                    const int f1 = f | (1 << i);
#pragma unroll
                    for (int c = 0; c < 4; ++c) {
                        const float send = upper ? v[4 * f + c] : v[4 * f1 + c];
                        const float recv = __shfl_xor_sync(0xffffffffu, send, 1 << (2 + i));
                        if (upper) v[4 * f + c] = recv;
                        else v[4 * f1 + c] = recv;
                    }
                }
            }
            const int k = k0 + 2 * (lane >> 2);
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                if (!((vm >> (4 * s + (lane & 3))) & 1)) continue;
                float2* d = rowp[s];
                if (k + 1 < K && (K % 2) == 0) {    // 16-byte aligned: row * K and k even
                    *reinterpret_cast<float4*>(d + k) = make_float4(v[4 * s], v[4 * s + 1], v[4 * s + 2], v[4 * s + 3]);
                } else {
                    if (k < K) d[k] = make_float2(v[4 * s], v[4 * s + 1]);
                    if (k + 1 < K) d[k + 1] = make_float2(v[4 * s + 2], v[4 * s + 3]);
                }
            }
        }
    } else {
        const int i = tile * 128 + r;
        const bool valid = good && i < t.rows[m] && m + 2 * i + par < t.lmax;
        const int64_t lmo = t.lm_off[m];
        for (int c0 = cb; c0 < nt_cols; c0 += 64) {
            float v[32];
            acc_ld32(taddr + c0, xoff, v);
            if (!valid) continue;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int k = (ct * ctw + c0) / 2 + q;
                if (k >= K) break;
                float2* d = coeffs + (int64_t)k * ldc + lmo + 2 * i + par;
                float2 val = make_float2(v[2 * q], v[2 * q + 1]);
                if (t.fp16) {
                    const float f = t.kscale_ana[k].x;
                    val.x = val.x * mscale * f;
                    val.y = val.y * mscale * f;
                }
                if (add) {
                    const float2 o = *d;
                    val.x += o.x;
                    val.y += o.y;
                }
                *d = val;
            }
        }
    }
}

template <bool SYN>
__global__ void __launch_bounds__(TC_THREADS, 1)
    legendre_tc_kernel(const TcDev t, const TcItem* __restrict__ items, int nitems, int K, int ctw, int nt_cols,
                       int stages, uint32_t acc_cols, int split, float2* __restrict__ four, float2* __restrict__ coeffs,
                       int64_t ldc, int add) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int ct = blockIdx.y;                       // column tile (ctw columns)
    // per item buffer: the leading-product accumulator, then (split) the cross-product one
    const uint32_t buf_cols = (split ? 2u : 1u) * acc_cols;
    const uint32_t xoff = split ? acc_cols : 0u;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int a_bytes = t.npa * A_PIECE_BYTES;
    const int b_piece_bytes = nt_cols * 128;
    const int stage_bytes = a_bytes + t.npb * b_piece_bytes;
    uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + (size_t)stages * stage_bytes);
    uint64_t* empty_bar = full_bar + stages;
    uint64_t* accf = empty_bar + stages;             // accumulator a ready   (tcgen05.commit)
    uint64_t* acce = accf + 2;                       // accumulator a drained (256 epilogue threads)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(acce + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    ItemInfo* info = reinterpret_cast<ItemInfo*>(smem + (size_t)stages * stage_bytes + 256);
    {   // this CTA's items ix = blockIdx.x + i gridDim.x, the first TC_ITEM_CACHE of them
        const int n_my = (int)blockIdx.x < nitems ? (nitems - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
        for (int i = threadIdx.x; i < min(n_my, TC_ITEM_CACHE); i += blockDim.x)
            info[i] = item_info<SYN>(t, items[blockIdx.x + i * gridDim.x]);
    }
    auto get = [&](int i, int ix) { return i < TC_ITEM_CACHE ? info[i] : item_info<SYN>(t, items[ix]); };

    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; ++s) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&accf[a], 1);
            mbar_init(&acce[a], 256);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * buf_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------ producer
        const int64_t img_tile_bytes = SYN ? t.syn_tile_bytes : t.ana_tile_bytes;
        const uint8_t* img = reinterpret_cast<const uint8_t*>(SYN ? t.syn_img : t.ana_img);
        const int64_t col_off = SYN ? (int64_t)ct * ctw * 128 : (int64_t)ct * (ctw / 64) * BOX_BYTES;
        int g = 0;
        bool ok = true;
        for (int i = 0, ix = blockIdx.x; ix < nitems && ok && !*abort_flag; ++i, ix += gridDim.x) {
            const ItemInfo f = get(i, ix);
            const int m = f.it.m, par = f.it.par, tile = f.it.tile;
            const int nsteps = f.nsteps;
            const CUtensorMap* map = t.maps + (2 * m + par);
            const int64_t tb = f.tb;
            for (int ks = 0; ks < nsteps; ++ks, ++g) {
                const int s = g % stages;
                if (g >= stages && !mbar_wait(&empty_bar[s], ((g / stages) - 1) & 1)) {
                    *abort_flag = 1;
                    atomicExch(t.err, 1);
                    ok = false;
                    break;
                }
                uint8_t* st = smem + (size_t)s * stage_bytes;
                mbar_expect_tx(&full_bar[s], (uint32_t)stage_bytes);
                for (int pa = 0; pa < t.npa; ++pa) {
                    uint8_t* a = st + pa * A_PIECE_BYTES;
                    if (SYN) {   // rings [128 tile, +128) of rows [64 ks, +64)
                        tma_load_3d(a, map, tile * 128, ks * BLK, pa, &full_bar[s]);
                        tma_load_3d(a + BOX_BYTES, map, tile * 128 + BLK, ks * BLK, pa, &full_bar[s]);
                    } else {     // rows [128 tile, +128) of rings [64 ks, +64)
                        tma_load_3d(a, map, ks * BLK, tile * 128, pa, &full_bar[s]);
                        tma_load_3d(a + BOX_BYTES, map, ks * BLK, tile * 128 + BLK, pa, &full_bar[s]);
                    }
                }
                for (int pb = 0; pb < t.npb; ++pb) {
                    const uint8_t* src = img + ((tb + ks) * t.npb + pb) * img_tile_bytes + col_off;
                    bulk_load(st + a_bytes + pb * b_piece_bytes, src, (uint32_t)b_piece_bytes, &full_bar[s]);
                }
            }
        }
        // No copy may still be landing in shared memory when the CTA exits: wait for the
        // last fill of every stage (already complete unless the MMA thread gave up).
        for (int u = g - 1; u >= 0 && u >= g - stages; --u)
            if (!mbar_wait(&full_bar[u % stages], (u / stages) & 1)) atomicExch(t.err, 5);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------ MMA issuer
        const uint32_t idesc = idesc_f16(t.fp16 ? 0u : 1u, SYN ? 1u : 0u, SYN ? 0u : 1u, (uint32_t)nt_cols);
        // Three products L0 B0 + (L0 B1 + L1 B0) with split accumulators: B0 and B1 lie next
        // to each other in the stage, so L0 x [B0; B1] is one MMA of N = 2 nt_cols whose two
        // halves are exactly the leading and the cross accumulator; L1 x B0 then adds to the
        // cross half. Two MMAs per step instead of three, and A piece 0 is read once.
        const bool stacked = split && t.nprod == 3 && t.npa == 2 && t.npb == 2 && 2 * nt_cols <= 256 &&
                             xoff == (uint32_t)nt_cols &&
                             t.prod == ((0u | (0u << 2)) | ((0u | (1u << 2)) << 4) | ((1u | (0u << 2)) << 8));
        const uint32_t idesc2 = idesc_f16(t.fp16 ? 0u : 1u, SYN ? 1u : 0u, SYN ? 0u : 1u, (uint32_t)(2 * nt_cols));
        int g = 0, ti = 0;
        bool ok = true;
        for (int i = 0, ix = blockIdx.x; ix < nitems && ok && !*abort_flag; ++i, ix += gridDim.x) {
            const ItemInfo f = get(i, ix);
            const int nsteps = f.nsteps;
            if (nsteps == 0) continue;
            const int kch = t.kchunk > 0 ? t.kchunk : nsteps;
          for (int ks0 = 0; ks0 < nsteps && ok; ks0 += kch) {
            const int a = ti & 1;
            if (ti >= 2 && !mbar_wait(&acce[a], ((ti / 2) - 1) & 1)) {
                *abort_flag = 1;
                atomicExch(t.err, 4);
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t dacc = tmem + (uint32_t)a * buf_cols;
            for (int ks = ks0; ks < min(nsteps, ks0 + kch); ++ks, ++g) {
                const int s = g % stages;
                if (!mbar_wait(&full_bar[s], (g / stages) & 1)) {
                    *abort_flag = 1;
                    atomicExch(t.err, 2);
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t st = smem_u32(smem + (size_t)s * stage_bytes);
                if (stacked) {
                    for (int kk = 0; kk < BLK / 16; ++kk) {
                        const uint32_t a0 = st, a1 = st + A_PIECE_BYTES, b0 = st + a_bytes;
                        uint64_t da0, da1, db;
                        if (SYN) {
                            da0 = sdesc(a0 + kk * 2048, BOX_BYTES, 1024);
                            da1 = sdesc(a1 + kk * 2048, BOX_BYTES, 1024);
                            db = sdesc(b0 + kk * 32, 16, 1024);
                        } else {
                            da0 = sdesc(a0 + kk * 32, 16, 1024);
                            da1 = sdesc(a1 + kk * 32, 16, 1024);
                            db = sdesc(b0 + kk * 2048, BOX_BYTES, 1024);
                        }
                        umma_f16(dacc, da0, db, idesc2, (ks == ks0 && kk == 0) ? 0u : 1u);   // L0 [B0; B1]
                        umma_f16(dacc + xoff, da1, db, idesc, 1u);                           // L1 B0
                    }
                    umma_commit(&empty_bar[s]);
                    continue;
                }
                for (int kk = 0; kk < BLK / 16; ++kk) {
                    for (int q = 0; q < t.nprod; ++q) {
                        const int pa = (t.prod >> (4 * q)) & 3, pb = (t.prod >> (4 * q + 2)) & 3;
                        // product 0 is piece 0 x piece 0 (the leading one); with split the
                        // others go to the cross accumulator, whose first write is product 1
                        const bool cross = split && q > 0;
                        const uint32_t dst = cross ? dacc + xoff : dacc;
                        const bool first = ks == ks0 && kk == 0 && q == (cross ? 1 : 0);
                        const uint32_t aa = st + pa * A_PIECE_BYTES;
                        const uint32_t bb = st + a_bytes + pb * b_piece_bytes;
                        uint64_t da, db;
                        if (SYN) {
                            da = sdesc(aa + kk * 2048, BOX_BYTES, 1024);     // MN-major: 16 rows per step
                            db = sdesc(bb + kk * 32, 16, 1024);              // K-major: 32 B per step
                        } else {
                            da = sdesc(aa + kk * 32, 16, 1024);
                            db = sdesc(bb + kk * 2048, BOX_BYTES, 1024);
                        }
                        umma_f16(dst, da, db, idesc, first ? 0u : 1u);
                    }
                }
                umma_commit(&empty_bar[s]);      // frees the stage once these MMAs complete
            }
            umma_commit(&accf[a]);               // accumulator ready (or drained after an abort)
            ++ti;
          }
        }
        // Every MMA must have completed before the tensor memory is released.
        if (ti > 0 && !mbar_wait(&accf[(ti - 1) & 1], ((ti - 1) / 2) & 1)) atomicExch(t.err, 6);
    } else if (warp >= 2) {
        // ------------------------------------------------ epilogue
        // warp w reads TMEM lanes 32 (w % 4) .. + 31 (rows r); the two warps of a lane
        // quarter take alternate 32-column chunks
        const int quarter = warp % 4, half = (warp - 2) / 4;
        const int r = quarter * 32 + lane;
        int ti = 0;
        for (int q = 0, ix = blockIdx.x; ix < nitems; ++q, ix += gridDim.x) {
            const ItemInfo f = get(q, ix);
            const TcItem it = f.it;
            if (f.nsteps == 0) {      // analysis of an order no ring carries: zeros
                if (!SYN && !add && !*abort_flag) {
                    const int i = it.tile * 128 + r;
                    if (i < t.rows[it.m] && it.m + 2 * i + it.par < t.lmax)
                        for (int c = 2 * half; c < nt_cols && ct * ctw + c < 2 * K; c += 4)
                            coeffs[(int64_t)((ct * ctw + c) / 2) * ldc + t.lm_off[it.m] + 2 * i + it.par] =
                                make_float2(0.f, 0.f);
                }
                continue;
            }
            const int nsteps = f.nsteps;
            const int kch = t.kchunk > 0 ? t.kchunk : nsteps;
            bool ok = true;
            for (int ks0 = 0; ks0 < nsteps; ks0 += kch) {
                const int a = ti & 1;
                // warp-uniform outcome: tcgen05.ld below is a warp-collective instruction
                ok = __all_sync(0xffffffffu, mbar_wait(&accf[a], (ti / 2) & 1));
                if (!ok) {
                    *abort_flag = 1;
                    atomicExch(t.err, 3);
                }
                tc_fence_after();
                const uint32_t taddr = tmem + (uint32_t)a * buf_cols + ((uint32_t)(quarter * 32) << 16);
                epilogue_store<SYN>(t, it, ct, ctw, nt_cols, K, taddr, xoff, r, 32 * half, four, coeffs, ldc, add,
                                    ok && !*abort_flag, ks0 > 0);
                tc_fence_before();
                mbar_arrive(&acce[a]);
                ++ti;
                if (!ok) break;
            }
            if (!ok) break;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * buf_cols)
                     : "memory");
    }
}

// ---------------------------------------------------------------- synthesis data image
// coefficients [k][lm] complex FP32 -> per (m, p, kt, piece) K-major SWIZZLE_128B tiles
// of nmax rows (columns c = 2k + re/im) x 64 parity rows (128 B).

// Synthesis data image. CTA: order m, 64-row block kt, 32 layers. The CTA first stages
// the 128 packed coefficients (both parities) of each of its layers in shared memory
// with asynchronous copies, a warp copying 512 consecutive bytes per instruction (16-byte
// copies where the run is 16-byte aligned, 8-byte copies otherwise; coefficients past the
// order's last one staged as zeros). Then one thread per (8-row chunk ib8, layer k) reads
// its 16 coefficients from shared memory and writes, per parity, real/imaginary column
// and piece, one whole 16-byte chunk of the swizzled K-major tile: rows 8 ib8 .. 8 ib8 + 7
// of column c = 2 k + ri (the 8 threads of a layer fill the tile row's 128 bytes).
// Shared layout: per layer 8 runs of 16 coefficients, 144 bytes apart, so that the 8
// threads of a layer read distinct banks.
constexpr int IMG_RUN = 144;                 // bytes per staged run of 16 coefficients (128 + 16 pad)
constexpr int IMG_LAYER = 8 * IMG_RUN;       // bytes per staged layer

__device__ __forceinline__ void cp_async_16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_8(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
}

// One 128-coefficient block kt of order m for the 32 layers from kbase: staged in shared
// memory by asynchronous copies, scaled by sc (the fp16 data scale of this thread's layer;
// 1 for bf16), split into NPB 16-bit pieces and written as swizzled image rows.
template <int NPB, bool F16>
__device__ __forceinline__ void syn_image_block(const TcDev& t, const float2* __restrict__ coeffs, int64_t ldc,
                                                int K, int m, int kt, int kbase, float sc, uint8_t* stage) {
    const int lmrem = t.lmax - m - 2 * BLK * kt;             // packed coefficients left from this block
    const float2* src0 = coeffs + t.lm_off[m] + 2 * BLK * kt;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(stage);
    const bool al16 = ((reinterpret_cast<uintptr_t>(src0) & 15) == 0) && ((ldc & 1) == 0);
    if (al16) {
        // 32 layers x 64 pairs of coefficients: lanes take consecutive pairs of a layer
        for (int w = threadIdx.x; w < 32 * 64; w += 256) {
            const int kl = w >> 6, e2 = w & 63, e = 2 * e2;
            const uint32_t soff = kl * IMG_LAYER + (e >> 4) * IMG_RUN + (e & 15) * 8;
            if (kbase + kl < K && e + 1 < lmrem)
                cp_async_16(sbase + soff, src0 + (int64_t)(kbase + kl) * ldc + e);
            else
                *reinterpret_cast<float4*>(stage + soff) =
                    make_float4(0.f, 0.f, 0.f, 0.f);   // past the order (or K), or half of the last pair below
            if (kbase + kl < K && e < lmrem && e + 1 >= lmrem)
                *reinterpret_cast<float2*>(stage + soff) = src0[(int64_t)(kbase + kl) * ldc + e];
        }
    } else {
        for (int w = threadIdx.x; w < 32 * 128; w += 256) {
            const int kl = w >> 7, e = w & 127;
            const uint32_t soff = kl * IMG_LAYER + (e >> 4) * IMG_RUN + (e & 15) * 8;
            if (kbase + kl < K && e < lmrem)
                cp_async_8(sbase + soff, src0 + (int64_t)(kbase + kl) * ldc + e);
            else
                *reinterpret_cast<float2*>(stage + soff) = make_float2(0.f, 0.f);
        }
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const int ib8 = threadIdx.x & 7;
    const int k = kbase + (threadIdx.x >> 3);
    if (k < K) {
        float2 v[16];
        const float4* run = reinterpret_cast<const float4*>(stage + (threadIdx.x >> 3) * IMG_LAYER + ib8 * IMG_RUN);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float4 f = run[q];
            v[2 * q] = make_float2(f.x, f.y);
            v[2 * q + 1] = make_float2(f.z, f.w);
        }
        if (F16) {
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = make_float2(v[q].x * sc, v[q].y * sc);
        }
        uint8_t* img = reinterpret_cast<uint8_t*>(const_cast<uint16_t*>(t.syn_img));
#pragma unroll
        for (int par = 0; par < 2; ++par) {
            const int64_t tile = t.syn_tile_base[m] + (int64_t)par * t.nkt[m] + kt;
#pragma unroll
            for (int ri = 0; ri < 2; ++ri) {
                const int c = 2 * k + ri;
                uint32_t w[NPB][4];
#pragma unroll
                for (int h = 0; h < 4; ++h) {
                    float r0 = ri ? v[2 * (2 * h) + par].y : v[2 * (2 * h) + par].x;
                    float r1 = ri ? v[2 * (2 * h + 1) + par].y : v[2 * (2 * h + 1) + par].x;
#pragma unroll
                    for (int q = 0; q < NPB; ++q) {
                        w[q][h] = q + 1 < NPB ? piece_bits2<F16, true>(r0, r1) : piece_bits2<F16, false>(r0, r1);
                    }
                }
                const int64_t off = (int64_t)(c / 8) * 1024 + (c % 8) * 128 + ((ib8 ^ (c % 8)) * 16);
#pragma unroll
                for (int q = 0; q < NPB; ++q)
                    *reinterpret_cast<uint4*>(img + (tile * NPB + q) * t.syn_tile_bytes + off) =
                        make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
            }
        }
    }
}

// bf16 pieces: one block (m, kt, 32 layers).
template <int NPB>
__global__ void __launch_bounds__(256) syn_image_kernel(const TcDev t, const float2* __restrict__ coeffs,
                                                        int64_t ldc, int K) {
    __shared__ __align__(16) uint8_t stage[32 * IMG_LAYER];
    const int m = blockIdx.x;
    const int kt = blockIdx.y;
    if (kt >= t.nkt[m]) return;
    syn_image_block<NPB, false>(t, coeffs, ldc, K, m, kt, blockIdx.z * 32, 1.f, stage);
}

// fp16 pieces: one block per (m, 32 layers) takes all blocks kt of the order. It first
// reduces each layer's max-abs over the order's coefficients (8 lanes per layer), which
// sets the data scale 2^(15 - e_mk) of that order and layer (stored for the GEMM's
// epilogue as (2^(e_mk - 15), 2^(15 - e_mk))), then writes the blocks; the second read
// of the coefficients comes from L2.
__global__ void __launch_bounds__(256) syn_image_f16_kernel(const TcDev t, const float2* __restrict__ coeffs,
                                                            int64_t ldc, int K) {
    __shared__ __align__(16) uint8_t stage[32 * IMG_LAYER];
    const int m = blockIdx.x;
    const int kbase = blockIdx.z * 32;
    const int k = kbase + (threadIdx.x >> 3);
    const int n = t.lmax - m;                                // coefficients of order m
    float mx = 0.f;
    if (k < K) {
        const float2* src = coeffs + (int64_t)k * ldc + t.lm_off[m];
        int e = threadIdx.x & 7;
        for (; e + 24 < n; e += 32) {                        // four loads in flight
            const float2 a = __ldg(src + e), b = __ldg(src + e + 8), c = __ldg(src + e + 16), d = __ldg(src + e + 24);
            mx = fmaxf(mx, fmaxf(fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(b.x), fabsf(b.y))),
                                 fmaxf(fmaxf(fabsf(c.x), fabsf(c.y)), fmaxf(fabsf(d.x), fabsf(d.y)))));
        }
        for (; e < n; e += 8) {
            const float2 a = __ldg(src + e);
            mx = fmaxf(mx, fmaxf(fabsf(a.x), fabsf(a.y)));
        }
    }
    // the 8 lanes of a layer are consecutive lanes of one warp
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 2));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, 4));
    const int ex = scale_exp(mx);
    if (k < K && (threadIdx.x & 7) == 0)
        t.mkscale_syn[(int64_t)m * K + k] = make_float2(ldexpf(1.f, ex - F16_TOP), ldexpf(1.f, F16_TOP - ex));
    const float sc = ldexpf(1.f, F16_TOP - ex);
    for (int kt = 0; kt < t.nkt[m]; ++kt) {
        if (kt > 0) __syncthreads();                         // the stage's previous block is consumed
        syn_image_block<2, true>(t, coeffs, ldc, K, m, kt, kbase, sc, stage);
    }
}

// Per-layer max-abs of the transform inputs (the fp16 data scaling): 16-byte loads
// where aligned, one atomic max (on the bits of a non-negative float) per warp.
__device__ __forceinline__ void warp_atomic_max(float* out, float mx) {
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<unsigned int*>(out), __float_as_uint(mx));
}
__global__ void absmax_kernel(const float* __restrict__ x, int64_t ld, int64_t n, float* __restrict__ out) {
    const int k = blockIdx.y;
    const float* row = x + (int64_t)k * ld;
    float mx = 0.f;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i0 = 0;
    if ((reinterpret_cast<uintptr_t>(row) & 15) == 0) {
        const float4* r4 = reinterpret_cast<const float4*>(row);
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n / 4; i += stride) {
            const float4 v = __ldg(r4 + i);
            mx = fmaxf(mx, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
        }
        i0 = n / 4 * 4;
    }
    for (int64_t i = i0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
        mx = fmaxf(mx, fabsf(__ldg(row + i)));
    warp_atomic_max(out + k, mx);
}
// (2^(e - 15), 2^(15 - e)) with bound = mul * max-abs, |bound| 2^-e < 1
__global__ void kscale_kernel(const float* __restrict__ absmax, float mul, int K, float2* __restrict__ out) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        const int e = scale_exp(absmax[k] * mul);
        out[k] = make_float2(ldexpf(1.f, e - F16_TOP), ldexpf(1.f, F16_TOP - e));
    }
}

// ---------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 get_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

TcDev make_dev(const Plan& p) {
    const TcState& s = *static_cast<const TcState*>(p.tc);
    TcDev t{};
    t.maps = s.d_maps;
    t.nr = s.d_nr;
    t.j0 = p.d_j0;
    t.rows = p.d_rows;
    t.lm_off = p.d_lm_off;
    t.syn_tile_base = s.d_syn_base;
    t.ana_tile_base = s.d_ana_base;
    t.nkt = s.d_nkt;
    t.njt = s.d_njt;
    t.rings = p.d_rings;
    t.syn_img = s.d_syn_img;
    t.ana_img = s.d_ana_img;
    t.err = p.d_err;
    t.nh = p.nh;
    t.lmax = p.lmax;
    t.mmax = p.mmax;
    t.npa = s.npa;
    t.npb = s.npb;
    t.nprod = s.nprod;
    t.prod = s.prod;
    t.syn_tile_bytes = s.syn_tile_bytes;
    t.ana_tile_bytes = s.ana_tile_bytes;
    t.nmax = s.nmax;
    t.fp16 = s.fp16;
    t.mexp = s.d_mexp;
    t.kscale_syn = s.d_kscale;
    t.mkscale_syn = s.d_mkscale;
    t.kscale_ana = s.d_kscale ? s.d_kscale + p.d.nlayers : nullptr;
    return t;
}

int smem_for(int npa, int npb, int nt_cols, int& stages) {
    const int stage_bytes = npa * A_PIECE_BYTES + npb * nt_cols * 128;
    const int budget = 227 * 1024 - 1024 - 256 - TC_ITEM_BYTES;   // alignment slack, barriers, item table
    stages = std::min(4, budget / stage_bytes);
    return 1024 + stages * stage_bytes + 256 + TC_ITEM_BYTES;
}

// Failure-detection check of the bounded waits. One thread waits through the routine of
// the kernels' pipelines (mbar_wait_for), first for an mbarrier phase it completes itself
// (must succeed), then for one that nothing completes (must expire after limit_ns). It
// stores SHT_STATUS_DIAG_EXPIRED when both behave, SHT_STATUS_DIAG_FAILED otherwise, and
// returns: nothing is in flight and the context stays usable.
__global__ void wait_probe_kernel(int32_t* err, uint64_t limit_ns) {
    __shared__ __align__(8) uint64_t bar[2];
    if (threadIdx.x != 0) return;
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_arrive(&bar[0]);
    const bool done = mbar_wait_for(&bar[0], 0, limit_ns);
    const bool expired = !mbar_wait_for(&bar[1], 0, limit_ns);
    atomicExch(err, done && expired ? SHT_STATUS_DIAG_EXPIRED : SHT_STATUS_DIAG_FAILED);
}

}  // namespace

cudaError_t launch_wait_probe(int32_t* err, uint64_t limit_ns, cudaStream_t s) {
    wait_probe_kernel<<<1, 32, 0, s>>>(err, limit_ns);
    return cudaGetLastError();
}

int tc_supported() { return get_encoder() != nullptr; }

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() { return get_encoder(); }

cudaError_t tc_prepare(Plan& p) {
    TcState* s = new TcState();
    p.tc = s;
    if (p.d.precision == SHT_PREC_BF16X3) {
        s->npa = 2; s->npb = 2; s->nprod = 3;
        s->prod = (0u | (0u << 2)) | ((0u | (1u << 2)) << 4) | ((1u | (0u << 2)) << 8);
    } else if (p.d.precision == SHT_PREC_FP16X3) {
        s->npa = 2; s->npb = 2; s->nprod = 3; s->fp16 = 1;
        s->prod = (0u | (0u << 2)) | ((0u | (1u << 2)) << 4) | ((1u | (0u << 2)) << 8);
    } else if (p.d.precision == SHT_PREC_BF16X5) {
        s->npa = 3; s->npb = 2; s->nprod = 5;
        s->prod = (0u | (0u << 2)) | ((0u | (1u << 2)) << 4) | ((1u | (0u << 2)) << 8) | ((1u | (1u << 2)) << 12) |
                  ((2u | (0u << 2)) << 16);
    } else {
        return cudaErrorNotSupported;
    }
    const int nh = p.nh, mmax = p.mmax;
    // image columns: whole column tiles (kTcTileCols) once a call can need more than one
    s->nmax = 2 * p.d.nlayers <= kTcTileCols ? (2 * p.d.nlayers + 63) / 64 * 64
                                             : (2 * p.d.nlayers + kTcTileCols - 1) / kTcTileCols * kTcTileCols;

    // --- Legendre pieces [m][p][piece][i][j - j0] with row pitch rounded to 8 rings ---
    std::vector<int32_t> nr(mmax), pitch(mmax), nkt(mmax), njt(mmax);
    std::vector<int64_t> blk_off(2 * mmax);
    int64_t total = 0;
    for (int m = 0; m < mmax; ++m) {
        nr[m] = nh - p.j0[m];
        pitch[m] = std::max(8, (nr[m] + 7) / 8 * 8);
        nkt[m] = (p.rows[m] + BLK - 1) / BLK;
        njt[m] = (nr[m] + BLK - 1) / BLK;
        for (int par = 0; par < 2; ++par) {
            blk_off[2 * m + par] = total;
            total += (int64_t)s->npa * p.rows[m] * pitch[m];
        }
    }
    std::vector<uint16_t> lam((size_t)total, 0);
    std::vector<int32_t> mexp(mmax, 0);
    {
        const int nthreads = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
        // Lam(l, m) of ring j in FP64 for m <= mt(j): fn(m, column, L)
        auto columns = [&](int j, std::vector<double>& col, auto&& fn) {
            const double colat = M_PI / 2 - p.latd[j] * M_PI / 180.0;
            const double xc = std::cos(colat);
            const double sn = std::sqrt(std::max(0.0, 1.0 - xc * xc));
            double pmm = 1.0 / std::sqrt(4.0 * M_PI);
            for (int m = 0; m <= p.mt[j]; ++m) {
                if (m > 0) pmm = -std::sqrt((2.0 * m + 1.0) / (2.0 * m)) * sn * pmm;
                const int L = p.lmax - m;
                col[0] = pmm;
                if (L >= 2) {
                    double p0 = pmm, p1 = std::sqrt(2.0 * m + 3.0) * xc * pmm;
                    col[1] = p1;
                    double a_prev = std::sqrt((4.0 * (m + 1) * (m + 1) - 1.0) / ((m + 1.0) * (m + 1.0) - 1.0 * m * m));
                    for (int l = m + 2; l < p.lmax; ++l) {
                        const double a = std::sqrt((4.0 * l * l - 1.0) / (1.0 * l * l - 1.0 * m * m));
                        const double p2 = a * (xc * p1 - p0 / a_prev);
                        col[l - m] = p2;
                        p0 = p1;
                        p1 = p2;
                        a_prev = a;
                    }
                }
                fn(m, col, L);
            }
        };
        if (s->fp16) {   // pass 1: e_m from max |Lam| of every order
            std::vector<std::vector<double>> mx(nthreads, std::vector<double>(mmax, 0.0));
            auto work = [&](int tid) {
                std::vector<double> col(p.lmax);
                for (int j = tid; j < nh; j += nthreads)
                    columns(j, col, [&](int m, const std::vector<double>& c, int L) {
                        for (int i = 0; i < L; ++i) mx[tid][m] = std::max(mx[tid][m], std::fabs(c[i]));
                    });
            };
            std::vector<std::thread> th;
            for (int t = 0; t < nthreads; ++t) th.emplace_back(work, t);
            for (auto& t : th) t.join();
            for (int m = 0; m < mmax; ++m) {
                double v = 0.0;
                for (int t = 0; t < nthreads; ++t) v = std::max(v, mx[t][m]);
                int ex = 0;
                if (v > 0.0) std::frexp(v, &ex);
                mexp[m] = ex;
            }
        }
        auto work = [&](int tid) {
            std::vector<double> col(p.lmax);
            for (int j = tid; j < nh; j += nthreads)
                columns(j, col, [&](int m, const std::vector<double>& c, int L) {
                    const int jj = j - p.j0[m];
                    const double sc = s->fp16 ? std::ldexp(1.0, F16_TOP - mexp[m]) : 1.0;
                    for (int i = 0; i < L; ++i) {
                        const int par = i & 1, row = i >> 1;
                        double r = c[i] * sc;
                        for (int q = 0; q < s->npa; ++q) {
                            uint16_t bits;
                            if (s->fp16) {
                                const __half h = __float2half_rn((float)r);
                                bits = __half_as_ushort(h);
                                r -= (double)__half2float(h);
                            } else {
                                const __nv_bfloat16 h = __float2bfloat16_rn((float)r);
                                bits = __bfloat16_as_ushort(h);
                                r -= (double)__bfloat162float(h);
                            }
                            lam[blk_off[2 * m + par] + ((int64_t)q * p.rows[m] + row) * pitch[m] + jj] = bits;
                        }
                    }
                });
        };
        std::vector<std::thread> th;
        for (int t = 0; t < nthreads; ++t) th.emplace_back(work, t);
        for (auto& t : th) t.join();
    }
    cudaError_t e;
    if ((e = cudaMalloc(&s->d_lam, std::max<int64_t>(16, total) * 2)) != cudaSuccess) return e;
    if ((e = cudaMemcpy(s->d_lam, lam.data(), total * 2, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    p.table_bytes += total * 2;

    // --- tensor maps, one per (m, p): dims {rings, parity rows, pieces}, box 64 x 64 x 1 ---
    auto enc = get_encoder();
    if (!enc) return cudaErrorNotSupported;
    std::vector<CUtensorMap> maps(2 * mmax);
    std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
    for (int m = 0; m < mmax; ++m)
        for (int par = 0; par < 2; ++par) {
            if (nr[m] == 0) continue;
            cuuint64_t dims[3] = {(cuuint64_t)nr[m], (cuuint64_t)p.rows[m], (cuuint64_t)s->npa};
            cuuint64_t strides[2] = {(cuuint64_t)pitch[m] * 2, (cuuint64_t)pitch[m] * 2 * p.rows[m]};
            cuuint32_t box[3] = {BLK, BLK, 1};
            cuuint32_t estr[3] = {1, 1, 1};
            CUresult r = enc(&maps[2 * m + par], s->fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3,
                             s->d_lam + blk_off[2 * m + par], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
        }
    if ((e = cudaMalloc(&s->d_maps, maps.size() * sizeof(CUtensorMap))) != cudaSuccess) return e;
    if ((e = cudaMemcpy(s->d_maps, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice)) !=
        cudaSuccess)
        return e;

    // --- data images ---
    s->syn_tile_bytes = (int64_t)s->nmax * 128;
    s->ana_tile_bytes = (int64_t)(s->nmax / 64) * BOX_BYTES;
    std::vector<int64_t> syn_base(mmax), ana_base(mmax);
    int64_t ns = 0, na = 0;
    for (int m = 0; m < mmax; ++m) {
        syn_base[m] = ns;
        ns += 2LL * nkt[m];
        ana_base[m] = na;
        na += 2LL * njt[m];
    }
    if ((e = cudaMalloc(&s->d_syn_img, std::max<int64_t>(1, ns) * s->npb * s->syn_tile_bytes)) != cudaSuccess) return e;
    if ((e = cudaMalloc(&s->d_ana_img, std::max<int64_t>(1, na) * s->npb * s->ana_tile_bytes)) != cudaSuccess) return e;
    if ((e = cudaMemset(s->d_syn_img, 0, std::max<int64_t>(1, ns) * s->npb * s->syn_tile_bytes)) != cudaSuccess) return e;
    if ((e = cudaMemset(s->d_ana_img, 0, std::max<int64_t>(1, na) * s->npb * s->ana_tile_bytes)) != cudaSuccess) return e;

    auto up32 = [&](int32_t** d, const std::vector<int32_t>& v) {
        cudaError_t ee = cudaMalloc(d, v.size() * 4);
        return ee != cudaSuccess ? ee : cudaMemcpy(*d, v.data(), v.size() * 4, cudaMemcpyHostToDevice);
    };
    auto up64 = [&](int64_t** d, const std::vector<int64_t>& v) {
        cudaError_t ee = cudaMalloc(d, v.size() * 8);
        return ee != cudaSuccess ? ee : cudaMemcpy(*d, v.data(), v.size() * 8, cudaMemcpyHostToDevice);
    };
    if ((e = up32(&s->d_nr, nr)) != cudaSuccess) return e;
    if ((e = up32(&s->d_nkt, nkt)) != cudaSuccess) return e;
    if ((e = up32(&s->d_njt, njt)) != cudaSuccess) return e;
    if ((e = up64(&s->d_syn_base, syn_base)) != cudaSuccess) return e;
    if ((e = up64(&s->d_ana_base, ana_base)) != cudaSuccess) return e;

    // --- work items (heavy orders first) ---
    std::vector<TcItem> syn, ana;
    for (int m = 0; m < mmax; ++m)
        for (int par = 0; par < 2; ++par) {
            for (int tl = 0; tl * 128 < nr[m]; ++tl) syn.push_back({m, par, tl, 0});
            for (int tl = 0; tl * 128 < p.rows[m]; ++tl) ana.push_back({m, par, tl, 0});
        }
    auto upi = [&](TcItem** d, const std::vector<TcItem>& v) {
        cudaError_t ee = cudaMalloc(d, std::max<size_t>(1, v.size()) * sizeof(TcItem));
        return ee != cudaSuccess ? ee : cudaMemcpy(*d, v.data(), v.size() * sizeof(TcItem), cudaMemcpyHostToDevice);
    };
    if ((e = upi(&s->d_syn_items, syn)) != cudaSuccess) return e;
    if ((e = upi(&s->d_ana_items, ana)) != cudaSuccess) return e;
    s->n_syn_items = (int)syn.size();
    s->n_ana_items = (int)ana.size();

    // --- the image the FFT analysis kernel writes ---
    p.ana_img.base = s->d_ana_img;
    p.ana_img.tile_base = s->d_ana_base;
    p.ana_img.njt = s->d_njt;
    p.ana_img.j0 = p.d_j0;
    p.ana_img.npieces = s->npb;
    p.ana_img.tile_bytes = (int32_t)s->ana_tile_bytes;
    p.ana_img.fp16 = s->fp16;
    if (s->fp16) {
        if ((e = up32(&s->d_mexp, mexp)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&s->d_absmax, 2 * sizeof(float) * std::max(1, p.d.nlayers))) != cudaSuccess) return e;
        if ((e = cudaMemset(s->d_absmax, 0, 2 * sizeof(float) * std::max(1, p.d.nlayers))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&s->d_kscale, 2 * sizeof(float2) * std::max(1, p.d.nlayers))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&s->d_mkscale, sizeof(float2) * (size_t)p.mmax * std::max(1, p.d.nlayers))) != cudaSuccess)
            return e;
        double wmax = 0.0;
        for (int j = 0; j < p.nlat; ++j) wmax = std::max(wmax, p.weights[j]);
        s->ana_mul = (float)(4.0 * M_PI * wmax * 1.0000001);
        p.ana_img.kscale = s->d_kscale + p.d.nlayers;
    }

    s->max_smem = 227 * 1024;
    {
        int dev = 0, nsm = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && nsm > 0)
            s->nsm = nsm;
    }
    if ((e = cudaFuncSetAttribute(legendre_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  s->max_smem)) != cudaSuccess)
        return e;
    return cudaFuncSetAttribute(legendre_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, s->max_smem);
}

void tc_release(Plan& p) {
    TcState* s = static_cast<TcState*>(p.tc);
    if (!s) return;
    void* ptrs[] = {s->d_maps, s->d_lam, s->d_nr, s->d_nkt, s->d_njt, s->d_syn_base, s->d_ana_base,
                    s->d_syn_img, s->d_ana_img, s->d_syn_items, s->d_ana_items, s->d_mexp, s->d_absmax,
                    s->d_kscale, s->d_mkscale};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    delete s;
    p.tc = nullptr;
}

static uint32_t tmem_cols_for(int n) {
    uint32_t c = 32;
    while ((int)c < n) c <<= 1;
    return c;
}

cudaError_t launch_legendre_synthesis_tc(const Plan& p, const float2* coeffs, int64_t ldc, int K, cudaStream_t st) {
    const TcState& s = *static_cast<const TcState*>(p.tc);
    const TcDev t = make_dev(p);
    cudaError_t e;
    const dim3 ig(p.mmax, (p.rows[0] + BLK - 1) / BLK, (K + 31) / 32);
    if (s.fp16)
        syn_image_f16_kernel<<<dim3(p.mmax, 1, (K + 31) / 32), 256, 0, st>>>(t, coeffs, ldc, K);
    else if (s.npb == 2)
        syn_image_kernel<2><<<ig, 256, 0, st>>>(t, coeffs, ldc, K);
    else
        syn_image_kernel<3><<<ig, 256, 0, st>>>(t, coeffs, ldc, K);
    e = cudaGetLastError();
    if (e != cudaSuccess || s.n_syn_items == 0) return e;
    const int ncols = 2 * K;
    const int nct = (ncols + s.ctw - 1) / s.ctw;
    const int nt_cols = std::min(s.ctw, (ncols + 63) / 64 * 64);
    int stages;
    const int smem = smem_for(s.npa, s.npb, nt_cols, stages);
    legendre_tc_kernel<true><<<dim3(std::min(s.n_syn_items, s.nsm), nct), TC_THREADS, smem, st>>>(
        t, s.d_syn_items, s.n_syn_items, K, s.ctw, nt_cols, stages, tmem_cols_for(nt_cols), 1, p.d_four, nullptr,
        0, 0);
    return cudaGetLastError();
}

// mul: bound of the analysis data per unit grid value; 0 = the transform's (4 pi max w)
// ---------------------------------------------------------------- dense matrix transforms
// A matrix operand [depth][M] (M contiguous, FP32) as 16-bit pieces [piece][depth][Mp]
// (Mp = M rounded up to 8 for 16-byte TMA strides), scaled by 2^(15 - e) for fp16.
__global__ void matrix_pieces_kernel(const float* __restrict__ a, int64_t depth, int M, int Mp, int npa, int fp16,
                                     float scale, uint16_t* __restrict__ out) {
    const int64_t total = depth * (int64_t)Mp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = i / Mp;
        const int m = (int)(i - d * Mp);
        float r = m < M ? a[d * M + m] * scale : 0.f;
        for (int q = 0; q < npa; ++q) {
            const uint32_t b = fp16 ? piece_bits<true>(r) : piece_bits<false>(r);
            out[(int64_t)q * total + i] = (uint16_t)b;
        }
    }
}

// B operand image of a matrix product: layer columns n < K of depth values from
// in[n ld + d] (FP32), as K-major SWIZZLE_128B tiles per (64-deep block, piece),
// nmax columns; depth past the end written as zeros.
template <int NPB, bool F16>
__global__ void __launch_bounds__(256) matrix_image_kernel(const float* __restrict__ in, int64_t ld, int depth, int K,
                                                           const float2* __restrict__ kscale, uint16_t* __restrict__ img,
                                                           int64_t tile_bytes) {
    const int kt = blockIdx.x;
    const int ib8 = threadIdx.x & 7;
    const int n = blockIdx.y * 32 + (threadIdx.x >> 3);
    if (n >= K) return;
    const int d0 = kt * BLK + 8 * ib8;
    float v[8];
    const float sc = F16 ? kscale[n].y : 1.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = d0 + q < depth ? __ldg(in + (int64_t)n * ld + d0 + q) * sc : 0.f;
    uint32_t w[NPB][4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
        float r0 = v[2 * h], r1 = v[2 * h + 1];
#pragma unroll
        for (int q = 0; q < NPB; ++q) {
            w[q][h] = q + 1 < NPB ? piece_bits2<F16, true>(r0, r1) : piece_bits2<F16, false>(r0, r1);
        }
    }
    const int64_t off = (int64_t)(n / 8) * 1024 + (n % 8) * 128 + ((ib8 ^ (n % 8)) * 16);
    uint8_t* base = reinterpret_cast<uint8_t*>(img);
#pragma unroll
    for (int q = 0; q < NPB; ++q)
        *reinterpret_cast<uint4*>(base + ((int64_t)kt * NPB + q) * tile_bytes + off) =
            make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
}

struct TcMatrixDir {               // one matrix (analysis or synthesis direction)
    int depth = 0, M = 0, Mp = 0, nkt = 0;
    uint16_t* d_a = nullptr;       // pieces
    CUtensorMap* d_map = nullptr;
    int32_t* d_nkt = nullptr;
    int32_t* d_mexp = nullptr;     // fp16: e of the matrix
    TcItem* d_items = nullptr;
    int nitems = 0;
};

struct TcMatrix {
    int npa = 2, npb = 2, nprod = 3, fp16 = 0;
    uint32_t prod = 0;
    int nmax = 0, nsm = 148, nlayers = 0;
    TcMatrixDir dir[2];            // 0: analysis (A = F^T as [npoints][2 nlm]), 1: synthesis
    int64_t* d_base = nullptr;     // {0}
    uint16_t* d_img = nullptr;
    int64_t tile_bytes = 0;
    float* d_absmax = nullptr;
    float2* d_kscale = nullptr;
};

cudaError_t tc_matrix_create(TcMatrix** out, int precision, const float* const a[2], const int depth[2],
                             const int M[2], int nlayers) {
    TcMatrix* x = new TcMatrix();
    *out = x;
    if (precision == SHT_PREC_BF16X3 || precision == SHT_PREC_FP16X3) {
        x->npa = 2; x->npb = 2; x->nprod = 3; x->fp16 = precision == SHT_PREC_FP16X3;
        x->prod = (0u | (0u << 2)) | ((0u | (1u << 2)) << 4) | ((1u | (0u << 2)) << 8);
    } else if (precision == SHT_PREC_BF16X5) {
        x->npa = 3; x->npb = 2; x->nprod = 5;
        x->prod = (0u | (0u << 2)) | ((0u | (1u << 2)) << 4) | ((1u | (0u << 2)) << 8) | ((1u | (1u << 2)) << 12) |
                  ((2u | (0u << 2)) << 16);
    } else {
        return cudaErrorNotSupported;
    }
    x->nlayers = nlayers;
    x->nmax = nlayers <= 256 ? (nlayers + 63) / 64 * 64 : (nlayers + 255) / 256 * 256;
    x->tile_bytes = (int64_t)x->nmax * 128;
    {
        int dev = 0, nsm = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && nsm > 0)
            x->nsm = nsm;
    }
    cudaError_t e;
    auto enc = get_encoder();
    if (!enc) return cudaErrorNotSupported;
    const int64_t zero = 0;
    if ((e = cudaMalloc(&x->d_base, sizeof(int64_t))) != cudaSuccess) return e;
    if ((e = cudaMemcpy(x->d_base, &zero, sizeof(int64_t), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    int max_nkt = 0;
    for (int d = 0; d < 2; ++d) {
        TcMatrixDir& m = x->dir[d];
        m.depth = depth[d];
        m.M = M[d];
        m.Mp = (M[d] + 7) / 8 * 8;
        m.nkt = (depth[d] + BLK - 1) / BLK;
        max_nkt = std::max(max_nkt, m.nkt);
        // fp16: e of max |A| (the whole matrix shares one power-of-two scale)
        int ex = 0;
        if (x->fp16) {
            float* d_mx = nullptr;
            if ((e = cudaMalloc(&d_mx, sizeof(float))) != cudaSuccess) return e;
            cudaMemset(d_mx, 0, sizeof(float));
            absmax_kernel<<<dim3(4 * x->nsm, 1), 256>>>(a[d], (int64_t)depth[d] * M[d], (int64_t)depth[d] * M[d], d_mx);
            float mx = 0.f;
            e = cudaMemcpy(&mx, d_mx, sizeof(float), cudaMemcpyDeviceToHost);
            cudaFree(d_mx);
            if (e != cudaSuccess) return e;
            if (mx > 0.f) std::frexp((double)mx, &ex);
        }
        const int64_t total = (int64_t)m.depth * m.Mp;
        if ((e = cudaMalloc(&m.d_a, std::max<int64_t>(16, total * x->npa * 2))) != cudaSuccess) return e;
        matrix_pieces_kernel<<<4 * x->nsm, 256>>>(a[d], m.depth, m.M, m.Mp, x->npa, x->fp16,
                                                  x->fp16 ? std::ldexp(1.f, F16_TOP - ex) : 1.f, m.d_a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        CUtensorMap map;
        std::memset(&map, 0, sizeof map);
        cuuint64_t dims[3] = {(cuuint64_t)m.Mp, (cuuint64_t)m.depth, (cuuint64_t)x->npa};
        cuuint64_t strides[2] = {(cuuint64_t)m.Mp * 2, (cuuint64_t)m.Mp * 2 * m.depth};
        cuuint32_t box[3] = {BLK, BLK, 1};
        cuuint32_t estr[3] = {1, 1, 1};
        if (enc(&map, x->fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, m.d_a, dims,
                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return cudaErrorInvalidValue;
        if ((e = cudaMalloc(&m.d_map, sizeof(CUtensorMap))) != cudaSuccess) return e;
        if ((e = cudaMemcpy(m.d_map, &map, sizeof map, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&m.d_nkt, sizeof(int32_t))) != cudaSuccess) return e;
        if ((e = cudaMemcpy(m.d_nkt, &m.nkt, sizeof(int32_t), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&m.d_mexp, sizeof(int32_t))) != cudaSuccess) return e;
        if ((e = cudaMemcpy(m.d_mexp, &ex, sizeof(int32_t), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        std::vector<TcItem> items;
        for (int tl = 0; tl * 128 < m.M; ++tl) items.push_back({0, 0, tl, 0});
        m.nitems = (int)items.size();
        if ((e = cudaMalloc(&m.d_items, items.size() * sizeof(TcItem))) != cudaSuccess) return e;
        if ((e = cudaMemcpy(m.d_items, items.data(), items.size() * sizeof(TcItem), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return e;
    }
    const int64_t img_bytes = (int64_t)max_nkt * x->npb * x->tile_bytes;
    if ((e = cudaMalloc(&x->d_img, std::max<int64_t>(16, img_bytes))) != cudaSuccess) return e;
    if ((e = cudaMemset(x->d_img, 0, std::max<int64_t>(16, img_bytes))) != cudaSuccess) return e;
    if (x->fp16) {
        if ((e = cudaMalloc(&x->d_absmax, sizeof(float) * std::max(1, nlayers))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&x->d_kscale, sizeof(float2) * std::max(1, nlayers))) != cudaSuccess) return e;
    }
    if ((e = cudaFuncSetAttribute(legendre_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  227 * 1024)) != cudaSuccess)
        return e;
    return cudaDeviceSynchronize();
}

void tc_matrix_destroy(TcMatrix* x) {
    if (!x) return;
    for (auto& m : x->dir) {
        void* ptrs[] = {m.d_a, m.d_map, m.d_nkt, m.d_mexp, m.d_items};
        for (void* q : ptrs)
            if (q) cudaFree(q);
    }
    void* ptrs[] = {x->d_base, x->d_img, x->d_absmax, x->d_kscale};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    delete x;
}

// out[n ldo + row] = sum_d A[d][row] in[n ld + d] (times row_scale[row]) for n < K.
cudaError_t tc_matrix_apply(const TcMatrix* x, int which, const float* in, int64_t ld, float* out, int64_t ldo, int K,
                            const float* row_scale, int32_t* d_err, cudaStream_t st) {
    const TcMatrixDir& m = x->dir[which];
    if (K <= 0 || K > x->nlayers) return cudaErrorInvalidValue;
    cudaError_t e;
    if (x->fp16) {
        if ((e = cudaMemsetAsync(x->d_absmax, 0, sizeof(float) * K, st)) != cudaSuccess) return e;
        absmax_kernel<<<dim3(std::max(1, 2 * x->nsm / K) * 4, K), 256, 0, st>>>(in, ld, m.depth, x->d_absmax);
        kscale_kernel<<<1, 256, 0, st>>>(x->d_absmax, 1.f, K, x->d_kscale);
    }
    const dim3 ig(m.nkt, (K + 31) / 32);
    if (x->fp16)
        matrix_image_kernel<2, true><<<ig, 256, 0, st>>>(in, ld, m.depth, K, x->d_kscale, x->d_img, x->tile_bytes);
    else
        matrix_image_kernel<2, false><<<ig, 256, 0, st>>>(in, ld, m.depth, K, nullptr, x->d_img, x->tile_bytes);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    TcDev t{};
    t.maps = m.d_map;
    t.syn_tile_base = x->d_base;
    t.nkt = m.d_nkt;
    t.syn_img = x->d_img;
    t.err = d_err;
    t.npa = x->npa;
    t.npb = x->npb;
    t.nprod = x->nprod;
    t.prod = x->prod;
    t.syn_tile_bytes = x->tile_bytes;
    t.nmax = x->nmax;
    t.fp16 = x->fp16;
    t.mexp = m.d_mexp;
    t.kscale_syn = x->d_kscale;
    t.matrix = 1;
    t.mrows = m.M;
    t.mout = out;
    t.ldo = ldo;
    t.row_scale = row_scale;
    t.kchunk = 8;                  // 512-deep accumulation chunks
    const int nct = (K + 255) / 256;
    const int nt_cols = std::min(256, (K + 63) / 64 * 64);
    int stages;
    const int smem = smem_for(x->npa, x->npb, nt_cols, stages);
    legendre_tc_kernel<true><<<dim3(std::min(m.nitems, x->nsm), nct), TC_THREADS, smem, st>>>(
        t, m.d_items, m.nitems, K, 256, nt_cols, stages, tmem_cols_for(nt_cols), 0, nullptr, nullptr, 0, 0);
    return cudaGetLastError();
}

// Column tile width of a tensor-core plan's Legendre GEMMs: 128 (one tile for 64 layers)
// or 64. Each output column is computed alike in either; the speed differs.
int tc_tile_cols(const Plan& p) { return p.tc ? static_cast<const TcState*>(p.tc)->ctw : 0; }
bool tc_set_tile_cols(Plan& p, int cols) {
    if (!p.tc || (cols != 64 && cols != kTcTileCols)) return false;
    static_cast<TcState*>(p.tc)->ctw = cols;
    return true;
}

cudaError_t tc_analysis_scale(const Plan& p, const float* grid, int64_t ldg, int K, cudaStream_t st, float mul) {
    const TcState* s = static_cast<const TcState*>(p.tc);
    if (!s || !s->fp16 || K <= 0) return cudaSuccess;
    float* out = s->d_absmax + p.d.nlayers;
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(float) * K, st);
    if (e != cudaSuccess) return e;
    absmax_kernel<<<dim3(std::max(1, 2 * s->nsm / std::max(1, K)) * 4, K), 256, 0, st>>>(grid, ldg, p.npoints, out);
    kscale_kernel<<<1, 256, 0, st>>>(out, mul > 0.f ? mul : s->ana_mul, K, s->d_kscale + p.d.nlayers);
    return cudaGetLastError();
}

cudaError_t launch_legendre_analysis_tc(const Plan& p, float2* coeffs, int64_t ldc, int K, bool add, cudaStream_t st) {
    const TcState& s = *static_cast<const TcState*>(p.tc);
    if (s.n_ana_items == 0) return cudaSuccess;
    const TcDev t = make_dev(p);
    const int ncols = 2 * K;
    const int nct = (ncols + s.ctw - 1) / s.ctw;
    const int nt_cols = std::min(s.ctw, (ncols + 63) / 64 * 64);
    int stages;
    const int smem = smem_for(s.npa, s.npb, nt_cols, stages);
    legendre_tc_kernel<false><<<dim3(std::min(s.n_ana_items, s.nsm), nct), TC_THREADS, smem, st>>>(
        t, s.d_ana_items, s.n_ana_items, K, s.ctw, nt_cols, stages, tmem_cols_for(nt_cols), 1, nullptr, coeffs,
        ldc, add ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace sht
