// Legendre stage in FP32 on the CUDA cores (the plain form, matching the
// reference's Float32 arithmetic).
//
// Replaces SpeedyTransforms/src/legendre.jl:2-195 (CPU even/odd fused matvec and
// outer-product accumulate) and SpeedyTransforms/src/legendre_ka.jl:19-200 (the
// one-thread-per-output KernelAbstractions kernels).
//
// For every order m the stage is a pair of dense GEMMs, one per parity of l - m
// (the north/south symmetry lambda_lm(-x) = (-1)^(l-m) lambda_lm(x)):
//   synthesis  X_p[j, c] = sum_i Lam[m][p][i][j] * a[m + 2i + p, c]      -> E (p=0), O (p=1)
//   analysis   a[m + 2i + p, c] = sum_j Lam[m][p][i][j] * Y_p[j, c]      Y_0 = E, Y_1 = O
// with c running over the 2K real columns (re, im of each layer). One CTA of 128
// threads computes a 64 x BN tile of one parity (BN = 32, 64 or 128 real columns,
// register tiles of 8 x BN/16 per thread). The contraction runs in steps of 8 in the
// same order for every BN, so the tile width changes the speed, not the result: the
// autotuner picks it per plan and direction, and the grouped launch of a batch of
// transforms (one CTA loop over the tiles of all of them) reuses the same tile bodies.
#include "sht_internal.h"

namespace sht {

namespace {

constexpr int BM = 64;    // rings (synthesis) or parity rows (analysis) per CTA
constexpr int BK = 8;     // contraction depth per shared-memory stage
constexpr int NT = 128;   // threads
constexpr int SS = 3;     // shared-memory stages of the tiles (asynchronous copies)
constexpr int BPAD = 4;   // floats of padding per B row: the synthesis copies of 8 rows land in distinct banks

__device__ __forceinline__ void cp_async_zfill(void* dst, const void* src, int bytes, int src_bytes) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int N>
struct Vec;
template <>
struct Vec<2> {
    static __device__ __forceinline__ void ld(const float* p, float* v) {
        const float2 a = *reinterpret_cast<const float2*>(p);
        v[0] = a.x;
        v[1] = a.y;
    }
};
template <>
struct Vec<4> {
    static __device__ __forceinline__ void ld(const float* p, float* v) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    }
};

// 8 x TN register tile, TN = BN / 16: rows ty*4 + {0..3} and 32 + ty*4 + {0..3};
// columns tx*H + {0..H-1} and BN/2 + tx*H + {0..H-1} (H = TN/2, TN >= 4) or
// tx*2 + {0, 1} (TN = 2); tx < 16, ty < 8. Columns 2c, 2c + 1 of a thread are the
// re, im parts of one layer.
template <int BN>
struct Cols {
    static constexpr int TN = BN / 16;
    static constexpr bool SPLIT = TN >= 4;
    static constexpr int H = SPLIT ? TN / 2 : TN;
    static __device__ __forceinline__ int col(int tx, int c) {
        return SPLIT ? (c < H ? tx * H + c : BN / 2 + tx * H + (c - H)) : tx * TN + c;
    }
};

template <int BN>
__device__ __forceinline__ void mma_step(const float (&As)[BK][BM], const float (&Bs)[BK][BN + BPAD], int tx, int ty,
                                         float (&acc)[8][BN / 16]) {
    constexpr int TN = Cols<BN>::TN, H = Cols<BN>::H;
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
        const float4 a0 = *reinterpret_cast<const float4*>(&As[kk][ty * 4]);
        const float4 a1 = *reinterpret_cast<const float4*>(&As[kk][32 + ty * 4]);
        float bv[TN];
        if constexpr (Cols<BN>::SPLIT) {
            Vec<H>::ld(&Bs[kk][tx * H], bv);
            Vec<H>::ld(&Bs[kk][BN / 2 + tx * H], bv + H);
        } else {
            Vec<TN>::ld(&Bs[kk][tx * TN], bv);
        }
        const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int c = 0; c < TN; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
    }
}

template <int BN>
__device__ __forceinline__ int col_of(int tx, int c) {
    return Cols<BN>::col(tx, c);
}

template <int BN>
__device__ void syn_tile(const LegView& v, int m, int tile, int ct, int par, float (&As)[SS][BK][BM],
                         float (&Bs)[SS][BK][BN + BPAD]) {
    constexpr int TN = BN / 16;
    constexpr int NB = BN / 32;                   // complex coefficients per thread and stage
    const int j0 = tile * BM;
    const int kt0 = ct * (BN / 2);
    const int rows = v.rows[m];
    const float* L = v.lam + v.lam_off[m] + (int64_t)par * rows * v.nh_pad;
    const int64_t lmo = v.lm_off[m];
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;
    const int a_i = t / 16, a_j = (t % 16) * 4;   // one float4 of Lam per thread
    // B copies: lane (row b_r of the step, layer group b_g); a warp reads 4 layers x 8 rows,
    // i.e. 4 runs of 128 contiguous bytes of the coefficients, per instruction
    const int b_r = t % BK, b_g = t / BK;         // b_g < 16; layers b_g + 16 q
    static_assert(NT / BK == 16 && BN / 2 == 16 * (BN / 32), "16 layer groups of NB layers");

    float acc[8][TN];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) acc[r][c] = 0.f;

    // SS-stage pipeline of asynchronous copies into shared memory (zero-filled outside the
    // order's rows and degrees): the copies of step st + SS - 1 are in flight while step st
    // computes; the contraction order is the same as with any other staging
    const float* La = L + j0 + a_j;
    auto issue = [&](int step) {
        const int stg = step % SS, i0 = step * BK;
        const int i = i0 + a_i;
        const bool aok = i < rows;
        cp_async_zfill(&As[stg][a_i][a_j], aok ? La + (int64_t)i * v.nh_pad : L, 16, aok ? 16 : 0);
        const int ii = i0 + b_r;
        const bool rok = ii < rows && m + 2 * ii + par < v.lmax;
#pragma unroll
        for (int q = 0; q < NB; ++q) {
            const int kl = b_g + 16 * q;
            const int kb = kt0 + kl;
            const bool bok = rok && kb < v.K;
            cp_async_zfill(&Bs[stg][b_r][2 * kl],
                           bok ? (const void*)(v.cin + (int64_t)kb * v.ldc + lmo + 2 * ii + par) : (const void*)v.cin, 8,
                           bok ? 8 : 0);
        }
        cp_async_commit();
    };
    const int nsteps = (rows + BK - 1) / BK;
    __syncthreads();                               // the previous tile's reads of As/Bs are done
#pragma unroll
    for (int st = 0; st < SS - 1; ++st) {
        if (st < nsteps) issue(st);
        else cp_async_commit();
    }
    for (int st = 0; st < nsteps; ++st) {
        cp_async_wait<SS - 2>();                   // this thread's copies of step st have landed
        __syncthreads();                           // everyone's; step st - 1's stage is free
        if (st + SS - 1 < nsteps) issue(st + SS - 1);
        else cp_async_commit();
        mma_step<BN>(As[st % SS], Bs[st % SS], tx, ty, acc);
    }
    // epilogue: rows -> rings, column pairs -> complex layers
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int j = j0 + (r < 4 ? ty * 4 + r : 32 + ty * 4 + (r - 4));
        if (j >= v.nh) continue;
        const RingDesc& rd = v.rings[j];
        if (m > rd.mt) continue;
        float2* dst = v.four + ((rd.gofs + m) * 2 + par) * v.K;
#pragma unroll
        for (int c = 0; c < TN; c += 2) {
            const int k = kt0 + col_of<BN>(tx, c) / 2;
            if (k < v.K) dst[k] = make_float2(acc[r][c], acc[r][c + 1]);
        }
    }
}

// mma_step with A stored row-major, [BM][BK] (rows i, BK rings each), as the analysis
// copies Lam rows straight into shared memory: four k at a time, a float4 per row.
// The FMA order per accumulator (k ascending) is that of mma_step.
template <int BN>
__device__ __forceinline__ void mma_step_rows(const float (&Ar)[BM][BK], const float (&Bs)[BK][BN + BPAD], int tx, int ty,
                                              float (&acc)[8][BN / 16]) {
    constexpr int TN = Cols<BN>::TN, H = Cols<BN>::H;
#pragma unroll
    for (int kq = 0; kq < BK; kq += 4) {
        float4 a[8];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            a[r] = *reinterpret_cast<const float4*>(&Ar[ty * 4 + r][kq]);
            a[4 + r] = *reinterpret_cast<const float4*>(&Ar[32 + ty * 4 + r][kq]);
        }
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int kk = kq + e;
            float bv[TN];
            if constexpr (Cols<BN>::SPLIT) {
                Vec<H>::ld(&Bs[kk][tx * H], bv);
                Vec<H>::ld(&Bs[kk][BN / 2 + tx * H], bv + H);
            } else {
                Vec<TN>::ld(&Bs[kk][tx * TN], bv);
            }
            float av[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) av[r] = e == 0 ? a[r].x : e == 1 ? a[r].y : e == 2 ? a[r].z : a[r].w;
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < TN; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
        }
    }
}

template <int BN>
__device__ void ana_tile(const LegView& v, int m, int tile, int ct, int par, float (&As)[SS][BK][BM],
                         float (&Bs)[SS][BK][BN + BPAD]) {
    constexpr int TN = BN / 16;
    constexpr int NB = BN / 32;
    const int i_base = tile * BM;
    const int kt0 = ct * (BN / 2);
    const int rows = v.rows[m];
    const float* L = v.lam + v.lam_off[m] + (int64_t)par * rows * v.nh_pad;
    const int64_t lmo = v.lm_off[m];
    const int j0m = v.j0[m];
    const int jstart = (j0m / BK) * BK;
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;
    const int a_i = t / 2, a_j = (t % 2) * 4;     // 64 rows x 8 rings: one 16-byte copy per thread
    const int b_k = t % (BN / 2), b_j0 = t / (BN / 2);
    constexpr int BSTEP = NT / (BN / 2);
    // Lam rows land as they are stored (rows i, rings j): [SS][BM][BK] over the same bytes
    float (&Ar)[SS][BM][BK] = *reinterpret_cast<float (*)[SS][BM][BK]>(&As);

    float acc[8][TN];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < TN; ++c) acc[r][c] = 0.f;

    // SS-stage pipeline of asynchronous copies (zero-filled outside the order's rows and
    // the rings that carry it), as in syn_tile
    const int k = kt0 + b_k;
    const int i = i_base + a_i;
    auto issue = [&](int step) {
        const int stg = step % SS, jc = jstart + step * BK;
        const bool aok = i < rows && jc < v.nh;
        cp_async_zfill(&Ar[stg][a_i][a_j], aok ? L + (int64_t)i * v.nh_pad + jc + a_j : L, 16, aok ? 16 : 0);
#pragma unroll
        for (int q = 0; q < NB; ++q) {
            const int j = jc + b_j0 + BSTEP * q;
            // rings j >= j0(m) carry order m (m <= mt(j)); one load of the ring's scratch base
            const bool bok = j < v.nh && k < v.K && j >= j0m;
            cp_async_zfill(&Bs[stg][b_j0 + BSTEP * q][2 * b_k],
                           bok ? (const void*)(v.four + ((__ldg(v.gofs + j) + m) * 2 + par) * v.K + k)
                               : (const void*)v.four,
                           8, bok ? 8 : 0);
        }
        cp_async_commit();
    };
    const int nsteps = (v.nh - jstart + BK - 1) / BK;
    __syncthreads();                               // the previous tile's reads of As/Bs are done
#pragma unroll
    for (int st = 0; st < SS - 1; ++st) {
        if (st < nsteps) issue(st);
        else cp_async_commit();
    }
    for (int st = 0; st < nsteps; ++st) {
        cp_async_wait<SS - 2>();                   // this thread's copies of step st have landed
        __syncthreads();                           // everyone's; step st - 1's stage is free
        if (st + SS - 1 < nsteps) issue(st + SS - 1);
        else cp_async_commit();
        mma_step_rows<BN>(Ar[st % SS], Bs[st % SS], tx, ty, acc);
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = i_base + (r < 4 ? ty * 4 + r : 32 + ty * 4 + (r - 4));
        const int l = m + 2 * i + par;
        if (i >= rows || l >= v.lmax) continue;
#pragma unroll
        for (int c = 0; c < TN; c += 2) {
            const int k = kt0 + col_of<BN>(tx, c) / 2;
            if (k >= v.K) continue;
            float2* dst = v.cout + (int64_t)k * v.ldc + lmo + 2 * i + par;
            float2 x = make_float2(acc[r][c], acc[r][c + 1]);
            if (v.add) {
                const float2 o = *dst;
                x.x += o.x;
                x.y += o.y;
            }
            *dst = x;
        }
    }
}

template <int BN>
__global__ void __launch_bounds__(NT) legendre_synthesis_fp32_kernel(const LegItem* __restrict__ items,
                                                                     const LegView v) {
    __shared__ __align__(16) float As[SS][BK][BM];
    __shared__ __align__(16) float Bs[SS][BK][BN + BPAD];
    const LegItem it = items[blockIdx.x];
    syn_tile<BN>(v, it.m, it.tile, blockIdx.y, blockIdx.z, As, Bs);
}

template <int BN>
__global__ void __launch_bounds__(NT) legendre_analysis_fp32_kernel(const LegItem* __restrict__ items,
                                                                    const LegView v) {
    __shared__ __align__(16) float As[SS][BK][BM];
    __shared__ __align__(16) float Bs[SS][BK][BN + BPAD];
    const LegItem it = items[blockIdx.x];
    ana_tile<BN>(v, it.m, it.tile, blockIdx.y, blockIdx.z, As, Bs);
}

// Persistent grouped launch over the tiles of many transforms: CTA b takes the items
// b, b + gridDim.x, ... of the batch's list (task, m, tile, column tile, parity).
template <int BN>
__global__ void __launch_bounds__(NT) legendre_grouped_kernel(const LegView* __restrict__ views,
                                                              const GroupItem* __restrict__ items, int nitems,
                                                              int synthesis) {
    __shared__ __align__(16) float As[SS][BK][BM];
    __shared__ __align__(16) float Bs[SS][BK][BN + BPAD];
    for (int ix = blockIdx.x; ix < nitems; ix += gridDim.x) {
        const GroupItem it = items[ix];
        const LegView& v = views[it.task];
        if (synthesis)
            syn_tile<BN>(v, it.a, it.b, it.c >> 1, it.c & 1, As, Bs);
        else
            ana_tile<BN>(v, it.a, it.b, it.c >> 1, it.c & 1, As, Bs);
    }
}

template <int BN>
cudaError_t launch_syn(const Plan& p, const LegView& v, cudaStream_t s) {
    dim3 g(p.n_syn_items, (2 * v.K + BN - 1) / BN, 2);
    legendre_synthesis_fp32_kernel<BN><<<g, NT, 0, s>>>(p.d_syn_items, v);
    return cudaGetLastError();
}
template <int BN>
cudaError_t launch_ana(const Plan& p, const LegView& v, const LegItem* items, int nitems, cudaStream_t s) {
    dim3 g(nitems, (2 * v.K + BN - 1) / BN, 2);
    legendre_analysis_fp32_kernel<BN><<<g, NT, 0, s>>>(items, v);
    return cudaGetLastError();
}

}  // namespace

LegView leg_view(const Plan& p, const float2* cin, float2* cout, int64_t ldc, const float2* four, int K, bool add) {
    LegView v{};
    v.lam = p.d_lam;
    v.lam_off = p.d_lam_off;
    v.rows = p.d_rows;
    v.j0 = p.d_j0;
    v.lm_off = p.d_lm_off;
    v.rings = p.d_rings;
    v.gofs = p.d_gofs;
    v.nh = p.nh;
    v.nh_pad = p.nh_pad;
    v.lmax = p.lmax;
    v.cin = cin;
    v.cout = cout;
    v.ldc = ldc;
    v.four = const_cast<float2*>(four);
    v.K = K;
    v.add = add ? 1 : 0;
    return v;
}

cudaError_t launch_legendre_synthesis_fp32(const Plan& p, const float2* coeffs, int64_t ldc, int K, cudaStream_t s) {
    if (p.n_syn_items == 0 || K == 0) return cudaSuccess;
    const LegView v = leg_view(p, coeffs, nullptr, ldc, p.d_four, K, false);
    switch (p.leg_bn_syn) {
        case 32: return launch_syn<32>(p, v, s);
        case 64: return launch_syn<64>(p, v, s);
        default: return launch_syn<128>(p, v, s);
    }
}

cudaError_t launch_legendre_analysis_fp32(const Plan& p, float2* coeffs, int64_t ldc, int K, bool add,
                                          cudaStream_t s) {
    return launch_legendre_analysis_fp32_from(p, p.d_four, coeffs, ldc, K, add, s);
}

// The FP32 Legendre analysis reading the Fourier coefficients from a caller-chosen
// scratch (the static-scratch analysis entry point uses it).
cudaError_t launch_legendre_analysis_fp32_from(const Plan& p, const float2* scratch, float2* coeffs, int64_t ldc,
                                               int K, bool add, cudaStream_t s) {
    if (p.n_ana_items == 0 || K == 0) return cudaSuccess;
    const LegView v = leg_view(p, nullptr, coeffs, ldc, scratch, K, add);
    switch (p.leg_bn_ana) {
        case 32: return launch_ana<32>(p, v, p.d_ana_items, p.n_ana_items, s);
        case 64: return launch_ana<64>(p, v, p.d_ana_items, p.n_ana_items, s);
        default: return launch_ana<128>(p, v, p.d_ana_items, p.n_ana_items, s);
    }
}

// Persistent grid of the grouped launch per tile width (32, 64, 128): the SMs times
// the CTAs that fit on one.
cudaError_t legendre_grouped_grids(int nsm, int (&grid)[3]) {
    int occ = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, legendre_grouped_kernel<32>, NT, 0);
    if (e != cudaSuccess) return e;
    grid[0] = nsm * std::max(1, occ);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, legendre_grouped_kernel<64>, NT, 0)) != cudaSuccess)
        return e;
    grid[1] = nsm * std::max(1, occ);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, legendre_grouped_kernel<128>, NT, 0)) != cudaSuccess)
        return e;
    grid[2] = nsm * std::max(1, occ);
    return cudaSuccess;
}

cudaError_t launch_legendre_grouped(const LegView* views, const GroupItem* items, int nitems, int bn, bool synthesis,
                                    int grid, cudaStream_t s) {
    if (nitems == 0) return cudaSuccess;
    const int g = std::max(1, std::min(nitems, grid));
    switch (bn) {
        case 32: legendre_grouped_kernel<32><<<g, NT, 0, s>>>(views, items, nitems, synthesis ? 1 : 0); break;
        case 64: legendre_grouped_kernel<64><<<g, NT, 0, s>>>(views, items, nitems, synthesis ? 1 : 0); break;
        default: legendre_grouped_kernel<128><<<g, NT, 0, s>>>(views, items, nitems, synthesis ? 1 : 0); break;
    }
    return cudaGetLastError();
}

}  // namespace sht
