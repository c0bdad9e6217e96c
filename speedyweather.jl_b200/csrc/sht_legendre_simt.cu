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
// with c running over the 2K real columns (re, im of each layer). One CTA
// computes a 64 x 128 tile of one parity with register tiles of 8 x 8 per thread.
#include "sht_internal.h"

namespace sht {

namespace {

constexpr int BM = 64;    // rings (synthesis) or parity rows (analysis) per CTA
constexpr int BN = 128;   // real columns per CTA (64 complex layers)
constexpr int BK = 8;     // contraction depth per shared-memory stage
constexpr int NT = 128;   // threads

__global__ void __launch_bounds__(NT) legendre_synthesis_fp32_kernel(
    const LegItem* __restrict__ items, const float* __restrict__ lam, const int64_t* __restrict__ lam_off,
    const int32_t* __restrict__ rows_of, const int64_t* __restrict__ lm_off, const RingDesc* __restrict__ rings,
    int nh, int nh_pad, int lmax, const float2* __restrict__ coeffs, int64_t ldc, float2* __restrict__ four, int K) {
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    const LegItem it = items[blockIdx.x];
    const int m = it.m;
    const int par = blockIdx.z;
    const int j0 = it.tile * BM;
    const int kt0 = blockIdx.y * (BN / 2);
    const int rows = rows_of[m];
    const float* L = lam + lam_off[m] + (int64_t)par * rows * nh_pad;
    const int64_t lmo = lm_off[m];
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;   // 16 column groups x 8 row groups

    // global load mapping
    const int a_i = t / 16, a_j = (t % 16) * 4;   // one float4 of Lam per thread
    const int b_k = t % 64, b_i0 = (t / 64);     // 4 complex coefficients per thread

    float acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.f;

    auto load_tiles = [&](int i0, float4& ra, float2 (&rb)[4]) {
        const int i = i0 + a_i;
        ra = (i < rows) ? *reinterpret_cast<const float4*>(L + (int64_t)i * nh_pad + j0 + a_j)
                        : make_float4(0.f, 0.f, 0.f, 0.f);
        const int k = kt0 + b_k;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int ii = i0 + b_i0 + 2 * q;
            const int l = m + 2 * ii + par;
            rb[q] = (ii < rows && l < lmax && k < K) ? coeffs[(int64_t)k * ldc + lmo + 2 * ii + par]
                                                     : make_float2(0.f, 0.f);
        }
    };
    auto store_tiles = [&](int buf, const float4& ra, const float2 (&rb)[4]) {
        *reinterpret_cast<float4*>(&As[buf][a_i][a_j]) = ra;
#pragma unroll
        for (int q = 0; q < 4; ++q) *reinterpret_cast<float2*>(&Bs[buf][b_i0 + 2 * q][2 * b_k]) = rb[q];
    };

    float4 ra;
    float2 rb[4];
    load_tiles(0, ra, rb);
    store_tiles(0, ra, rb);
    __syncthreads();
    int buf = 0;
    for (int i0 = 0; i0 < rows; i0 += BK) {
        const bool more = i0 + BK < rows;
        if (more) load_tiles(i0 + BK, ra, rb);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][32 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
        }
        if (more) {
            store_tiles(buf ^ 1, ra, rb);
            __syncthreads();
            buf ^= 1;
        }
    }
    // epilogue: rows -> rings, column pairs -> complex layers
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int j = j0 + (r < 4 ? ty * 4 + r : 32 + ty * 4 + (r - 4));
        if (j >= nh) continue;
        const RingDesc& rd = rings[j];
        if (m > rd.mt) continue;
        float2* dst = four + ((rd.gofs + m) * 2 + par) * K;
#pragma unroll
        for (int cp = 0; cp < 4; ++cp) {
            const int col = (cp < 2 ? tx * 4 + 2 * cp : 64 + tx * 4 + 2 * (cp - 2));
            const int k = kt0 + col / 2;
            if (k < K) dst[k] = make_float2(acc[r][2 * cp], acc[r][2 * cp + 1]);
        }
    }
    (void)nh_pad;
}

__global__ void __launch_bounds__(NT) legendre_analysis_fp32_kernel(
    const LegItem* __restrict__ items, const float* __restrict__ lam, const int64_t* __restrict__ lam_off,
    const int32_t* __restrict__ rows_of, const int32_t* __restrict__ j0_of, const int64_t* __restrict__ lm_off,
    const RingDesc* __restrict__ rings, int nh, int nh_pad, int lmax, const float2* __restrict__ four,
    float2* __restrict__ coeffs, int64_t ldc, int K, int add) {
    __shared__ __align__(16) float As[2][BK][BM];
    __shared__ __align__(16) float Bs[2][BK][BN];
    const LegItem it = items[blockIdx.x];
    const int m = it.m;
    const int par = blockIdx.z;
    const int i_base = it.tile * BM;
    const int kt0 = blockIdx.y * (BN / 2);
    const int rows = rows_of[m];
    const float* L = lam + lam_off[m] + (int64_t)par * rows * nh_pad;
    const int64_t lmo = lm_off[m];
    const int jstart = (j0_of[m] / BK) * BK;
    const int t = threadIdx.x;
    const int tx = t % 16, ty = t / 16;

    const int a_i = t / 2, a_j = (t % 2) * 4;     // 64 rows x 8 rings: one float4 per thread
    const int b_k = t % 64, b_j0 = t / 64;       // 4 complex per thread

    float acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[r][c] = 0.f;

    auto load_tiles = [&](int jc, float4& ra, float2 (&rb)[4]) {
        const int i = i_base + a_i;
        ra = (i < rows && jc < nh) ? *reinterpret_cast<const float4*>(L + (int64_t)i * nh_pad + jc + a_j)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
        const int k = kt0 + b_k;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = jc + b_j0 + 2 * q;
            float2 v = make_float2(0.f, 0.f);
            if (j < nh && k < K) {
                const RingDesc& rd = rings[j];
                if (m <= rd.mt) v = four[((rd.gofs + m) * 2 + par) * K + k];
            }
            rb[q] = v;
        }
    };
    auto store_tiles = [&](int buf, const float4& ra, const float2 (&rb)[4]) {
        As[buf][a_j + 0][a_i] = ra.x;
        As[buf][a_j + 1][a_i] = ra.y;
        As[buf][a_j + 2][a_i] = ra.z;
        As[buf][a_j + 3][a_i] = ra.w;
#pragma unroll
        for (int q = 0; q < 4; ++q) *reinterpret_cast<float2*>(&Bs[buf][b_j0 + 2 * q][2 * b_k]) = rb[q];
    };

    float4 ra;
    float2 rb[4];
    load_tiles(jstart, ra, rb);
    store_tiles(0, ra, rb);
    __syncthreads();
    int buf = 0;
    for (int jc = jstart; jc < nh; jc += BK) {
        const bool more = jc + BK < nh;
        if (more) load_tiles(jc + BK, ra, rb);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][kk][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][kk][32 + ty * 4]);
            const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][kk][tx * 4]);
            const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][kk][64 + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int c = 0; c < 8; ++c) acc[r][c] = fmaf(av[r], bv[c], acc[r][c]);
        }
        if (more) {
            store_tiles(buf ^ 1, ra, rb);
            __syncthreads();
            buf ^= 1;
        }
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = i_base + (r < 4 ? ty * 4 + r : 32 + ty * 4 + (r - 4));
        const int l = m + 2 * i + par;
        if (i >= rows || l >= lmax) continue;
#pragma unroll
        for (int cp = 0; cp < 4; ++cp) {
            const int col = (cp < 2 ? tx * 4 + 2 * cp : 64 + tx * 4 + 2 * (cp - 2));
            const int k = kt0 + col / 2;
            if (k >= K) continue;
            float2* dst = coeffs + (int64_t)k * ldc + lmo + 2 * i + par;
            float2 v = make_float2(acc[r][2 * cp], acc[r][2 * cp + 1]);
            if (add) {
                const float2 o = *dst;
                v.x += o.x;
                v.y += o.y;
            }
            *dst = v;
        }
    }
    (void)nh_pad;
}

}  // namespace

cudaError_t launch_legendre_synthesis_fp32(const Plan& p, const float2* coeffs, int64_t ldc, int K, cudaStream_t s) {
    if (p.n_syn_items == 0) return cudaSuccess;
    dim3 g(p.n_syn_items, (2 * K + BN - 1) / BN, 2);
    legendre_synthesis_fp32_kernel<<<g, NT, 0, s>>>(p.d_syn_items, p.d_lam, p.d_lam_off, p.d_rows, p.d_lm_off,
                                                    p.d_rings, p.nh, p.nh_pad, p.lmax, coeffs, ldc, p.d_four, K);
    return cudaGetLastError();
}

cudaError_t launch_legendre_analysis_fp32(const Plan& p, float2* coeffs, int64_t ldc, int K, bool add,
                                          cudaStream_t s) {
    if (p.n_ana_items == 0) return cudaSuccess;
    dim3 g(p.n_ana_items, (2 * K + BN - 1) / BN, 2);
    legendre_analysis_fp32_kernel<<<g, NT, 0, s>>>(p.d_ana_items, p.d_lam, p.d_lam_off, p.d_rows, p.d_j0,
                                                   p.d_lm_off, p.d_rings, p.nh, p.nh_pad, p.lmax, p.d_four, coeffs,
                                                   ldc, K, add ? 1 : 0);
    return cudaGetLastError();
}

}  // namespace sht

namespace sht {
// The FP32 Legendre analysis reading the Fourier coefficients from a caller-chosen
// scratch (used by the static-scratch analysis entry point).
cudaError_t launch_legendre_analysis_fp32_from(const Plan& p, const float2* scratch, float2* coeffs, int64_t ldc,
                                               int K, bool add, cudaStream_t s) {
    if (p.n_ana_items == 0) return cudaSuccess;
    dim3 g(p.n_ana_items, (2 * K + BN - 1) / BN, 2);
    legendre_analysis_fp32_kernel<<<g, NT, 0, s>>>(p.d_ana_items, p.d_lam, p.d_lam_off, p.d_rows, p.d_j0, p.d_lm_off,
                                                   p.d_rings, p.nh, p.nh_pad, p.lmax, scratch, coeffs, ldc, K,
                                                   add ? 1 : 0);
    return cudaGetLastError();
}
}  // namespace sht
