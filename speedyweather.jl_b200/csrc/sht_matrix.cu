// Dense-matrix spectral transforms: MatrixSpectralTransform.
//
// Replaces SpeedyTransforms/src/matrix_transform.jl:56-260. As there, the matrices are
// the transforms of unit vectors (forward_matrix!, backward_matrix!, :134-173), here
// computed by this library's FP32 transforms on the GPU, 256 unit columns per call,
// written directly in the layouts the products read:
//   F^T [npoints][2 nlm]  row ij = analysis of the unit grid vector e_ij, as floats
//                         (re, im of each coefficient), so coeffs = F^T-product of field
//   B_r [2 nlm][npoints]  row 2lm = synthesis of coeffs e_lm (= Re B[:, lm]), row 2lm+1 =
//                         synthesis of i e_lm (= -Im B[:, lm]), so field = B_r-product of
//                         the coefficients viewed as floats (Re B Re c - Im B Im c)
// Products: with an SHT_PREC_FP32 description three TF32 products on the tensor cores
// (sht_matrix_tf32.cu: the matrix streamed once as FP32 and split in shared memory; the
// reference's Float32 mul!, :206-258); with a split 16-bit precision the persistent
// tcgen05 kernel of sht_legendre_tc.cu in its matrix mode (the matrix in 16-bit pieces
// by TMA, the layers as the N columns). unscale_coslat scales the synthesised rings by
// 1/cos(lat) (:255-257), in the products' epilogue.


#include <cmath>
#include <vector>

#include "sht_internal.h"

namespace sht {
const Plan* plan_impl(const sht_plan* plan);
int set_error(int code, const char* msg);
}  // namespace sht

using namespace sht;

struct sht_matrix {
    sht_plan* base = nullptr;         // FP32 transform the matrices are built with
    sht_desc d{};
    int64_t npoints = 0, nlm = 0;
    float* d_F = nullptr;             // F^T [npoints][2 nlm] (freed once the products' operands exist)
    float* d_B = nullptr;             // B_r [2 nlm][npoints]
    float* d_row_scale = nullptr;     // [npoints]: 1 / cos(lat) of the point's ring
    int32_t* d_err = nullptr;
    TcMatrix* tc = nullptr;           // split 16-bit precisions
    MxTf32* mx = nullptr;             // SHT_PREC_FP32
};

namespace {

thread_local char g_msg[512];

int mfail(int code, const char* what) { return set_error(code, what); }
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

// x[k ld + first + k] = 1 for k < K (the rest zeroed beforehand): K unit columns
__global__ void unit_columns_kernel(float* x, int64_t ld, int K, int64_t first) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < K) x[(int64_t)k * ld + first + k] = 1.f;
}

void release(sht_matrix* m) {
    if (m->tc) tc_matrix_destroy(m->tc);
    if (m->mx) mx_tf32_destroy(m->mx);
    void* ptrs[] = {m->d_F, m->d_B, m->d_row_scale, m->d_err};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (m->base) sht_plan_destroy(m->base);
}

int build(sht_matrix* m) {
    constexpr int CH = 256;
    sht_desc bd = m->d;
    bd.precision = SHT_PREC_FP32;
    bd.nlayers = CH;
    int rc = sht_plan_create(&bd, &m->base);
    if (rc != SHT_OK) return rc;
    const Plan& p = *plan_impl(m->base);
    m->npoints = p.npoints;
    m->nlm = p.nlm;
    const int64_t np = p.npoints, n2 = 2 * p.nlm;
    cudaError_t e;
    if ((e = cudaMalloc(&m->d_F, np * n2 * sizeof(float))) != cudaSuccess) return mcuda(e, "sht_matrix_create");
    if ((e = cudaMalloc(&m->d_B, np * n2 * sizeof(float))) != cudaSuccess) return mcuda(e, "sht_matrix_create");
    float* unit = nullptr;
    const int64_t unit_floats = (int64_t)CH * std::max(np, n2);
    if ((e = cudaMalloc(&unit, unit_floats * sizeof(float))) != cudaSuccess) return mcuda(e, "sht_matrix_create");
    // F^T: analyses of unit grid vectors, rows c0 .. c0 + K - 1
    for (int64_t c0 = 0; c0 < np && rc == SHT_OK; c0 += CH) {
        const int K = (int)std::min<int64_t>(CH, np - c0);
        cudaMemset(unit, 0, (int64_t)K * np * sizeof(float));
        unit_columns_kernel<<<(K + 127) / 128, 128>>>(unit, np, K, c0);
        rc = sht_analyze(m->base, unit, np, m->d_F + c0 * n2, p.nlm, K, 0, nullptr);
    }
    // B_r: syntheses of unit coefficients (re, then im, of each lm), rows q0 .. q0 + K - 1
    for (int64_t q0 = 0; q0 < n2 && rc == SHT_OK; q0 += CH) {
        const int K = (int)std::min<int64_t>(CH, n2 - q0);
        cudaMemset(unit, 0, (int64_t)K * n2 * sizeof(float));
        unit_columns_kernel<<<(K + 127) / 128, 128>>>(unit, n2, K, q0);
        rc = sht_synthesize(m->base, unit, p.nlm, m->d_B + q0 * np, np, K, 0, nullptr);
    }
    cudaFree(unit);
    if (rc != SHT_OK) return rc;
    // 1 / cos(lat) per grid point (ring-major north to south)
    std::vector<float> rs(np);
    {
        int64_t ij = 0;
        for (int j = 0; j < p.nlat; ++j) {
            const float c = (float)(1.0 / std::cos(p.latd[j] * M_PI / 180.0));
            for (int i = 0; i < p.nlons[j]; ++i) rs[ij++] = c;
        }
    }
    if ((e = cudaMalloc(&m->d_row_scale, np * sizeof(float))) != cudaSuccess) return mcuda(e, "sht_matrix_create");
    if ((e = cudaMemcpy(m->d_row_scale, rs.data(), np * sizeof(float), cudaMemcpyHostToDevice)) != cudaSuccess)
        return mcuda(e, "sht_matrix_create");
    if ((e = cudaMalloc(&m->d_err, sizeof(int32_t))) != cudaSuccess) return mcuda(e, "sht_matrix_create");
    cudaMemset(m->d_err, 0, sizeof(int32_t));
    const float* a[2] = {m->d_F, m->d_B};
    const int depth[2] = {(int)np, (int)n2};
    const int M[2] = {(int)n2, (int)np};
    if (m->d.precision == SHT_PREC_FP32) {
        if ((e = mx_tf32_create(&m->mx, a, depth, M, m->d.nlayers)) != cudaSuccess)
            return mcuda(e, "sht_matrix_create (TF32 matrices)");
    } else if ((e = tc_matrix_create(&m->tc, m->d.precision, a, depth, M, m->d.nlayers)) != cudaSuccess) {
        return mcuda(e, "sht_matrix_create (tensor-core matrices)");
    }
    cudaFree(m->d_F);                 // the products' operands replace the unit-vector matrices
    cudaFree(m->d_B);
    m->d_F = m->d_B = nullptr;
    return SHT_OK;
}

int check_args(const sht_matrix* m, int K, int64_t ldc, int64_t ldg, const void* a, const void* b, const char* what) {
    if (!m) return mfail(SHT_EINVAL, "matrix transform: NULL handle");
    if (K < 0 || K > m->d.nlayers) {
        snprintf(g_msg, sizeof g_msg, "%s: DimensionMismatch: K = %d layers, nlayers = %d", what, K, m->d.nlayers);
        return mfail(SHT_EINVAL, g_msg);
    }
    if (ldc < m->nlm || ldg < m->npoints) {
        snprintf(g_msg, sizeof g_msg, "%s: DimensionMismatch: leading dimension below nlm / npoints", what);
        return mfail(SHT_EINVAL, g_msg);
    }
    if (K > 0 && (!a || !b)) return mfail(SHT_EINVAL, "matrix transform: NULL array");
    return SHT_OK;
}

}  // namespace

int sht_matrix_create(const sht_desc* d, sht_matrix** out) {
    if (!d || !out) return mfail(SHT_EINVAL, "sht_matrix_create: NULL argument");
    *out = nullptr;
    if (d->nlayers < 1) return mfail(SHT_EINVAL, "sht_matrix_create: nlayers must be >= 1");
    if (d->precision != SHT_PREC_FP32 && d->nlayers > 1024)
        return mfail(SHT_EINVAL, "sht_matrix_create: tensor-core precisions support nlayers <= 1024");
    sht_matrix* m = new sht_matrix();
    m->d = *d;
    DevGuard g(d->device);
    const int rc = build(m);
    if (rc != SHT_OK) {
        release(m);
        delete m;
        return rc;
    }
    *out = m;
    return SHT_OK;
}

int sht_matrix_synthesize(sht_matrix* m, const void* coeffs, int64_t ldc, float* grid, int64_t ldg, int K,
                          unsigned flags, void* stream) {
    int rc = check_args(m, K, ldc, ldg, coeffs, grid, "sht_matrix_synthesize");
    if (rc != SHT_OK || K == 0) return rc;
    if (flags & ~SHT_UNSCALE_COSLAT) return mfail(SHT_EINVAL, "sht_matrix_synthesize: flags other than SHT_UNSCALE_COSLAT");
    DevGuard g(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    const bool unscale = flags & SHT_UNSCALE_COSLAT;
    const float* rs = unscale ? m->d_row_scale : nullptr;
    const cudaError_t e = m->mx ? mx_tf32_apply(m->mx, 1, (const float*)coeffs, 2 * ldc, grid, ldg, K, rs, m->d_err, s)
                                : tc_matrix_apply(m->tc, 1, (const float*)coeffs, 2 * ldc, grid, ldg, K, rs, m->d_err, s);
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_matrix_synthesize");
}

int sht_matrix_analyze(sht_matrix* m, const float* grid, int64_t ldg, void* coeffs, int64_t ldc, int K, unsigned flags,
                       void* stream) {
    int rc = check_args(m, K, ldc, ldg, coeffs, grid, "sht_matrix_analyze");
    if (rc != SHT_OK || K == 0) return rc;
    if (flags) return mfail(SHT_EINVAL, "sht_matrix_analyze: takes no flags");
    DevGuard g(m->d.device);
    cudaStream_t s = (cudaStream_t)stream;
    const cudaError_t e = m->mx ? mx_tf32_apply(m->mx, 0, grid, ldg, (float*)coeffs, 2 * ldc, K, nullptr, m->d_err, s)
                                : tc_matrix_apply(m->tc, 0, grid, ldg, (float*)coeffs, 2 * ldc, K, nullptr, m->d_err, s);
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_matrix_analyze");
}

int sht_matrix_device_status(sht_matrix* m, int32_t* status) {
    if (!m || !status) return mfail(SHT_EINVAL, "sht_matrix_device_status: NULL argument");
    DevGuard g(m->d.device);
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(status, m->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(m->d_err, 0, sizeof(int32_t));
    return e == cudaSuccess ? SHT_OK : mcuda(e, "sht_matrix_device_status");
}

int sht_matrix_destroy(sht_matrix* m) {
    if (!m) return SHT_OK;
    DevGuard g(m->d.device);
    release(m);
    delete m;
    return SHT_OK;
}
