// Spectral operators on packed lower-triangular coefficients [nlm, K] complex.
//
// Replace the KernelAbstractions kernels of SpeedyTransforms/src/spectral_gradients.jl:
// _divergence_kernel! (:105-125, curl and divergence), _UV_from_vor_kernel! (:269-298),
// _UV_from_vordiv_kernel! (:331-366), ∇²_kernel! (:411-421) and dpdy_kernel! (:509-527),
// with the precomputed factors of SpeedyTransforms/src/gradient_arrays.jl.
// All are memory-bound stencils along l within one order column: one thread per
// (lm, layer), neighbours lm +- 1 come from the same cache lines.
#include "sht_internal.h"

namespace sht {

namespace {

constexpr int OPS_THREADS = 256;

__device__ __forceinline__ float2 mulf(float a, float2 z) { return make_float2(a * z.x, a * z.y); }
__device__ __forceinline__ float2 imul(float a, float2 z) { return make_float2(-a * z.y, a * z.x); }  // i*a*z
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

__global__ void divcurl_kernel(float2* __restrict__ out, const float2* __restrict__ u, const float2* __restrict__ v,
                               const float* __restrict__ grad, int64_t nlm, int64_t ldc, int curl, int flipsign,
                               int add, float inv_radius, int scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int64_t k = blockIdx.y;
    const float2* uk = u + k * ldc;
    const float2* vk = v + k * ldc;
    float2* ok = out + k * ldc;
    float2 res;
    if (lm == nlm - 1) {
        res = make_float2(0.f, 0.f);
    } else {
        float2 base;
        if (lm == 0) {
            const float2 c = mulf(grad[G_GRAD_Y_VORDIV2 * nlm + 0], vk[1]);
            base = curl ? make_float2(-c.x, -c.y) : c;
        } else {
            const float2 a = imul(grad[G_GRAD_X_VORDIV * nlm + lm], uk[lm]);
            const float2 b = mulf(grad[G_GRAD_Y_VORDIV1 * nlm + lm], vk[lm - 1]);
            const float2 c = mulf(grad[G_GRAD_Y_VORDIV2 * nlm + lm], vk[lm + 1]);
            base = curl ? sub2(add2(a, b), c) : add2(sub2(a, b), c);
        }
        if (flipsign) base = make_float2(-base.x, -base.y);
        res = add ? add2(ok[lm], base) : base;
    }
    if (scale) res = mulf(inv_radius, res);
    ok[lm] = res;
}

__global__ void uv_kernel(float2* __restrict__ U, float2* __restrict__ V, const float2* __restrict__ vor,
                          const float2* __restrict__ div, const float* __restrict__ grad,
                          const int32_t* __restrict__ l_of, int64_t nlm, int64_t ldc, int lmax, float radius,
                          int scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int64_t k = blockIdx.y;
    const float2* z = vor + k * ldc;
    const float x = grad[G_VORDIV_TO_UV_X * nlm + lm];
    const float u1 = grad[G_VORDIV_TO_UV1 * nlm + lm];
    const float u2 = grad[G_VORDIV_TO_UV2 * nlm + lm];
    const int l = l_of[lm];
    float2 Uo, Vo;
    if (div == nullptr) {
        if (lm == 0) {
            Uo = mulf(u2, z[1]);
            Vo = imul(x, z[0]);
        } else if (l == lmax - 2) {
            Uo = mulf(-u1, z[lm - 1]);
            Vo = imul(x, z[lm]);
        } else if (l == lmax - 1) {
            Uo = mulf(-u1, z[lm - 1]);
            Vo = make_float2(0.f, 0.f);
        } else {
            Uo = sub2(mulf(u2, z[lm + 1]), mulf(u1, z[lm - 1]));
            Vo = imul(x, z[lm]);
        }
    } else {
        const float2* d = div + k * ldc;
        if (lm == 0) {
            Uo = add2(imul(x, d[0]), mulf(u2, z[1]));
            Vo = sub2(imul(x, z[0]), mulf(u2, d[1]));
        } else if (l == lmax - 2) {
            Uo = sub2(imul(x, d[lm]), mulf(u1, z[lm - 1]));
            Vo = add2(imul(x, z[lm]), mulf(u1, d[lm - 1]));
        } else if (l == lmax - 1) {
            Uo = mulf(-u1, z[lm - 1]);
            Vo = mulf(u1, d[lm - 1]);
        } else {
            const float2 dzt = sub2(mulf(u2, z[lm + 1]), mulf(u1, z[lm - 1]));
            const float2 ddt = sub2(mulf(u1, d[lm - 1]), mulf(u2, d[lm + 1]));
            Uo = add2(imul(x, d[lm]), dzt);
            Vo = add2(imul(x, z[lm]), ddt);
        }
    }
    if (scale) {
        Uo = mulf(radius, Uo);
        Vo = mulf(radius, Vo);
    }
    U[k * ldc + lm] = Uo;
    V[k * ldc + lm] = Vo;
}

__global__ void laplace_kernel(float2* __restrict__ out, const float2* __restrict__ in, const float* __restrict__ eig,
                               const int32_t* __restrict__ l_of, int64_t nlm, int64_t ldc, int flipsign, int add,
                               float scale, int do_scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int64_t i = blockIdx.y * ldc + lm;
    float2 a = mulf(eig[l_of[lm]], in[i]);
    if (flipsign) a = make_float2(-a.x, -a.y);
    float2 r = add ? add2(out[i], a) : a;
    if (do_scale) r = mulf(scale, r);
    out[i] = r;
}

__global__ void gradient_kernel(float2* __restrict__ dpdx, float2* __restrict__ dpdy, const float2* __restrict__ p,
                                const float* __restrict__ grad, const int32_t* __restrict__ m_of, int64_t nlm,
                                int64_t ldc, float inv_radius, int scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int64_t k = blockIdx.y;
    const float2* pk = p + k * ldc;
    float2 dx = imul((float)m_of[lm], pk[lm]);
    const float gy1 = grad[G_GRAD_Y1 * nlm + lm];
    const float gy2 = grad[G_GRAD_Y2 * nlm + lm];
    float2 dy;
    if (lm == 0) {
        dy = mulf(gy2, pk[1]);
    } else if (lm == nlm - 1) {
        dy = mulf(gy1, pk[lm - 1]);
    } else {
        dy = add2(mulf(gy1, pk[lm - 1]), mulf(gy2, pk[lm + 1]));
    }
    if (scale) {
        dx = mulf(inv_radius, dx);
        dy = mulf(inv_radius, dy);
    }
    dpdx[k * ldc + lm] = dx;
    dpdy[k * ldc + lm] = dy;
}

inline dim3 ops_grid(int64_t nlm, int K) { return dim3((unsigned)((nlm + OPS_THREADS - 1) / OPS_THREADS), K); }

}  // namespace

cudaError_t launch_divcurl(const Plan& p, float2* out, const float2* u, const float2* v, int64_t ldc, int K, bool curl,
                           bool flipsign, bool add, float inv_radius, cudaStream_t s) {
    // curl swaps u and v (spectral_gradients.jl:40)
    const float2* a = curl ? v : u;
    const float2* b = curl ? u : v;
    divcurl_kernel<<<ops_grid(p.nlm, K), OPS_THREADS, 0, s>>>(out, a, b, p.d_grad, p.nlm, ldc, curl, flipsign, add,
                                                              inv_radius, inv_radius != 1.0f);
    return cudaGetLastError();
}

cudaError_t launch_uv_from_vordiv(const Plan& p, float2* U, float2* V, const float2* vor, const float2* div,
                                  int64_t ldc, int K, float radius, cudaStream_t s) {
    uv_kernel<<<ops_grid(p.nlm, K), OPS_THREADS, 0, s>>>(U, V, vor, div, p.d_grad, p.d_l_of, p.nlm, ldc, p.lmax,
                                                         radius, radius != 1.0f);
    return cudaGetLastError();
}

cudaError_t launch_laplace(const Plan& p, float2* out, const float2* in, int64_t ldc, int K, bool inverse,
                           bool flipsign, bool add, float scale, cudaStream_t s) {
    laplace_kernel<<<ops_grid(p.nlm, K), OPS_THREADS, 0, s>>>(out, in, inverse ? p.d_eig_inv : p.d_eig, p.d_l_of,
                                                              p.nlm, ldc, flipsign, add, scale, scale != 1.0f);
    return cudaGetLastError();
}

cudaError_t launch_gradient(const Plan& p, float2* dpdx, float2* dpdy, const float2* in, int64_t ldc, int K,
                            float inv_radius, cudaStream_t s) {
    gradient_kernel<<<ops_grid(p.nlm, K), OPS_THREADS, 0, s>>>(dpdx, dpdy, in, p.d_grad, p.d_m_of, p.nlm, ldc,
                                                               inv_radius, inv_radius != 1.0f);
    return cudaGetLastError();
}

}  // namespace sht
