// Spectral operators on packed lower-triangular coefficients [nlm, K] complex.
//
// Replace the KernelAbstractions kernels of SpeedyTransforms/src/spectral_gradients.jl:
// _divergence_kernel! (:105-125, curl and divergence), _UV_from_vor_kernel! (:269-298),
// _UV_from_vordiv_kernel! (:331-366), ∇²_kernel! (:411-421) and dpdy_kernel! (:509-527),
// with the precomputed factors of SpeedyTransforms/src/gradient_arrays.jl.
// All are memory-bound stencils along l within one order column: one thread per
// (lm, 1 to 8 layers), neighbours lm +- 1 come from the same cache lines.
#include "sht_internal.h"

namespace sht {

namespace {

constexpr int OPS_THREADS = 256;

__device__ __forceinline__ float2 mulf(float a, float2 z) { return make_float2(a * z.x, a * z.y); }
__device__ __forceinline__ float2 imul(float a, float2 z) { return make_float2(-a * z.y, a * z.x); }  // i*a*z
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// One thread per (lm, KL consecutive layers): the per-lm factors are read once and every
// layer's loads are issued before the first store, so each thread keeps KL x (1 .. 3)
// loads in flight. KL (8, 4 or 1) is chosen per call so that the grid still fills the GPU.

template <int KL>
__global__ void divcurl_kernel(float2* __restrict__ out, const float2* __restrict__ u, const float2* __restrict__ v,
                               const float* __restrict__ grad, int64_t nlm, int64_t ldc, int K, int curl,
                               int flipsign, int add, float inv_radius, int scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int k0 = blockIdx.y * KL;
    const bool last = lm == nlm - 1, first = lm == 0;
    const float gx = (first || last) ? 0.f : grad[G_GRAD_X_VORDIV * nlm + lm];
    const float g1 = (first || last) ? 0.f : grad[G_GRAD_Y_VORDIV1 * nlm + lm];
    const float g2 = last ? 0.f : grad[G_GRAD_Y_VORDIV2 * nlm + lm];
    float2 ua[KL], vm[KL], vp[KL], oa[KL];
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        const int64_t i = (int64_t)(k0 + t) * ldc + lm;
        ua[t] = vm[t] = vp[t] = oa[t] = make_float2(0.f, 0.f);
        if (k0 + t < K && !last) {
            if (!first) {
                ua[t] = u[i];
                vm[t] = v[i - 1];
            }
            vp[t] = v[i + 1];
            if (add) oa[t] = out[i];
        }
    }
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        if (k0 + t >= K) break;
        float2 res;
        if (last) {
            res = make_float2(0.f, 0.f);
        } else {
            float2 base;
            if (first) {
                const float2 c = mulf(g2, vp[t]);
                base = curl ? make_float2(-c.x, -c.y) : c;
            } else {
                const float2 a = imul(gx, ua[t]);
                const float2 b = mulf(g1, vm[t]);
                const float2 c = mulf(g2, vp[t]);
                base = curl ? sub2(add2(a, b), c) : add2(sub2(a, b), c);
            }
            if (flipsign) base = make_float2(-base.x, -base.y);
            res = add ? add2(oa[t], base) : base;
        }
        if (scale) res = mulf(inv_radius, res);
        out[(int64_t)(k0 + t) * ldc + lm] = res;
    }
}

template <int KL>
__global__ void uv_kernel(float2* __restrict__ U, float2* __restrict__ V, const float2* __restrict__ vor,
                          const float2* __restrict__ div, const float* __restrict__ grad,
                          const int32_t* __restrict__ l_of, int64_t nlm, int64_t ldc, int K, int lmax, float radius,
                          int scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int k0 = blockIdx.y * KL;
    const float x = grad[G_VORDIV_TO_UV_X * nlm + lm];
    const float u1 = grad[G_VORDIV_TO_UV1 * nlm + lm];
    const float u2 = grad[G_VORDIV_TO_UV2 * nlm + lm];
    const int l = l_of[lm];
    // which neighbours the stencil row of this lm uses
    const bool first = lm == 0, top1 = l == lmax - 2, top0 = l == lmax - 1;
    const bool has_m = !first, has_p = !(top1 || top0), has_c = !top0;
    float2 zc[KL], zm[KL], zp[KL], dc[KL], dm[KL], dp[KL];
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        const int64_t i = (int64_t)(k0 + t) * ldc + lm;
        zc[t] = zm[t] = zp[t] = dc[t] = dm[t] = dp[t] = make_float2(0.f, 0.f);
        if (k0 + t < K) {
            if (has_c || first) zc[t] = vor[i];
            if (has_m) zm[t] = vor[i - 1];
            if (has_p || first) zp[t] = vor[i + 1];
            if (div != nullptr) {
                if (has_c || first) dc[t] = div[i];
                if (has_m) dm[t] = div[i - 1];
                if (has_p || first) dp[t] = div[i + 1];
            }
        }
    }
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        if (k0 + t >= K) break;
        float2 Uo, Vo;
        if (div == nullptr) {
            if (first) {
                Uo = mulf(u2, zp[t]);
                Vo = imul(x, zc[t]);
            } else if (top1) {
                Uo = mulf(-u1, zm[t]);
                Vo = imul(x, zc[t]);
            } else if (top0) {
                Uo = mulf(-u1, zm[t]);
                Vo = make_float2(0.f, 0.f);
            } else {
                Uo = sub2(mulf(u2, zp[t]), mulf(u1, zm[t]));
                Vo = imul(x, zc[t]);
            }
        } else {
            if (first) {
                Uo = add2(imul(x, dc[t]), mulf(u2, zp[t]));
                Vo = sub2(imul(x, zc[t]), mulf(u2, dp[t]));
            } else if (top1) {
                Uo = sub2(imul(x, dc[t]), mulf(u1, zm[t]));
                Vo = add2(imul(x, zc[t]), mulf(u1, dm[t]));
            } else if (top0) {
                Uo = mulf(-u1, zm[t]);
                Vo = mulf(u1, dm[t]);
            } else {
                const float2 dzt = sub2(mulf(u2, zp[t]), mulf(u1, zm[t]));
                const float2 ddt = sub2(mulf(u1, dm[t]), mulf(u2, dp[t]));
                Uo = add2(imul(x, dc[t]), dzt);
                Vo = add2(imul(x, zc[t]), ddt);
            }
        }
        if (scale) {
            Uo = mulf(radius, Uo);
            Vo = mulf(radius, Vo);
        }
        U[(int64_t)(k0 + t) * ldc + lm] = Uo;
        V[(int64_t)(k0 + t) * ldc + lm] = Vo;
    }
}

template <int KL>
__global__ void laplace_kernel(float2* __restrict__ out, const float2* __restrict__ in, const float* __restrict__ eig,
                               const int32_t* __restrict__ l_of, int64_t nlm, int64_t ldc, int K, int flipsign,
                               int add, float scale, int do_scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int k0 = blockIdx.y * KL;
    const float e = eig[l_of[lm]];
    float2 x[KL], o[KL];
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        const int64_t i = (int64_t)(k0 + t) * ldc + lm;
        x[t] = o[t] = make_float2(0.f, 0.f);
        if (k0 + t < K) {
            x[t] = in[i];
            if (add) o[t] = out[i];
        }
    }
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        if (k0 + t >= K) break;
        float2 a = mulf(e, x[t]);
        if (flipsign) a = make_float2(-a.x, -a.y);
        float2 r = add ? add2(o[t], a) : a;
        if (do_scale) r = mulf(scale, r);
        out[(int64_t)(k0 + t) * ldc + lm] = r;
    }
}

template <int KL>
__global__ void gradient_kernel(float2* __restrict__ dpdx, float2* __restrict__ dpdy, const float2* __restrict__ p,
                                const float* __restrict__ grad, const int32_t* __restrict__ m_of, int64_t nlm,
                                int64_t ldc, int K, float inv_radius, int scale) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int k0 = blockIdx.y * KL;
    const float mf = (float)m_of[lm];
    const float gy1 = grad[G_GRAD_Y1 * nlm + lm];
    const float gy2 = grad[G_GRAD_Y2 * nlm + lm];
    const bool first = lm == 0, last = lm == nlm - 1;
    float2 pc[KL], pm[KL], pp[KL];
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        const int64_t i = (int64_t)(k0 + t) * ldc + lm;
        pc[t] = pm[t] = pp[t] = make_float2(0.f, 0.f);
        if (k0 + t < K) {
            pc[t] = p[i];
            if (!first) pm[t] = p[i - 1];
            if (!last) pp[t] = p[i + 1];
        }
    }
#pragma unroll
    for (int t = 0; t < KL; ++t) {
        if (k0 + t >= K) break;
        float2 dx = imul(mf, pc[t]);
        float2 dy;
        if (first) {
            dy = mulf(gy2, pp[t]);
        } else if (last) {
            dy = mulf(gy1, pm[t]);
        } else {
            dy = add2(mulf(gy1, pm[t]), mulf(gy2, pp[t]));
        }
        if (scale) {
            dx = mulf(inv_radius, dx);
            dy = mulf(inv_radius, dy);
        }
        dpdx[(int64_t)(k0 + t) * ldc + lm] = dx;
        dpdy[(int64_t)(k0 + t) * ldc + lm] = dy;
    }
}

// Layers per thread: as many as keep >= 2 x 148 x 256 threads in the grid (at most `most`).
inline int ops_layers(int64_t nlm, int K, int most) {
    for (int kl = most; kl > 1; kl /= 2)
        if (nlm * ((K + kl - 1) / kl) >= 2 * 148 * 256) return kl;
    return 1;
}
inline dim3 ops_grid(int64_t nlm, int K, int kl) {
    return dim3((unsigned)((nlm + OPS_THREADS - 1) / OPS_THREADS), (unsigned)((K + kl - 1) / kl));
}

}  // namespace

cudaError_t launch_divcurl(const Plan& p, float2* out, const float2* u, const float2* v, int64_t ldc, int K, bool curl,
                           bool flipsign, bool add, float inv_radius, cudaStream_t s) {
    // curl swaps u and v (spectral_gradients.jl:40)
    const float2* a = curl ? v : u;
    const float2* b = curl ? u : v;
    const int kl = ops_layers(p.nlm, K, 8);
    auto kern = kl == 8 ? divcurl_kernel<8> : kl == 4 ? divcurl_kernel<4> : kl == 2 ? divcurl_kernel<2> : divcurl_kernel<1>;
    kern<<<ops_grid(p.nlm, K, kl), OPS_THREADS, 0, s>>>(out, a, b, p.d_grad, p.nlm, ldc, K, curl, flipsign, add,
                                                        inv_radius, inv_radius != 1.0f);
    return cudaGetLastError();
}

cudaError_t launch_uv_from_vordiv(const Plan& p, float2* U, float2* V, const float2* vor, const float2* div,
                                  int64_t ldc, int K, float radius, cudaStream_t s) {
    const int kl = ops_layers(p.nlm, K, 4);     // six neighbour arrays per layer: at most 4 layers in registers
    auto kern = kl == 4 ? uv_kernel<4> : kl == 2 ? uv_kernel<2> : uv_kernel<1>;
    kern<<<ops_grid(p.nlm, K, kl), OPS_THREADS, 0, s>>>(U, V, vor, div, p.d_grad, p.d_l_of, p.nlm, ldc, K, p.lmax,
                                                        radius, radius != 1.0f);
    return cudaGetLastError();
}

cudaError_t launch_laplace(const Plan& p, float2* out, const float2* in, int64_t ldc, int K, bool inverse,
                           bool flipsign, bool add, float scale, cudaStream_t s) {
    const int kl = ops_layers(p.nlm, K, 8);
    auto kern = kl == 8 ? laplace_kernel<8> : kl == 4 ? laplace_kernel<4> : kl == 2 ? laplace_kernel<2> : laplace_kernel<1>;
    kern<<<ops_grid(p.nlm, K, kl), OPS_THREADS, 0, s>>>(out, in, inverse ? p.d_eig_inv : p.d_eig, p.d_l_of, p.nlm, ldc,
                                                        K, flipsign, add, scale, scale != 1.0f);
    return cudaGetLastError();
}

cudaError_t launch_gradient(const Plan& p, float2* dpdx, float2* dpdy, const float2* in, int64_t ldc, int K,
                            float inv_radius, cudaStream_t s) {
    const int kl = ops_layers(p.nlm, K, 8);
    auto kern = kl == 8 ? gradient_kernel<8> : kl == 4 ? gradient_kernel<4> : kl == 2 ? gradient_kernel<2> : gradient_kernel<1>;
    kern<<<ops_grid(p.nlm, K, kl), OPS_THREADS, 0, s>>>(dpdx, dpdy, in, p.d_grad, p.d_m_of, p.nlm, ldc, K, inv_radius,
                                                        inv_radius != 1.0f);
    return cudaGetLastError();
}

}  // namespace sht
