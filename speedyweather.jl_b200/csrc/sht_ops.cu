// Spectral operators on packed lower-triangular coefficients [nlm, K] complex.
//
// Replace the KernelAbstractions kernels of SpeedyTransforms/src/spectral_gradients.jl:
// _divergence_kernel! (:105-125, curl and divergence), _UV_from_vor_kernel! (:269-298),
// _UV_from_vordiv_kernel! (:331-366), ∇²_kernel! (:411-421) and dpdy_kernel! (:509-527),
// with the precomputed factors of SpeedyTransforms/src/gradient_arrays.jl.
// All are memory-bound stencils along l within one order column: one thread per
// (lm, 1 to 8 layers), neighbours lm +- 1 come from the same cache lines.
#include <algorithm>

#include "sht_internal.h"

namespace sht {

namespace {

constexpr int OPS_THREADS = 256;

// Products and sums rounded one by one (no contraction into fused multiply-adds), so that
// the single-operator kernels and the batched kernel below give the same bits.
__device__ __forceinline__ float2 mulf(float a, float2 z) { return make_float2(__fmul_rn(a, z.x), __fmul_rn(a, z.y)); }
__device__ __forceinline__ float2 imul(float a, float2 z) {   // i*a*z
    return make_float2(-__fmul_rn(a, z.y), __fmul_rn(a, z.x));
}
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// ---- the arithmetic of each operator for one coefficient, given its loaded neighbours ----

// divergence (curl with u and v swapped and the sign of the stencil flipped); the last
// coefficient (the extra degree) is zero
__device__ __forceinline__ float2 divcurl_value(bool first, bool last, float gx, float g1, float g2, float2 ua,
                                                float2 vm, float2 vp, float2 oa, int curl, int flipsign, int add,
                                                float inv_radius, int scale) {
    float2 res;
    if (last) {
        res = make_float2(0.f, 0.f);
    } else {
        float2 base;
        if (first) {
            const float2 c = mulf(g2, vp);
            base = curl ? neg2(c) : c;
        } else {
            const float2 a = imul(gx, ua);
            const float2 b = mulf(g1, vm);
            const float2 c = mulf(g2, vp);
            base = curl ? sub2(add2(a, b), c) : add2(sub2(a, b), c);
        }
        if (flipsign) base = neg2(base);
        res = add ? add2(oa, base) : base;
    }
    return scale ? mulf(inv_radius, res) : res;
}

__device__ __forceinline__ float2 laplace_value(float e, float2 x, float2 o, int flipsign, int add, float scale,
                                                int do_scale) {
    float2 a = mulf(e, x);
    if (flipsign) a = neg2(a);
    const float2 r = add ? add2(o, a) : a;
    return do_scale ? mulf(scale, r) : r;
}

__device__ __forceinline__ void gradient_value(bool first, bool last, float mf, float gy1, float gy2, float2 pc,
                                               float2 pm, float2 pp, float inv_radius, int scale, float2& dx,
                                               float2& dy) {
    dx = imul(mf, pc);
    if (first)
        dy = mulf(gy2, pp);
    else if (last)
        dy = mulf(gy1, pm);
    else
        dy = add2(mulf(gy1, pm), mulf(gy2, pp));
    if (scale) {
        dx = mulf(inv_radius, dx);
        dy = mulf(inv_radius, dy);
    }
}

// UV from vorticity (and divergence if has_div); first: lm = 0, top1/top0: l = lmax - 2 / lmax - 1
__device__ __forceinline__ void uv_value(bool has_div, bool first, bool top1, bool top0, float x, float u1, float u2,
                                         float2 zc, float2 zm, float2 zp, float2 dc, float2 dm, float2 dp,
                                         float radius, int scale, float2& Uo, float2& Vo) {
    if (!has_div) {
        if (first) {
            Uo = mulf(u2, zp);
            Vo = imul(x, zc);
        } else if (top1) {
            Uo = mulf(-u1, zm);
            Vo = imul(x, zc);
        } else if (top0) {
            Uo = mulf(-u1, zm);
            Vo = make_float2(0.f, 0.f);
        } else {
            Uo = sub2(mulf(u2, zp), mulf(u1, zm));
            Vo = imul(x, zc);
        }
    } else {
        if (first) {
            Uo = add2(imul(x, dc), mulf(u2, zp));
            Vo = sub2(imul(x, zc), mulf(u2, dp));
        } else if (top1) {
            Uo = sub2(imul(x, dc), mulf(u1, zm));
            Vo = add2(imul(x, zc), mulf(u1, dm));
        } else if (top0) {
            Uo = mulf(-u1, zm);
            Vo = mulf(u1, dm);
        } else {
            const float2 dzt = sub2(mulf(u2, zp), mulf(u1, zm));
            const float2 ddt = sub2(mulf(u1, dm), mulf(u2, dp));
            Uo = add2(imul(x, dc), dzt);
            Vo = add2(imul(x, zc), ddt);
        }
    }
    if (scale) {
        Uo = mulf(radius, Uo);
        Vo = mulf(radius, Vo);
    }
}

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
        out[(int64_t)(k0 + t) * ldc + lm] =
            divcurl_value(first, last, gx, g1, g2, ua[t], vm[t], vp[t], oa[t], curl, flipsign, add, inv_radius, scale);
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
        uv_value(div != nullptr, first, top1, top0, x, u1, u2, zc[t], zm[t], zp[t], dc[t], dm[t], dp[t], radius, scale,
                 Uo, Vo);
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
        out[(int64_t)(k0 + t) * ldc + lm] = laplace_value(e, x[t], o[t], flipsign, add, scale, do_scale);
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
        float2 dx, dy;
        gradient_value(first, last, mf, gy1, gy2, pc[t], pm[t], pp[t], inv_radius, scale, dx, dy);
        dpdx[(int64_t)(k0 + t) * ldc + lm] = dx;
        dpdy[(int64_t)(k0 + t) * ldc + lm] = dy;
    }
}

// ---- many operators in one launch ------------------------------------------------------
// One thread per (lm, layer k); it applies the ops in list order, each with the single-
// operator arithmetic above. The ops travel by value as a kernel parameter.
struct DevOp {
    int32_t kind, flags;
    float2* out;
    float2* out2;
    const float2* a;
    const float2* b;
    int64_t ldc;
    int32_t K;
    float s;              // 1 / radius (curl, divergence, gradient), radius (UV), Laplacian scale
    int32_t do_scale;
    int32_t pad;
};
struct DevOps {
    DevOp op[SHT_MAX_OPS];
    int32_t n;
};

__global__ void __launch_bounds__(OPS_THREADS) ops_batch_kernel(const DevOps ops, const float* __restrict__ grad,
                                                                const float* __restrict__ eig,
                                                                const float* __restrict__ eig_inv,
                                                                const int32_t* __restrict__ l_of,
                                                                const int32_t* __restrict__ m_of, int64_t nlm,
                                                                int lmax) {
    const int64_t lm = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (lm >= nlm) return;
    const int k = blockIdx.y;
    const bool first = lm == 0, last = lm == nlm - 1;
    for (int j = 0; j < ops.n; ++j) {
        const DevOp& o = ops.op[j];
        if (k >= o.K) continue;
        const int64_t i = (int64_t)k * o.ldc + lm;
        switch (o.kind) {
            case SHT_OP_CURL:
            case SHT_OP_DIVERGENCE: {
                const int curl = o.kind == SHT_OP_CURL;
                const int add = (o.flags & SHT_ADD) != 0;
                const float gx = (first || last) ? 0.f : grad[G_GRAD_X_VORDIV * nlm + lm];
                const float g1 = (first || last) ? 0.f : grad[G_GRAD_Y_VORDIV1 * nlm + lm];
                const float g2 = last ? 0.f : grad[G_GRAD_Y_VORDIV2 * nlm + lm];
                // curl swaps u and v (spectral_gradients.jl:40)
                const float2* u = curl ? o.b : o.a;
                const float2* v = curl ? o.a : o.b;
                float2 ua = make_float2(0.f, 0.f), vm = ua, vp = ua, oa = ua;
                if (!last) {
                    if (!first) {
                        ua = u[i];
                        vm = v[i - 1];
                    }
                    vp = v[i + 1];
                    if (add) oa = o.out[i];
                }
                o.out[i] = divcurl_value(first, last, gx, g1, g2, ua, vm, vp, oa, curl, (o.flags & SHT_FLIPSIGN) != 0,
                                         add, o.s, o.do_scale);
                break;
            }
            case SHT_OP_LAPLACE: {
                const int add = (o.flags & SHT_ADD) != 0;
                const float e = ((o.flags & SHT_INVERSE) ? eig_inv : eig)[l_of[lm]];
                const float2 x = o.a[i];
                const float2 old = add ? o.out[i] : make_float2(0.f, 0.f);
                o.out[i] = laplace_value(e, x, old, (o.flags & SHT_FLIPSIGN) != 0, add, o.s, o.do_scale);
                break;
            }
            case SHT_OP_GRADIENT: {
                const float2 pc = o.a[i];
                const float2 pm = first ? make_float2(0.f, 0.f) : o.a[i - 1];
                const float2 pp = last ? make_float2(0.f, 0.f) : o.a[i + 1];
                float2 dx, dy;
                gradient_value(first, last, (float)m_of[lm], grad[G_GRAD_Y1 * nlm + lm], grad[G_GRAD_Y2 * nlm + lm],
                               pc, pm, pp, o.s, o.do_scale, dx, dy);
                o.out[i] = dx;
                o.out2[i] = dy;
                break;
            }
            default: {   // SHT_OP_UV_FROM_VORDIV
                const int l = l_of[lm];
                const bool top1 = l == lmax - 2, top0 = l == lmax - 1;
                const bool has_m = !first, has_p = !(top1 || top0), has_c = !top0;
                const float2 z0 = make_float2(0.f, 0.f);
                const float2 zc = (has_c || first) ? o.a[i] : z0;
                const float2 zm = has_m ? o.a[i - 1] : z0;
                const float2 zp = (has_p || first) ? o.a[i + 1] : z0;
                float2 dc = z0, dm = z0, dp = z0;
                if (o.b != nullptr) {
                    if (has_c || first) dc = o.b[i];
                    if (has_m) dm = o.b[i - 1];
                    if (has_p || first) dp = o.b[i + 1];
                }
                float2 Uo, Vo;
                uv_value(o.b != nullptr, first, top1, top0, grad[G_VORDIV_TO_UV_X * nlm + lm],
                         grad[G_VORDIV_TO_UV1 * nlm + lm], grad[G_VORDIV_TO_UV2 * nlm + lm], zc, zm, zp, dc, dm, dp,
                         o.s, o.do_scale, Uo, Vo);
                o.out[i] = Uo;
                o.out2[i] = Vo;
                break;
            }
        }
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

// ops: validated by the caller (sht_operators)
cudaError_t launch_operators(const Plan& p, const sht_op* ops, int nops, cudaStream_t s) {
    DevOps d{};
    d.n = nops;
    int kmax = 0;
    for (int j = 0; j < nops; ++j) {
        const sht_op& o = ops[j];
        DevOp& q = d.op[j];
        q.kind = o.kind;
        q.flags = (int32_t)o.flags;
        q.out = (float2*)o.out;
        q.out2 = (float2*)o.out2;
        q.a = (const float2*)o.a;
        q.b = (const float2*)o.b;
        q.ldc = o.ldc;
        q.K = o.K;
        // the factors of the single calls (sht_plan.cu), computed the same way
        const double r = o.radius;
        if (o.kind == SHT_OP_LAPLACE) {
            const bool inv = (o.flags & SHT_INVERSE) != 0;
            q.s = (float)(r == 1.0 ? 1.0 : (inv ? r * r : 1.0 / (r * r)));
            q.do_scale = q.s != 1.0f;
        } else if (o.kind == SHT_OP_UV_FROM_VORDIV) {
            q.s = (float)r;
            q.do_scale = q.s != 1.0f;
        } else {
            q.s = (float)(1.0 / r);
            q.do_scale = q.s != 1.0f;
        }
        kmax = std::max(kmax, o.K);
    }
    if (kmax == 0) return cudaSuccess;
    const dim3 g((unsigned)((p.nlm + OPS_THREADS - 1) / OPS_THREADS), (unsigned)kmax);
    ops_batch_kernel<<<g, OPS_THREADS, 0, s>>>(d, p.d_grad, p.d_eig, p.d_eig_inv, p.d_l_of, p.d_m_of, p.nlm, p.lmax);
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
