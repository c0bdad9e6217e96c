// Fourier stage of the spherical harmonic transform: one launch per direction
// covers every ring pair and every layer of a full or octahedral Gaussian grid.
//
// Replaces the per-ring FFTW/cuFFT plans of SpeedyTransforms/src/fourier.jl:129-292
// and the gather/FFT/scatter CUDA graph of SpeedyTransforms/ext/gpu_graphs_common.jl:199-260.
//
// Design: one CTA per (northern ring j, chunk of C layers). The northern and the
// mirrored southern ring have the same length n, so their real sequences are
// packed into one complex sequence z = f_N + i f_S and transformed together by a
// mixed-radix Stockham FFT in shared memory (radices 2, 3, 4, 5, 7 in registers,
// any larger prime by a symmetric direct DFT). Twiddles come from a per-ring
// table exp(-2 pi i t / n) computed in FP64 on the host.
//
// The Fourier scratch holds, per ring j and order m <= mt(j), the even and odd
// hemispheric combinations the Legendre stage contracts with
//   E = dOmega_j (F_N + F_S),  O = dOmega_j (F_N - F_S)         (analysis)
//   G_N = E + O,  G_S = E - O                                   (synthesis)
// laid out [row = gofs_j + m][eo][k] complex FP32 (k = layer, fastest).
// FFTW's conventions are kept: r2c and c2r are unnormalised and c2r ignores the
// imaginary parts of the DC and Nyquist bins.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <map>
#include <mutex>

#include "sht_internal.h"

namespace sht {

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
template <bool INV>
__device__ __forceinline__ float2 twmul(float2 v, float2 w) {
    return INV ? cmulc(v, w) : cmul(v, w);
}
// Exact quotient x / d for 0 <= x < 2^22 and d >= 1 through a float reciprocal:
// (x + 0.5) / d is at least 0.5 / d away from an integer and the two roundings
// err by less than 1.2e-7 (x + 0.5) / d, so truncation gives floor(x / d). A few
// instructions instead of the integer division sequence, in every index loop.
struct Div {
    int d;
    float r;
};
__device__ __forceinline__ Div mkdiv(int d) { return Div{d, 1.0f / (float)d}; }
__device__ __forceinline__ int quo(int x, Div v) { return (int)(((float)x + 0.5f) * v.r); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// cos and sin of 2 pi t / P for the odd radices (t <= (P - 1) / 2)
__host__ __device__ constexpr float rot_cos(int P, int t) {
    return P == 3 ? -0.5f
         : P == 5 ? (t == 1 ? 0.30901699437494745f : -0.8090169943749473f)
                  : (t == 1 ? 0.6234898018587336f : t == 2 ? -0.22252093395631434f : -0.900968867902419f);
}
__host__ __device__ constexpr float rot_sin(int P, int t) {
    return P == 3 ? 0.8660254037844387f
         : P == 5 ? (t == 1 ? 0.9510565162951535f : 0.5877852522924732f)
                  : (t == 1 ? 0.7818314824680298f : t == 2 ? 0.9749279121818236f : 0.43388373911755823f);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2 a, float2 b, float2 c, float2 d, float2& y0, float2& y1, float2& y2,
                                     float2& y3) {
    const float2 s02 = cadd(a, c), d02 = csub(a, c);
    const float2 s13 = cadd(b, d), d13 = csub(b, d);
    // forward: y1 = d02 - i d13, y3 = d02 + i d13
    const float2 jd = INV ? make_float2(-d13.y, d13.x) : make_float2(d13.y, -d13.x);
    y0 = cadd(s02, s13);
    y2 = csub(s02, s13);
    y1 = cadd(d02, jd);
    y3 = csub(d02, jd);
}

// y = DFT_P(v) (forward: exp(-2 pi i rs/P); inverse: exp(+...)), P in {2, 3, 4, 5, 7, 8}.
template <int P, bool INV>
__device__ __forceinline__ void dft_small(const float2 (&v)[P], float2 (&y)[P]) {
    if constexpr (P == 2) {
        y[0] = cadd(v[0], v[1]);
        y[1] = csub(v[0], v[1]);
    } else if constexpr (P == 4) {
        dft4<INV>(v[0], v[1], v[2], v[3], y[0], y[1], y[2], y[3]);
    } else if constexpr (P == 8) {
        // two DFT_4 of the even and odd points, combined with exp(-+ i pi r / 4)
        float2 e[4], o[4];
        dft4<INV>(v[0], v[2], v[4], v[6], e[0], e[1], e[2], e[3]);
        dft4<INV>(v[1], v[3], v[5], v[7], o[0], o[1], o[2], o[3]);
        // (products rounded on their own: no contraction into the following sums, so
        // every kernel instantiating this gives the same bits)
        constexpr float h = 0.7071067811865476f;
        const float2 o1 = INV ? make_float2(__fmul_rn(h, o[1].x - o[1].y), __fmul_rn(h, o[1].x + o[1].y))
                              : make_float2(__fmul_rn(h, o[1].x + o[1].y), __fmul_rn(h, o[1].y - o[1].x));
        const float2 o2 = INV ? make_float2(-o[2].y, o[2].x) : make_float2(o[2].y, -o[2].x);
        const float2 o3 = INV ? make_float2(__fmul_rn(-h, o[3].x + o[3].y), __fmul_rn(h, o[3].x - o[3].y))
                              : make_float2(__fmul_rn(h, o[3].y - o[3].x), __fmul_rn(-h, o[3].x + o[3].y));
        y[0] = cadd(e[0], o[0]);
        y[4] = csub(e[0], o[0]);
        y[1] = cadd(e[1], o1);
        y[5] = csub(e[1], o1);
        y[2] = cadd(e[2], o2);
        y[6] = csub(e[2], o2);
        y[3] = cadd(e[3], o3);
        y[7] = csub(e[3], o3);
    } else {
        // odd P: symmetric direct DFT, y_r and y_{P-r} share the sums
        constexpr int H = (P - 1) / 2;
        float2 s = v[0];
#pragma unroll
        for (int q = 1; q < P; ++q) s = cadd(s, v[q]);
        y[0] = s;
#pragma unroll
        for (int r = 1; r <= H; ++r) {
            float2 A = make_float2(0.f, 0.f), B = make_float2(0.f, 0.f);
#pragma unroll
            for (int q = 1; q <= H; ++q) {
                const int t = (r * q) % P;
                const float cs = rot_cos(P, t <= H ? t : P - t);
                const float sn = t <= H ? rot_sin(P, t) : -rot_sin(P, P - t);
                const float2 a = cadd(v[q], v[P - q]);
                const float2 b = csub(v[q], v[P - q]);
                A.x = fmaf(a.x, cs, A.x); A.y = fmaf(a.y, cs, A.y);
                B.x = fmaf(b.x, sn, B.x); B.y = fmaf(b.y, sn, B.y);
            }
            if (!INV) {
                y[r] = make_float2(v[0].x + A.x + B.y, v[0].y + A.y - B.x);
                y[P - r] = make_float2(v[0].x + A.x - B.y, v[0].y + A.y + B.x);
            } else {
                y[r] = make_float2(v[0].x + A.x - B.y, v[0].y + A.y + B.x);
                y[P - r] = make_float2(v[0].x + A.x + B.y, v[0].y + A.y - B.x);
            }
        }
    }
}

// One Stockham stage of radix P over C vectors of length n; Ns = product of the
// radices of earlier stages. Output in natural order after the last stage. A work
// item is one butterfly position b for CT layers: its index arithmetic and twiddles
// are shared by the layers. The first stage (Ns = 1) has no twiddles.
#ifndef SHT_FFT_CT
#define SHT_FFT_CT 4
#endif
constexpr int CT = SHT_FFT_CT;

// RAW (FIRST only, analysis): the input of layer c is the raw ring data at X + c ldx
// (n northern floats, then n southern floats).
template <int P, bool INV, bool FIRST, bool RAW = false>
__device__ void stage_small(const float2* __restrict__ X, float2* __restrict__ Y, int n, int ldx, int C, int Ns,
                            const float2* __restrict__ W) {
    const int nb = n / P;
    const int tstride = n / (Ns * P);
    const int ncg = (C + CT - 1) / CT;
    const Div dnb = mkdiv(nb), dns = mkdiv(Ns);
    for (int w = threadIdx.x; w < ncg * nb; w += blockDim.x) {
        const int cg = quo(w, dnb);
        const int b = w - cg * nb;
        const int k = FIRST ? 0 : b - quo(b, dns) * Ns;
        float2 tw[P];
        if (!FIRST) {
            const int kt = k * tstride;
#pragma unroll
            for (int r = 1; r < P; ++r) tw[r] = W[r * kt];
        }
#pragma unroll
        for (int t = 0; t < CT; ++t) {
            const int c = cg * CT + t;
            if (c >= C) break;
            const float2* x = X + c * ldx + b;
            float2 v[P];
            if (RAW) {
                const float* raw = reinterpret_cast<const float*>(X + c * ldx) + b;
#pragma unroll
                for (int r = 0; r < P; ++r) v[r] = make_float2(raw[r * nb], raw[n + r * nb]);
            } else {
#pragma unroll
                for (int r = 0; r < P; ++r) v[r] = (FIRST || r == 0) ? x[r * nb] : twmul<INV>(x[r * nb], tw[r]);
            }
            float2 y[P];
            dft_small<P, INV>(v, y);
            float2* yo = Y + c * ldx + (b - k) * P + k;
#pragma unroll
            for (int r = 0; r < P; ++r) yo[r * Ns] = y[r];
        }
    }
}

// Twiddles of a prime stage that is not the first one, applied in place:
// x[c n + b + r nb] *= W^(r k tstride), k = b mod Ns.
template <bool INV>
__device__ void twiddle_pass(float2* __restrict__ X, int n, int ldx, int C, int Ns, int p, const float2* __restrict__ W) {
    const int nb = n / p;
    const int tstride = n / (Ns * p);
    const Div dnb = mkdiv(nb), dns = mkdiv(Ns);
    for (int w = threadIdx.x; w < C * nb; w += blockDim.x) {
        const int c = quo(w, dnb);
        const int b = w - c * nb;
        const int k = b - quo(b, dns) * Ns;
        if (k == 0) continue;
        float2* x = X + c * ldx + b;
        const int kt = k * tstride;
        for (int r = 1; r < p; ++r) x[r * nb] = twmul<INV>(x[r * nb], W[r * kt]);
    }
}

// Stage of an odd prime radix p > 8 as a symmetric direct DFT in Rader's ordering.
// With g a primitive root of p and h = (p - 1) / 2, the input pairs {q, p - q} are
// enumerated as q_b = g^-b and the output pairs {r, p - r} as r_a = g^a (a, b < h);
// every nonzero residue appears once since g^h = -1. Then r_a q_b = g^(a - b) and
//   A_a = sum_b u_b cos(2 pi g^(a-b) / p),  B_a = sum_b v_b sin(...),
//   u_b = x_qb + x_-qb,  v_b = x_qb - x_-qb,
//   y_ra = x_0 + A_a -+ i B_a,  y_-ra = x_0 + A_a +- i B_a       (forward / inverse)
// The weight depends on a - b only: a thread owning the GR outputs a0 .. a0 + GR - 1
// reads, for GR consecutive b, one window of 2 GR consecutive table entries
// T[a - b + hpad - 1] (16-byte loads shared by the warp) and does 4 GR FMAs per b.
// A first pass stores u_b, v_b (and x_0) of every column in Y, [b][column] with the
// column fastest; the main pass reads them with one 16-byte load per b and writes
// its outputs into X, which holds the stage's result.
// Table block of the prime (float2 units, hpad = h rounded up to GR):
//   T [2 hpad] | q_b [hpad int32] | r_a [hpad int32]
constexpr int GR = kPrimeGroup;

__host__ __device__ inline int prime_hpad(int p) { return ((p - 1) / 2 + GR - 1) / GR * GR; }

template <bool TAIL>
__device__ __forceinline__ void prime_block(float (&ar)[GR], float (&ai)[GR], float (&br)[GR], float (&bi)[GR],
                                            const float4* __restrict__ uv, int cols, const float2* __restrict__ T,
                                            int h, int B0, int tbase) {
    float2 wv[2 * GR];
    const float4* t4 = reinterpret_cast<const float4*>(T + tbase);
#pragma unroll
    for (int e = 0; e < GR; ++e) {
        const float4 f = t4[e];
        wv[2 * e] = make_float2(f.x, f.y);
        wv[2 * e + 1] = make_float2(f.z, f.w);
    }
#pragma unroll
    for (int s = 0; s < GR; ++s) {
        float4 q = make_float4(0.f, 0.f, 0.f, 0.f);
        if (!TAIL || B0 + s < h) q = uv[(B0 + s) * cols];
#pragma unroll
        for (int i = 0; i < GR; ++i) {
            const float2 wt = wv[i - s + GR - 1];
            ar[i] = fmaf(q.x, wt.x, ar[i]);
            ai[i] = fmaf(q.y, wt.x, ai[i]);
            br[i] = fmaf(q.z, wt.y, br[i]);
            bi[i] = fmaf(q.w, wt.y, bi[i]);
        }
    }
}

// RAW (first stage of the analysis only): layer c's input is still the raw ring data at
// X + c ldx (n northern floats, then n southern floats) instead of interleaved complex
// values; the pass that forms u_b, v_b reads it in place.
template <bool INV, bool RAW>
__device__ void stage_prime(float2* __restrict__ X, float2* __restrict__ Y, int n, int ldx, int C, int Ns, int p,
                            const float2* __restrict__ G) {
    const int nb = n / p;
    const int h = (p - 1) / 2;
    const int hpad = prime_hpad(p);
    const float2* T = G;
    const int* qb = reinterpret_cast<const int*>(G + 2 * hpad);
    const int* ra = qb + hpad;
    const int cols = C * nb;
    const Div dnb = mkdiv(nb), dns = mkdiv(Ns), dcols = mkdiv(cols);
    float4* UV = reinterpret_cast<float4*>(Y);      // [b < h][column]
    float2* X0 = Y + 2 * h * cols;                  // [column]; cols (2 h + 1) = C n <= C ldx
    for (int w = threadIdx.x; w < (h + 1) * cols; w += blockDim.x) {
        const int b = quo(w, dcols);
        const int col = w - b * cols;
        const int c = quo(col, dnb);
        const int i0 = col - c * nb;
        if (RAW) {
            const float* raw = reinterpret_cast<const float*>(X + c * ldx);
            if (b < h) {
                const int qn = qb[b] * nb;
                const float2 xq = make_float2(raw[i0 + qn], raw[n + i0 + qn]);
                const float2 xm = make_float2(raw[i0 + n - qn], raw[2 * n + i0 - qn]);
                UV[b * cols + col] = make_float4(xq.x + xm.x, xq.y + xm.y, xq.x - xm.x, xq.y - xm.y);
            } else {
                X0[col] = make_float2(raw[i0], raw[n + i0]);
            }
        } else {
            const float2* x = X + c * ldx + i0;
            if (b < h) {
                const int qn = qb[b] * nb;
                const float2 xq = x[qn], xm = x[n - qn];
                UV[b * cols + col] = make_float4(xq.x + xm.x, xq.y + xm.y, xq.x - xm.x, xq.y - xm.y);
            } else {
                X0[col] = x[0];
            }
        }
    }
    __syncthreads();
    // y_0 = x_0 + sum_b u_b
    for (int col = threadIdx.x; col < cols; col += blockDim.x) {
        const int c = quo(col, dnb);
        const int b = col - c * nb;
        const int k = b - quo(b, dns) * Ns;
        float2 s0 = X0[col], s1 = make_float2(0.f, 0.f);
        int q = 0;
        for (; q + 1 < h; q += 2) {
            const float4 a = UV[q * cols + col], e = UV[(q + 1) * cols + col];
            s0 = make_float2(s0.x + a.x, s0.y + a.y);
            s1 = make_float2(s1.x + e.x, s1.y + e.y);
        }
        if (q < h) {
            const float4 a = UV[q * cols + col];
            s0 = make_float2(s0.x + a.x, s0.y + a.y);
        }
        X[c * ldx + (b - k) * p + k] = cadd(s0, s1);
    }
    const int ng = hpad / GR;
    for (int w = threadIdx.x; w < cols * ng; w += blockDim.x) {
        const int g = quo(w, dcols);
        const int col = w - g * cols;
        const int c = quo(col, dnb);
        const int b = col - c * nb;
        const int k = b - quo(b, dns) * Ns;
        const int a0 = g * GR;
        float ar[GR], ai[GR], br[GR], bi[GR];
#pragma unroll
        for (int i = 0; i < GR; ++i) ar[i] = ai[i] = br[i] = bi[i] = 0.f;
        const float4* uv = UV + col;
        int B0 = 0;
        for (; B0 + GR <= h; B0 += GR) prime_block<false>(ar, ai, br, bi, uv, cols, T, h, B0, a0 - B0 + hpad - GR);
        if (B0 < h) prime_block<true>(ar, ai, br, bi, uv, cols, T, h, B0, a0 - B0 + hpad - GR);
        const float2 x0 = X0[col];
        float2* yo = X + c * ldx + (b - k) * p + k;
#pragma unroll
        for (int i = 0; i < GR; ++i) {
            const int a = a0 + i;
            if (a >= h) break;
            const int r = ra[a];
            float2 yr, ypr;
            if (!INV) {
                yr = make_float2(x0.x + ar[i] + bi[i], x0.y + ai[i] - br[i]);
                ypr = make_float2(x0.x + ar[i] - bi[i], x0.y + ai[i] + br[i]);
            } else {
                yr = make_float2(x0.x + ar[i] - bi[i], x0.y + ai[i] + br[i]);
                ypr = make_float2(x0.x + ar[i] + bi[i], x0.y + ai[i] - br[i]);
            }
            yo[r * Ns] = yr;
            yo[(p - r) * Ns] = ypr;
        }
    }
}

// Runs the stages from `first` on (1: the first, a prime radix, was done by the
// tensor-core kernel and its output is in X); returns the buffer holding the result.
// G: the ring's prime tables.
template <bool INV>
__device__ float2* run_fft(float2* X, float2* Y, int n, int ldx, int C, const RingDesc& rd, const float2* W,
                           const float2* G, bool raw_first = false, int first = 0) {
    int Ns = 1;
    if (first) {
        Ns = rd.fac[0];
        G += 3 * prime_hpad(rd.fac[0]);
    }
    for (int s = first; s < rd.nfac; ++s) {
        const int p = rd.fac[s];
        if (p > 8) {
            if (Ns > 1) {
                twiddle_pass<INV>(X, n, ldx, C, Ns, p, W);
                __syncthreads();
            }
            if (!INV && raw_first && s == 0)
                stage_prime<INV, true>(X, Y, n, ldx, C, Ns, p, G);    // result in X
            else
                stage_prime<INV, false>(X, Y, n, ldx, C, Ns, p, G);   // result in X
            G += 3 * prime_hpad(p);
            __syncthreads();
            Ns *= p;
            continue;
        } else if (!INV && raw_first && s == 0) {
            switch (p) {
                case 2: stage_small<2, INV, true, true>(X, Y, n, ldx, C, Ns, W); break;
                case 3: stage_small<3, INV, true, true>(X, Y, n, ldx, C, Ns, W); break;
                case 4: stage_small<4, INV, true, true>(X, Y, n, ldx, C, Ns, W); break;
                case 5: stage_small<5, INV, true, true>(X, Y, n, ldx, C, Ns, W); break;
                case 7: stage_small<7, INV, true, true>(X, Y, n, ldx, C, Ns, W); break;
                default: stage_small<8, INV, true, true>(X, Y, n, ldx, C, Ns, W); break;
            }
        } else if (Ns == 1) {
            switch (p) {
                case 2: stage_small<2, INV, true>(X, Y, n, ldx, C, Ns, W); break;
                case 3: stage_small<3, INV, true>(X, Y, n, ldx, C, Ns, W); break;
                case 4: stage_small<4, INV, true>(X, Y, n, ldx, C, Ns, W); break;
                case 5: stage_small<5, INV, true>(X, Y, n, ldx, C, Ns, W); break;
                case 7: stage_small<7, INV, true>(X, Y, n, ldx, C, Ns, W); break;
                default: stage_small<8, INV, true>(X, Y, n, ldx, C, Ns, W); break;
            }
        } else {
            switch (p) {
                case 2: stage_small<2, INV, false>(X, Y, n, ldx, C, Ns, W); break;
                case 3: stage_small<3, INV, false>(X, Y, n, ldx, C, Ns, W); break;
                case 4: stage_small<4, INV, false>(X, Y, n, ldx, C, Ns, W); break;
                case 5: stage_small<5, INV, false>(X, Y, n, ldx, C, Ns, W); break;
                case 7: stage_small<7, INV, false>(X, Y, n, ldx, C, Ns, W); break;
                default: stage_small<8, INV, false>(X, Y, n, ldx, C, Ns, W); break;
            }
        }
        __syncthreads();
        float2* t = X; X = Y; Y = t;
        Ns *= p;
    }
    return X;
}

__device__ __forceinline__ int smem_tw_len(int n) { return (n + 1) & ~1; }

// 16-byte asynchronous global -> shared copies (no register staging): a CTA issues
// all copies of its inputs at once, so its load phase is one memory round trip.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
// twiddles and prime tables (len float2, even; source 16-byte aligned)
__device__ __forceinline__ void copy_twiddles_async(float2* W, const float2* __restrict__ tw, int len) {
    for (int t = threadIdx.x; t < len / 2; t += blockDim.x) cp_async16(W + 2 * t, tw + 2 * t);
}

// X[c ldx + i] = (north ring value, south ring value) of layer k0 + c. Rings start at
// multiples of 4 points on these grids, so 16-byte vectors are used when the layer
// stride and base allow.
__device__ __forceinline__ void load_rings(float2* X, const float* __restrict__ grid, int64_t ldg, int64_t off_n,
                                           int64_t off_s, int k0, int C, int n, int ldx, Div dn) {
    const bool vec = ((ldg & 3) == 0) && ((reinterpret_cast<uintptr_t>(grid) & 15) == 0) && ((off_n & 3) == 0) &&
                     ((off_s & 3) == 0) && ((n & 3) == 0);
    if (vec) {
        const int n4 = n >> 2, tot = C * n4;
        const Div dn4 = mkdiv(n4);
        for (int w0 = threadIdx.x; w0 < tot; w0 += 4 * blockDim.x) {
            float4 a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int w = w0 + u * blockDim.x;
                if (w < tot) {
                    const int c = quo(w, dn4), i4 = w - c * n4;
                    const float* g = grid + (int64_t)(k0 + c) * ldg;
                    a[u] = __ldg(reinterpret_cast<const float4*>(g + off_n) + i4);
                    b[u] = __ldg(reinterpret_cast<const float4*>(g + off_s) + i4);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int w = w0 + u * blockDim.x;
                if (w < tot) {
                    const int c = quo(w, dn4), i4 = w - c * n4;
                    float4* x = reinterpret_cast<float4*>(X + c * ldx + 4 * i4);
                    x[0] = make_float4(a[u].x, b[u].x, a[u].y, b[u].y);
                    x[1] = make_float4(a[u].z, b[u].z, a[u].w, b[u].w);
                }
            }
        }
        return;
    }
    for (int w = threadIdx.x; w < C * n; w += blockDim.x) {
        const int c = quo(w, dn);
        const int i = w - c * n;
        const float* g = grid + (int64_t)(k0 + c) * ldg;
        X[c * ldx + i] = make_float2(g[off_n + i], g[off_s + i]);
    }
}

// grid rings of layer k0 + c (=, or += with add) <- (Re z, Im z)
__device__ __forceinline__ void store_rings(float* __restrict__ grid, int64_t ldg, int64_t off_n, int64_t off_s, int k0,
                                            int C, int n, int ldx, Div dn, const float2* z, int add) {
    const bool vec = ((ldg & 3) == 0) && ((reinterpret_cast<uintptr_t>(grid) & 15) == 0) && ((off_n & 3) == 0) &&
                     ((off_s & 3) == 0) && ((n & 3) == 0);
    if (vec) {
        const int n4 = n >> 2, tot = C * n4;
        const Div dn4 = mkdiv(n4);
        for (int w = threadIdx.x; w < tot; w += blockDim.x) {
            const int c = quo(w, dn4), i4 = w - c * n4;
            const float4* zz = reinterpret_cast<const float4*>(z + c * ldx + 4 * i4);
            const float4 p0 = zz[0], p1 = zz[1];
            float4 a = make_float4(p0.x, p0.z, p1.x, p1.z), b = make_float4(p0.y, p0.w, p1.y, p1.w);
            float4* gn = reinterpret_cast<float4*>(grid + (int64_t)(k0 + c) * ldg + off_n) + i4;
            float4* gs = reinterpret_cast<float4*>(grid + (int64_t)(k0 + c) * ldg + off_s) + i4;
            if (add) {
                const float4 on = *gn, os = *gs;
                a = make_float4(a.x + on.x, a.y + on.y, a.z + on.z, a.w + on.w);
                b = make_float4(b.x + os.x, b.y + os.y, b.z + os.z, b.w + os.w);
            }
            *gn = a;
            *gs = b;
        }
        return;
    }
    for (int w = threadIdx.x; w < C * n; w += blockDim.x) {
        const int c = quo(w, dn);
        const int i = w - c * n;
        float* g = grid + (int64_t)(k0 + c) * ldg;
        const float2 v = z[c * ldx + i];
        if (add) {
            g[off_n + i] += v.x;
            g[off_s + i] += v.y;
        } else {
            g[off_n + i] = v.x;
            g[off_s + i] = v.y;
        }
    }
}

// The next 16-bit piece (bf16 or fp16, round to nearest) of two reals r0 (low half) and
// r1 (high half), one paired rounding; the residuals r -= piece are formed only when
// another piece follows.
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

// Writes the 16-bit pieces (bf16 or fp16) of 8 reals as one 16-byte chunk per piece
// (pieces a tile apart); a partial chunk (mask of valid reals) is written element by
// element.
template <int NP, bool F16>
__device__ __forceinline__ void put_pieces(uint8_t* dst, int64_t piece_stride, const float (&v)[8], unsigned mask) {
    uint32_t w[NP][4];
#pragma unroll
    for (int h = 0; h < 4; ++h) {
        float r0 = v[2 * h], r1 = v[2 * h + 1];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            w[q][h] = q + 1 < NP ? piece_bits2<F16, true>(r0, r1) : piece_bits2<F16, false>(r0, r1);
        }
    }
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        uint8_t* d = dst + q * piece_stride;
        if (mask == 0xffu) {
            *reinterpret_cast<uint4*>(d) = make_uint4(w[q][0], w[q][1], w[q][2], w[q][3]);
        } else {
#pragma unroll
            for (int e = 0; e < 8; ++e)
                if (mask >> e & 1u) reinterpret_cast<uint16_t*>(d)[e] = (uint16_t)(w[q][e / 2] >> (16 * (e & 1)));
        }
    }
}

// shared memory: W (n twiddles, padded to even) | G (prime tables) | X (C ldx) | Y (C ldx);
// ldx >= n is the padded layer stride

// Weight of order m in the analysis epilogue, times (2 F_N +- 2 F_S): the solid angle
// / 2 for the transform; for the adjoint of the synthesis the rfft adjoint scale
// (1 for m = 0 and the Nyquist frequency, 2 otherwise; SpeedyTransformsEnzymeExt.jl:33-57)
// / 2, times 1/cos(lat) when the synthesis unscaled by it.
// image row of one order for one ring (analysis epilogue of tensor-core plans)
struct EpiRow {
    int64_t e;        // byte offset of the row in the E tile, without the column chunk
    int32_t o_tiles;  // tiles from the E tile to the O tile
    int32_t r8;       // swizzle phase (row mod 8)
};
static_assert(sizeof(EpiRow) == 16, "16 bytes per order fit the spare Stockham buffer");

__device__ __forceinline__ float ana_weight(const RingDesc& rd, int m, int adjoint, int unscale) {
    if (!adjoint) return 0.5f * rd.domega;
    const float sm = (m == 0 || 2 * m == rd.n) ? 1.f : 2.f;
    return 0.5f * sm * (unscale ? rd.coslat_inv : 1.f);
}

// grid -> Fourier scratch (E/O combinations weighted by the solid angle), one work
// item (ring, layer chunk) of one transform. IMG: the tensor-core operand-image epilogue
// is compiled in (the grouped batch launches, FP32 plans only, leave it out).
template <bool IMG>
__device__ void fft_analysis_body(const FftView& v, int ring, int chunk, float2* sm) {
    const RingDesc* __restrict__ rings = v.rings;
    const float2* __restrict__ twiddle = v.twiddle;
    const float* __restrict__ grid = v.gin;
    const int64_t ldg = v.ldg;
    float2* __restrict__ four = v.four;
    const int K = v.K;
    const TcImage& img = v.img;
    const int2 item = make_int2(ring, chunk);
    const RingDesc& rd = rings[item.x];
    const int k0 = item.y * rd.chunk;
    if (k0 >= K) return;
    const int C = min(rd.chunk, K - k0);
    const int n = rd.n;
    const int ldx = rd.ldx;
    const Div dn = mkdiv(n);
    float2* W = sm;
    float2* G = sm + smem_tw_len(n);
    float2* X = G + rd.gen_len;
    float2* Y = X + C * ldx;
    // Ring values of the C layers land raw in Y (layer c at Y + c ldx: n northern, then
    // n southern floats) by asynchronous copies issued together with the twiddles,
    // then are interleaved into X. In the aligned case they land raw in X instead and the
    // first FFT stage reads them in place (no interleave pass). Unaligned layouts take the
    // register path.
    const bool avec = ((ldg & 3) == 0) && ((reinterpret_cast<uintptr_t>(grid) & 15) == 0) &&
                      ((rd.off_north & 3) == 0) && ((rd.off_south & 3) == 0) && ((n & 3) == 0);
    const bool pre = v.ymid != nullptr && rd.pre;
    const bool raw_first = !pre && avec && rd.nfac > 0;
    float2* const land = raw_first ? X : Y;
    copy_twiddles_async(W, twiddle + rd.tw_off, smem_tw_len(n) + rd.gen_len);
    const int n4 = n >> 2;
    if (pre) {
        // the first stage's output, [k][n] per ring, straight into X (n even: 16-byte runs)
        const int n2 = n >> 1;
        const Div dn2 = mkdiv(n2);
        const float2* src0 = v.ymid + rd.yofs + (int64_t)k0 * n;
        for (int w = threadIdx.x; w < C * n2; w += blockDim.x) {
            const int c = quo(w, dn2);
            const int i2 = w - c * n2;
            cp_async16(X + c * ldx + 2 * i2, src0 + (int64_t)c * n + 2 * i2);
        }
    } else if (avec) {
        const Div d2n4 = mkdiv(2 * n4);
        for (int w = threadIdx.x; w < C * 2 * n4; w += blockDim.x) {
            const int c = quo(w, d2n4);
            const int r = w - c * 2 * n4;
            const int hs = r >= n4 ? 1 : 0;
            const int i4 = r - hs * n4;
            const float* src = grid + (int64_t)(k0 + c) * ldg + (hs ? rd.off_south : rd.off_north) + 4 * i4;
            cp_async16(reinterpret_cast<float*>(land + c * ldx) + hs * n + 4 * i4, src);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    if (raw_first || pre) {
        // the prime stage reads the raw layout, or the prime stage's output is in place
        // (visible after the barrier above)
    } else if (avec) {
        const Div dn4 = mkdiv(n4);
        for (int w = threadIdx.x; w < C * n4; w += blockDim.x) {
            const int c = quo(w, dn4);
            const int i4 = w - c * n4;
            const float* raw = reinterpret_cast<const float*>(Y + c * ldx);
            const float4 a = reinterpret_cast<const float4*>(raw)[i4];
            const float4 b = reinterpret_cast<const float4*>(raw + n)[i4];
            float4* x = reinterpret_cast<float4*>(X + c * ldx + 4 * i4);
            x[0] = make_float4(a.x, b.x, a.y, b.y);
            x[1] = make_float4(a.z, b.z, a.w, b.w);
        }
    } else {
        load_rings(X, grid, ldg, rd.off_north, rd.off_south, k0, C, n, ldx, dn);
    }
    if (!raw_first && !pre) __syncthreads();
    const float2* Z = run_fft<false>(X, Y, n, ldx, C, rd, W, G, raw_first, pre ? 1 : 0);
    const int adj = v.adjoint, unsc = v.unscale;
    const int nm = rd.mt + 1;
    if (IMG && img.base != nullptr) {
        // tensor-core operand: E (parity 0) and O (parity 1) split into 16-bit pieces,
        // written into the swizzled MN-major tile of (m, parity, ring block) at ring
        // row j - j0(m); 8 real columns (4 layers) form one 16-byte chunk
        const int cbeg = 2 * k0, cend = 2 * (k0 + C);
        const int gbeg = cbeg / 8, ngr = (cend + 7) / 8 - gbeg;
        const Div dngr = mkdiv(ngr);
        const int j = item.x;
        // per order: byte offset of this ring's row in the E tile (all but the column
        // chunk), distance to the O tile and the row's swizzle phase, computed once with
        // all table loads in flight, into the Stockham buffer the result does not occupy
        // (16 bytes per order <= its C ldx float2 since ldx >= 2 (mt + 1) and C >= 1)
        EpiRow* rows = reinterpret_cast<EpiRow*>(Z == X ? Y : X);
        const int64_t piece_span = (int64_t)(img.fp16 ? 2 : img.npieces) * img.tile_bytes;
        for (int m = threadIdx.x; m < nm; m += blockDim.x) {
            const int jj = j - img.j0[m];
            const int r = jj % 64;
            const int64_t t0 = img.tile_base[m] + jj / 64;
            rows[m] = EpiRow{t0 * piece_span + (r / 8) * 1024 + (r % 8) * 128, img.njt[m] * (img.fp16 ? 2 : img.npieces),
                             r % 8};
        }
        __syncthreads();
        for (int w = threadIdx.x; w < ngr * nm; w += blockDim.x) {
            const int m = quo(w, dngr);
            const int g = gbeg + (w - m * ngr);
            const int mm = m == 0 ? 0 : n - m;
            // layers 4 g .. 4 g + 3: real columns 8 g + 2 t (re) and 8 g + 2 t + 1 (im)
            float ev[8], ov[8];
            unsigned mask = 0;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const int kl = 4 * g + t - k0;
                ev[2 * t] = ev[2 * t + 1] = ov[2 * t] = ov[2 * t + 1] = 0.f;
                if (kl >= 0 && kl < C) {
                    const float2 a = Z[kl * ldx + m];
                    const float2 b = Z[kl * ldx + mm];
                    const float2 fn = make_float2(a.x + b.x, a.y - b.y);
                    const float2 fs = make_float2(a.y + b.y, b.x - a.x);
                    // fp16 pieces: the layer's data scale 2^(15 - e_k) folded into the weight
                    const float w0 = ana_weight(rd, m, adj, unsc);
                    const float hw = img.fp16 ? w0 * img.kscale[k0 + kl].y : w0;
                    ev[2 * t] = __fmul_rn(hw, fn.x + fs.x);
                    ev[2 * t + 1] = __fmul_rn(hw, fn.y + fs.y);
                    ov[2 * t] = __fmul_rn(hw, fn.x - fs.x);
                    ov[2 * t + 1] = __fmul_rn(hw, fn.y - fs.y);
                    mask |= 3u << (2 * t);
                }
            }
            // column block of 64 (8 KB apart), 8-row group, row, swizzled 16-byte chunk
            const EpiRow ro = rows[m];
            uint8_t* eb = reinterpret_cast<uint8_t*>(img.base) + ro.e + (int64_t)(g / 8) * 8192 +
                          (((g % 8) ^ ro.r8) * 16);
            const int64_t odist = (int64_t)ro.o_tiles * img.tile_bytes;
            if (img.fp16) {
                put_pieces<2, true>(eb, img.tile_bytes, ev, mask);
                put_pieces<2, true>(eb + odist, img.tile_bytes, ov, mask);
            } else if (img.npieces == 2) {
                put_pieces<2, false>(eb, img.tile_bytes, ev, mask);
                put_pieces<2, false>(eb + odist, img.tile_bytes, ov, mask);
            } else {
                put_pieces<3, false>(eb, img.tile_bytes, ev, mask);
                put_pieces<3, false>(eb + odist, img.tile_bytes, ov, mask);
            }
        }
        return;
    }
    // layer fastest across the lanes: a warp writes whole runs of C layers of a scratch
    // row; the padded layer stride of shared memory keeps the lanes' reads in distinct banks
    const Div dC = mkdiv(C);
    for (int w = threadIdx.x; w < C * nm; w += blockDim.x) {
        const int m = quo(w, dC);
        const int c = w - m * C;
        const float2 a = Z[c * ldx + m];
        const float2 b = Z[c * ldx + (m == 0 ? 0 : n - m)];
        // F_N = (a + conj b)/2, F_S = (a - conj b)/(2i)
        const float2 fn = make_float2(a.x + b.x, a.y - b.y);
        const float2 fs = make_float2(a.y + b.y, b.x - a.x);
        const float hw = ana_weight(rd, m, adj, unsc);
        const float2 e = make_float2(__fmul_rn(hw, fn.x + fs.x), __fmul_rn(hw, fn.y + fs.y));
        const float2 o = make_float2(__fmul_rn(hw, fn.x - fs.x), __fmul_rn(hw, fn.y - fs.y));
        const int64_t row = (rd.gofs + m) * 2;
        four[row * K + k0 + c] = e;
        four[(row + 1) * K + k0 + c] = o;
    }
}

// Fourier scratch -> grid, one work item (ring, layer chunk) of one transform
__device__ void fft_synthesis_body(const FftView& v, int ring, int chunk, float2* sm) {
    const RingDesc* __restrict__ rings = v.rings;
    const float2* __restrict__ twiddle = v.twiddle;
    const float2* __restrict__ four = v.four;
    float* __restrict__ grid = v.gout;
    const int64_t ldg = v.ldg;
    const int K = v.K, unscale = v.unscale, add = v.add;
    const int2 item = make_int2(ring, chunk);
    const RingDesc& rd = rings[item.x];
    const int k0 = item.y * rd.chunk;
    if (k0 >= K) return;
    const int C = min(rd.chunk, K - k0);
    const int n = rd.n;
    const int ldx = rd.ldx;
    const Div dn = mkdiv(n);
    float2* W = sm;
    float2* G = sm + smem_tw_len(n);
    float2* X = G + rd.gen_len;
    float2* Y = X + C * ldx;
    // The scratch rows r = 2 m + eo (m <= mt) of the C layers land in Y as [r][c] by
    // asynchronous copies issued together with the twiddles (2 (mt + 1) <= ldx). Odd
    // layer counts or offsets read the scratch directly.
    copy_twiddles_async(W, twiddle + rd.tw_off, smem_tw_len(n) + rd.gen_len);
    if (v.ymid != nullptr && rd.pre) {
        // the first stage ran on the tensor cores: its output, [k][n] per ring, into X
        const int n2 = n >> 1;
        const Div dn2 = mkdiv(n2);
        const float2* src0 = v.ymid + rd.yofs + (int64_t)k0 * n;
        for (int w = threadIdx.x; w < C * n2; w += blockDim.x) {
            const int c = quo(w, dn2);
            const int i2 = w - c * n2;
            cp_async16(X + c * ldx + 2 * i2, src0 + (int64_t)c * n + 2 * i2);
        }
        cp_async_wait_all();
        __syncthreads();
        const float2* z = run_fft<true>(X, Y, n, ldx, C, rd, W, G, false, 1);
        store_rings(grid, ldg, rd.off_north, rd.off_south, k0, C, n, ldx, dn, z, add);
        return;
    }
    const bool svec = ((K & 1) == 0) && ((k0 & 1) == 0) && ((C & 1) == 0) &&
                      ((reinterpret_cast<uintptr_t>(four) & 15) == 0);
    if (svec) {
        const int half = C / 2, nrow = 2 * (rd.mt + 1);
        const Div dh = mkdiv(half);
        const float2* src0 = four + 2 * rd.gofs * K + k0;
        for (int w = threadIdx.x; w < nrow * half; w += blockDim.x) {
            const int r = quo(w, dh);
            const int h = w - r * half;
            cp_async16(Y + r * C + 2 * h, src0 + (int64_t)r * K + 2 * h);
        }
    }
    cp_async_wait_all();
    __syncthreads();
    const int adj = v.adjoint;
    const int nhalf = n / 2;   // highest source frequency
    // layer fastest across the lanes (a warp reads whole runs of C layers of a scratch
    // row), four items per thread in flight: the scratch reads are the latency
    if (svec) {
        // staged rows, C even: an item is a pair of layers (16-byte loads of the row's run;
        // one index division and one weight per two layers), same arithmetic per value
        const int C2 = C / 2;
        const int tot2 = C2 * (nhalf + 1);
        const Div dC2 = mkdiv(C2);
        const float4* Y4 = reinterpret_cast<const float4*>(Y);
        for (int w0 = threadIdx.x; w0 < tot2; w0 += 4 * blockDim.x) {
            float4 e[4], o[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int w = w0 + u * blockDim.x;
                const int m = quo(w, dC2);
                const int c2 = w - m * C2;
                e[u] = o[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (w < tot2 && m <= rd.mt) {
                    e[u] = Y4[m * C + c2];          // Y[2 m C + 2 c2], two layers
                    o[u] = Y4[m * C + C2 + c2];     // Y[(2 m + 1) C + 2 c2]
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int w = w0 + u * blockDim.x;
                if (w >= tot2) break;
                const int m = quo(w, dC2);
                const int c = 2 * (w - m * C2);
                const float scale = syn_weight(rd, m, adj, unscale);
                const bool selfconj = (m == 0) || (2 * m == n);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const float2 eh = h ? make_float2(e[u].z, e[u].w) : make_float2(e[u].x, e[u].y);
                    const float2 oh = h ? make_float2(o[u].z, o[u].w) : make_float2(o[u].x, o[u].y);
                    const float2 gn = make_float2(__fmul_rn(scale, eh.x + oh.x), __fmul_rn(scale, eh.y + oh.y));
                    const float2 gs = make_float2(__fmul_rn(scale, eh.x - oh.x), __fmul_rn(scale, eh.y - oh.y));
                    float2* xr = X + (c + h) * ldx;
                    if (selfconj) {
                        xr[m] = make_float2(gn.x, gs.x);
                    } else {
                        xr[m] = make_float2(gn.x - gs.y, gn.y + gs.x);
                        xr[n - m] = make_float2(gn.x + gs.y, gs.x - gn.y);
                    }
                }
            }
        }
    }
    const int tot = svec ? 0 : C * (nhalf + 1);
    const Div dC = mkdiv(C);
    for (int w0 = threadIdx.x; w0 < tot; w0 += 4 * blockDim.x) {
        float2 e[4], o[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int w = w0 + u * blockDim.x;
            const int m = quo(w, dC);
            const int c = w - m * C;
            e[u] = o[u] = make_float2(0.f, 0.f);
            if (w < tot && m <= rd.mt) {
                const int64_t row = (rd.gofs + m) * 2;
                e[u] = four[row * K + k0 + c];
                o[u] = four[(row + 1) * K + k0 + c];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int w = w0 + u * blockDim.x;
            if (w >= tot) break;
            const int m = quo(w, dC);
            const int c = w - m * C;
            const float scale = syn_weight(rd, m, adj, unscale);
            // products rounded on their own (no contraction into the packing below)
            const float2 gn = make_float2(__fmul_rn(scale, e[u].x + o[u].x), __fmul_rn(scale, e[u].y + o[u].y));
            const float2 gs = make_float2(__fmul_rn(scale, e[u].x - o[u].x), __fmul_rn(scale, e[u].y - o[u].y));
            const bool selfconj = (m == 0) || (2 * m == n);
            if (selfconj) {
                X[c * ldx + m] = make_float2(gn.x, gs.x);
            } else {
                X[c * ldx + m] = make_float2(gn.x - gs.y, gn.y + gs.x);
                X[c * ldx + (n - m)] = make_float2(gn.x + gs.y, gs.x - gn.y);
            }
        }
    }
    __syncthreads();
    const float2* z = run_fft<true>(X, Y, n, ldx, C, rd, W, G);
    store_rings(grid, ldg, rd.off_north, rd.off_south, k0, C, n, ldx, dn, z, add);
}

__global__ void __launch_bounds__(kFftThreads, kFftCtasPerSm) fft_analysis_kernel(const int2* __restrict__ items,
                                                                                  const FftView v) {
    extern __shared__ float2 sm[];
    const int2 it = items[blockIdx.x];
    fft_analysis_body<true>(v, it.x, it.y, sm);
}

__global__ void __launch_bounds__(kFftThreads, kFftCtasPerSm) fft_synthesis_kernel(const int2* __restrict__ items,
                                                                                   const FftView v) {
    extern __shared__ float2 sm[];
    const int2 it = items[blockIdx.x];
    fft_synthesis_body(v, it.x, it.y, sm);
}

// Persistent grouped launch over the (ring, chunk) items of many transforms: CTA b
// takes the items b, b + gridDim.x, ... of the batch's list (task, ring, chunk).
// (one instantiation per direction: a single body per kernel keeps the registers in bounds)
template <bool SYN>
__global__ void __launch_bounds__(kFftGroupThreads, kFftCtasPerSm) fft_grouped_kernel(const FftView* __restrict__ views,
                                                                                 const GroupItem* __restrict__ items,
                                                                                 int nitems) {
    extern __shared__ float2 sm[];
    for (int ix = blockIdx.x; ix < nitems; ix += gridDim.x) {
        const GroupItem it = items[ix];
        __syncthreads();                  // the previous item is done with shared memory
        if (SYN)
            fft_synthesis_body(views[it.task], it.a, it.b, sm);
        else
            fft_analysis_body<false>(views[it.task], it.a, it.b, sm);
    }
}

// ---------------------------------------------------------------- fused transforms
// FFT and Legendre stage in one launch per direction, for FP32 plans whose per-cluster
// data fits in shared memory (the small truncations). A thread-block cluster of P CTAs
// handles one chunk of C layers; CTA `rank` owns the orders m = rank + P ml and the
// rings j = rank + P jl. The E/O Fourier rows pass between the two stages through the
// CTAs' shared memory (distributed shared memory within the cluster) instead of the
// global scratch:
//   synthesis  Legendre sums of my orders on every ring -> cluster barrier -> each of my
//              rings gathers its rows from the owners of its orders -> pack, FFT, store
//   analysis   FFT of my rings -> E/O rows of every order -> cluster barrier -> each of
//              my orders gathers its rows from the owners of the rings -> sums over the
//              rings in ring order
// Every value is computed with the same operations in the same order as by the separate
// Legendre and Fourier kernels (the Legendre sums are fma chains over l, resp. over the
// rings from j0(m) on; the FFT code is shared), so the two paths give the same bits.

__device__ __forceinline__ uint32_t cl_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cl_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// the float2 at the same shared-memory offset as p in the CTA of the cluster with rank r
__device__ __forceinline__ float2 cl_load(const float2* p, int r) {
    uint32_t a = (uint32_t)__cvta_generic_to_shared(p), b;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(b) : "r"(a), "r"(r));
    float2 v;
    asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(b) : "memory");
    return v;
}

constexpr int kFusedMaxC = 8;          // layers per cluster (register accumulators per thread)

__global__ void __launch_bounds__(kFftThreads, 1) fused_synthesis_kernel(const FusedView v) {
    extern __shared__ float2 sm[];
    const int P = v.P, rank = (int)cl_rank(), nh = v.nh;
    const int k0 = (blockIdx.x / P) * v.C;
    const int C = min(v.C, v.K - k0);
    float2* EOS = sm;                                             // [ml][j][p][c], stride v.C
    float2* TW = sm + (int64_t)v.nm_cta * nh * 2 * v.C;           // [jl][tw_max]: my rings' tables
    float2* X = TW + (int64_t)v.nr_cta * v.tw_max;
    float2* Y = X + (v.uniform ? v.nr_cta : 1) * v.C * v.ldx;
    // twiddles and prime tables of my rings, fetched while the Legendre sums run
    for (int j = rank, jl = 0; j < nh; j += P, ++jl) {
        const RingDesc& rd = v.rings[j];
        copy_twiddles_async(TW + (int64_t)jl * v.tw_max, v.twiddle + rd.tw_off, smem_tw_len(rd.n) + rd.gen_len);
    }
    // Legendre sums of my orders on every ring that carries them: a thread takes four
    // consecutive rings (one 16-byte load of Lambda per degree) and the C layers
    const int nj4 = (nh + 3) / 4;
    for (int w = threadIdx.x; w < v.nm_cta * 2 * nj4; w += blockDim.x) {
        const int j4 = w % nj4, mp = w / nj4, p = mp & 1, ml = mp >> 1;
        const int m = rank + P * ml;
        if (m >= v.mmax || 4 * j4 + 3 < v.j0[m]) continue;
        const int rows = v.rows[m];
        const int ni = min(rows, (v.lmax - m - p + 1) / 2);          // degrees l = m + 2 i + p < lmax
        const float4* L = reinterpret_cast<const float4*>(v.lam + v.lam_off[m] + (int64_t)p * rows * v.nh_pad) + j4;
        const int64_t ls = v.nh_pad / 4;
        const float2* cb = v.cin + (int64_t)k0 * v.ldc + v.lm_off[m] + p;
        float ar[4][kFusedMaxC], ai[4][kFusedMaxC];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int c = 0; c < kFusedMaxC; ++c) ar[q][c] = ai[q][c] = 0.f;
        int i = 0;
        for (; i + 4 <= ni; i += 4) {
            float4 lam[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) lam[u] = __ldg(L + (int64_t)(i + u) * ls);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float lq[4] = {lam[u].x, lam[u].y, lam[u].z, lam[u].w};
#pragma unroll
                for (int c = 0; c < kFusedMaxC; ++c) {
                    if (c < C) {
                        const float2 x = __ldg(cb + (int64_t)c * v.ldc + 2 * (i + u));
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            ar[q][c] = fmaf(lq[q], x.x, ar[q][c]);
                            ai[q][c] = fmaf(lq[q], x.y, ai[q][c]);
                        }
                    }
                }
            }
        }
        for (; i < ni; ++i) {
            const float4 l4 = __ldg(L + (int64_t)i * ls);
            const float lq[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
            for (int c = 0; c < kFusedMaxC; ++c) {
                if (c < C) {
                    const float2 x = __ldg(cb + (int64_t)c * v.ldc + 2 * i);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        ar[q][c] = fmaf(lq[q], x.x, ar[q][c]);
                        ai[q][c] = fmaf(lq[q], x.y, ai[q][c]);
                    }
                }
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = 4 * j4 + q;
            if (j < v.j0[m] || j >= nh) continue;
            float2* e = EOS + ((int64_t)(ml * nh + j) * 2 + p) * v.C;
#pragma unroll
            for (int c = 0; c < kFusedMaxC; ++c)
                if (c < C) e[c] = make_float2(ar[q][c], ai[q][c]);
        }
    }
    cp_async_wait_all();
    cl_sync();
    if (v.uniform) {
        // rings of one length (full grids): all my rings in one FFT, columns jl C + c
        const int R = rank < nh ? (nh - 1 - rank) / P + 1 : 0;
        if (R > 0) {
            const RingDesc& r0 = v.rings[rank];
            const int n = r0.n, ldx = v.ldx, CC = R * C, nrow = 2 * (r0.mt + 1);
            const float2* W = TW;
            const float2* G = W + smem_tw_len(n);
            for (int w = threadIdx.x; w < nrow * CC; w += blockDim.x) {
                const int r = w / CC, cc = w - r * CC, jl = cc / C, c = cc - jl * C, m = r >> 1, p = r & 1;
                const int j = rank + P * jl;
                Y[r * CC + cc] = cl_load(EOS + ((int64_t)((m / P) * nh + j) * 2 + p) * v.C + c, m % P);
            }
            __syncthreads();
            const int nhalf = n / 2;
            for (int w = threadIdx.x; w < CC * (nhalf + 1); w += blockDim.x) {
                const int m = w / CC, cc = w - m * CC;
                const RingDesc& rd = v.rings[rank + P * (cc / C)];
                float2 e = make_float2(0.f, 0.f), o = e;
                if (m <= rd.mt) {
                    e = Y[2 * m * CC + cc];
                    o = Y[(2 * m + 1) * CC + cc];
                }
                const float scale = syn_weight(rd, m, 0, v.unscale);
                const float2 gn = make_float2(__fmul_rn(scale, e.x + o.x), __fmul_rn(scale, e.y + o.y));
                const float2 gs = make_float2(__fmul_rn(scale, e.x - o.x), __fmul_rn(scale, e.y - o.y));
                if (m == 0 || 2 * m == n) {
                    X[cc * ldx + m] = make_float2(gn.x, gs.x);
                } else {
                    X[cc * ldx + m] = make_float2(gn.x - gs.y, gn.y + gs.x);
                    X[cc * ldx + (n - m)] = make_float2(gn.x + gs.y, gs.x - gn.y);
                }
            }
            __syncthreads();
            const float2* z = run_fft<true>(X, Y, n, ldx, CC, r0, W, G);
            const Div dn = mkdiv(n);
            for (int jl = 0; jl < R; ++jl) {
                const RingDesc& rd = v.rings[rank + P * jl];
                store_rings(v.gout, v.ldg, rd.off_north, rd.off_south, k0, C, n, ldx, dn, z + jl * C * ldx, v.add);
            }
        }
        cl_sync();
        return;
    }
    // my rings one after another: gather the rows, pack, FFT, store
    for (int j = rank; j < nh; j += P) {
        const RingDesc& rd = v.rings[j];
        const int n = rd.n, ldx = v.ldx;
        const float2* W = TW + (int64_t)(j / P) * v.tw_max;
        const float2* G = W + smem_tw_len(n);
        __syncthreads();                                          // the previous ring is done
        const int nrow = 2 * (rd.mt + 1);
        for (int w = threadIdx.x; w < nrow * C; w += blockDim.x) {
            const int r = w / C, c = w - r * C, m = r >> 1, p = r & 1;
            Y[r * C + c] = cl_load(EOS + ((int64_t)((m / P) * nh + j) * 2 + p) * v.C + c, m % P);
        }
        __syncthreads();
        const int nhalf = n / 2;
        for (int w = threadIdx.x; w < C * (nhalf + 1); w += blockDim.x) {
            const int m = w / C, c = w - m * C;
            float2 e = make_float2(0.f, 0.f), o = e;
            if (m <= rd.mt) {
                e = Y[2 * m * C + c];
                o = Y[(2 * m + 1) * C + c];
            }
            const float scale = syn_weight(rd, m, 0, v.unscale);
            const float2 gn = make_float2(__fmul_rn(scale, e.x + o.x), __fmul_rn(scale, e.y + o.y));
            const float2 gs = make_float2(__fmul_rn(scale, e.x - o.x), __fmul_rn(scale, e.y - o.y));
            if (m == 0 || 2 * m == n) {
                X[c * ldx + m] = make_float2(gn.x, gs.x);
            } else {
                X[c * ldx + m] = make_float2(gn.x - gs.y, gn.y + gs.x);
                X[c * ldx + (n - m)] = make_float2(gn.x + gs.y, gs.x - gn.y);
            }
        }
        __syncthreads();
        const float2* z = run_fft<true>(X, Y, n, ldx, C, rd, W, G);
        store_rings(v.gout, v.ldg, rd.off_north, rd.off_south, k0, C, n, ldx, mkdiv(n), z, v.add);
    }
    cl_sync();                                                    // my rows stay until all gathered
}

__global__ void __launch_bounds__(kFftThreads, 1) fused_analysis_kernel(const FusedView v) {
    extern __shared__ float2 sm[];
    const int P = v.P, rank = (int)cl_rank(), nh = v.nh;
    const int k0 = (blockIdx.x / P) * v.C;
    const int C = min(v.C, v.K - k0);
    const int nmr = v.mt_max + 1;
    float2* EOA = sm;                                             // [jl][m][p][c], stride v.C
    float2* TW = sm + (int64_t)v.nr_cta * nmr * 2 * v.C;          // [jl][tw_max]: my rings' tables
    float2* X = TW + (int64_t)v.nr_cta * v.tw_max;
    float2* Y = X + (v.uniform ? v.nr_cta : 1) * v.C * v.ldx;
    float2* EOM = TW;                                             // [ml][j][p][c] after the FFTs
    for (int j = rank, jl = 0; j < nh; j += P, ++jl) {
        const RingDesc& rd = v.rings[j];
        copy_twiddles_async(TW + (int64_t)jl * v.tw_max, v.twiddle + rd.tw_off, smem_tw_len(rd.n) + rd.gen_len);
    }
    // FFT of my rings and their E/O rows (the arithmetic of fft_analysis_body)
    if (v.uniform && rank < nh) {
        // rings of one length (full grids): all my rings in one FFT, columns jl C + c
        const int R = (nh - 1 - rank) / P + 1;
        const RingDesc& r0 = v.rings[rank];
        const int n = r0.n, ldx = v.ldx, CC = R * C, n4 = n >> 2;
        const float2* W = TW;
        const float2* G = W + smem_tw_len(n);
        bool avec = ((v.ldg & 3) == 0) && ((reinterpret_cast<uintptr_t>(v.gin) & 15) == 0) && ((n & 3) == 0);
        for (int jl = 0; jl < R; ++jl) {
            const RingDesc& rd = v.rings[rank + P * jl];
            avec = avec && ((rd.off_north & 3) == 0) && ((rd.off_south & 3) == 0);
        }
        const bool raw_first = avec && r0.nfac > 0;
        float2* const land = raw_first ? X : Y;
        if (avec) {
            const Div d2n4 = mkdiv(2 * n4);
            for (int w = threadIdx.x; w < CC * 2 * n4; w += blockDim.x) {
                const int cc = quo(w, d2n4);
                const int r = w - cc * 2 * n4;
                const int hs = r >= n4 ? 1 : 0;
                const int i4 = r - hs * n4;
                const int jl = cc / C, c = cc - jl * C;
                const RingDesc& rd = v.rings[rank + P * jl];
                const float* src = v.gin + (int64_t)(k0 + c) * v.ldg + (hs ? rd.off_south : rd.off_north) + 4 * i4;
                cp_async16(reinterpret_cast<float*>(land + cc * ldx) + hs * n + 4 * i4, src);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        if (raw_first) {
        } else if (avec) {
            const Div dn4 = mkdiv(n4);
            for (int w = threadIdx.x; w < CC * n4; w += blockDim.x) {
                const int cc = quo(w, dn4);
                const int i4 = w - cc * n4;
                const float* raw = reinterpret_cast<const float*>(Y + cc * ldx);
                const float4 a = reinterpret_cast<const float4*>(raw)[i4];
                const float4 b = reinterpret_cast<const float4*>(raw + n)[i4];
                float4* x = reinterpret_cast<float4*>(X + cc * ldx + 4 * i4);
                x[0] = make_float4(a.x, b.x, a.y, b.y);
                x[1] = make_float4(a.z, b.z, a.w, b.w);
            }
        } else {
            for (int jl = 0; jl < R; ++jl) {
                const RingDesc& rd = v.rings[rank + P * jl];
                load_rings(X + jl * C * ldx, v.gin, v.ldg, rd.off_north, rd.off_south, k0, C, n, ldx, mkdiv(n));
            }
        }
        if (!raw_first) __syncthreads();
        const float2* Z = run_fft<false>(X, Y, n, ldx, CC, r0, W, G, raw_first);
        const int nm = r0.mt + 1;
        for (int w = threadIdx.x; w < CC * nm; w += blockDim.x) {
            const int m = w / CC, cc = w - m * CC, jl = cc / C, c = cc - jl * C;
            const RingDesc& rd = v.rings[rank + P * jl];
            const float2 a = Z[cc * ldx + m];
            const float2 b = Z[cc * ldx + (m == 0 ? 0 : n - m)];
            const float2 fn = make_float2(a.x + b.x, a.y - b.y);
            const float2 fs = make_float2(a.y + b.y, b.x - a.x);
            const float hw = ana_weight(rd, m, 0, 0);
            float2* eo = EOA + ((int64_t)(jl * nmr + m) * 2) * v.C + c;
            eo[0] = make_float2(__fmul_rn(hw, fn.x + fs.x), __fmul_rn(hw, fn.y + fs.y));
            eo[v.C] = make_float2(__fmul_rn(hw, fn.x - fs.x), __fmul_rn(hw, fn.y - fs.y));
        }
    }
    for (int j = rank, jl = 0; j < nh && !v.uniform; j += P, ++jl) {
        const RingDesc& rd = v.rings[j];
        const int n = rd.n, ldx = v.ldx;
        const float2* W = TW + (int64_t)jl * v.tw_max;
        const float2* G = W + smem_tw_len(n);
        __syncthreads();
        const bool avec = ((v.ldg & 3) == 0) && ((reinterpret_cast<uintptr_t>(v.gin) & 15) == 0) &&
                          ((rd.off_north & 3) == 0) && ((rd.off_south & 3) == 0) && ((n & 3) == 0);
        const bool raw_first = avec && rd.nfac > 0;
        float2* const land = raw_first ? X : Y;
        const int n4 = n >> 2;
        if (avec) {
            const Div d2n4 = mkdiv(2 * n4);
            for (int w = threadIdx.x; w < C * 2 * n4; w += blockDim.x) {
                const int c = quo(w, d2n4);
                const int r = w - c * 2 * n4;
                const int hs = r >= n4 ? 1 : 0;
                const int i4 = r - hs * n4;
                const float* src = v.gin + (int64_t)(k0 + c) * v.ldg + (hs ? rd.off_south : rd.off_north) + 4 * i4;
                cp_async16(reinterpret_cast<float*>(land + c * ldx) + hs * n + 4 * i4, src);
            }
        }
        cp_async_wait_all();
        __syncthreads();
        if (raw_first) {
        } else if (avec) {
            const Div dn4 = mkdiv(n4);
            for (int w = threadIdx.x; w < C * n4; w += blockDim.x) {
                const int c = quo(w, dn4);
                const int i4 = w - c * n4;
                const float* raw = reinterpret_cast<const float*>(Y + c * ldx);
                const float4 a = reinterpret_cast<const float4*>(raw)[i4];
                const float4 b = reinterpret_cast<const float4*>(raw + n)[i4];
                float4* x = reinterpret_cast<float4*>(X + c * ldx + 4 * i4);
                x[0] = make_float4(a.x, b.x, a.y, b.y);
                x[1] = make_float4(a.z, b.z, a.w, b.w);
            }
        } else {
            load_rings(X, v.gin, v.ldg, rd.off_north, rd.off_south, k0, C, n, ldx, mkdiv(n));
        }
        if (!raw_first) __syncthreads();
        const float2* Z = run_fft<false>(X, Y, n, ldx, C, rd, W, G, raw_first);
        const int nm = rd.mt + 1;
        for (int w = threadIdx.x; w < C * nm; w += blockDim.x) {
            const int m = w / C, c = w - m * C;
            const float2 a = Z[c * ldx + m];
            const float2 b = Z[c * ldx + (m == 0 ? 0 : n - m)];
            const float2 fn = make_float2(a.x + b.x, a.y - b.y);
            const float2 fs = make_float2(a.y + b.y, b.x - a.x);
            const float hw = ana_weight(rd, m, 0, 0);
            float2* eo = EOA + ((int64_t)(jl * nmr + m) * 2) * v.C + c;
            eo[0] = make_float2(__fmul_rn(hw, fn.x + fs.x), __fmul_rn(hw, fn.y + fs.y));
            eo[v.C] = make_float2(__fmul_rn(hw, fn.x - fs.x), __fmul_rn(hw, fn.y - fs.y));
        }
    }
    cl_sync();
    // my orders' rows from every ring that carries them
    __syncthreads();
    for (int w = threadIdx.x; w < v.nm_cta * nh * 2 * C; w += blockDim.x) {
        const int c = w % C, r = w / C, p = r & 1, mj = r >> 1, j = mj % nh, ml = mj / nh;
        const int m = rank + P * ml;
        if (m >= v.mmax || j < v.j0[m]) continue;
        EOM[((int64_t)(ml * nh + j) * 2 + p) * v.C + c] =
            cl_load(EOA + ((int64_t)((j / P) * nmr + m) * 2 + p) * v.C + c, j % P);
    }
    cl_sync();                                                    // every gather done: no remote reads follow
    // Legendre sums over the rings j0(m) .. nh - 1, in ring order, for my orders
    const int rmax = (v.lmax + 1) / 2;
    for (int w = threadIdx.x; w < v.nm_cta * 2 * rmax; w += blockDim.x) {
        const int i = w % rmax, mp = w / rmax, p = mp & 1, ml = mp >> 1;
        const int m = rank + P * ml;
        if (m >= v.mmax) continue;
        const int rows = v.rows[m];
        if (i >= rows || m + 2 * i + p >= v.lmax) continue;
        const float* L = v.lam + v.lam_off[m] + ((int64_t)p * rows + i) * v.nh_pad;
        const float2* eo = EOM + ((int64_t)ml * nh * 2 + p) * v.C;
        float ar[kFusedMaxC], ai[kFusedMaxC];
#pragma unroll
        for (int c = 0; c < kFusedMaxC; ++c) ar[c] = ai[c] = 0.f;
        // rings j0(m) .. nh - 1 in order; Lambda four rings per 16-byte load
        const int jb = v.j0[m] & ~3;
        for (int j4 = jb; j4 < nh; j4 += 4) {
            const float4 l4 = __ldg(reinterpret_cast<const float4*>(L + j4));
            const float lq[4] = {l4.x, l4.y, l4.z, l4.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = j4 + q;
                if (j < v.j0[m] || j >= nh) continue;
#pragma unroll
                for (int c = 0; c < kFusedMaxC; ++c) {
                    if (c < C) {
                        const float2 x = eo[(int64_t)j * 2 * v.C + c];
                        ar[c] = fmaf(lq[q], x.x, ar[c]);
                        ai[c] = fmaf(lq[q], x.y, ai[c]);
                    }
                }
            }
        }
        float2* dst = v.cout + (int64_t)k0 * v.ldc + v.lm_off[m] + 2 * i + p;
#pragma unroll
        for (int c = 0; c < kFusedMaxC; ++c) {
            if (c < C) {
                float2 x = make_float2(ar[c], ai[c]);
                if (v.add) {
                    const float2 o = dst[(int64_t)c * v.ldc];
                    x.x += o.x;
                    x.y += o.y;
                }
                dst[(int64_t)c * v.ldc] = x;
            }
        }
    }
}

}  // namespace

static int fft_threads(const Plan&) { return kFftThreads; }

FftView fft_view(const Plan& p, const float* gin, float* gout, int64_t ldg, float2* four, int K, unsigned flags,
                 bool image, bool adjoint) {
    FftView v{};
    v.rings = p.d_rings;
    v.twiddle = p.d_twiddle;
    v.gin = gin;
    v.gout = gout;
    v.ldg = ldg;
    v.four = four;
    v.K = K;
    v.unscale = (flags & SHT_UNSCALE_COSLAT) ? 1 : 0;
    v.add = (flags & SHT_ADD) ? 1 : 0;
    v.adjoint = adjoint ? 1 : 0;
    if (image) v.img = p.ana_img;
    v.ymid = nullptr;   // set by the launches that run the tensor-core first stages
    return v;
}

cudaError_t launch_fft_grouped(const FftView* views, const GroupItem* items, int nitems, bool synthesis, int smem,
                               int grid, cudaStream_t s) {
    if (nitems == 0) return cudaSuccess;
    const int g = std::max(1, std::min(nitems, grid));
    if (synthesis)
        fft_grouped_kernel<true><<<g, kFftGroupThreads, smem, s>>>(views, items, nitems);
    else
        fft_grouped_kernel<false><<<g, kFftGroupThreads, smem, s>>>(views, items, nitems);
    return cudaGetLastError();
}

cudaError_t launch_fft_analysis(const Plan& p, const float* grid, int64_t ldg, int K, cudaStream_t s, bool to_image,
                                unsigned flags, bool adjoint) {
    const dim3 g(p.n_fft_items);
    if ((to_image || p.tc) && p.ana_img.fp16) {
        // bound of |E|, |O| per unit grid value: 4 pi max w (the transform: E = dOmega (F_N + F_S),
        // |F| <= n max|f|) or, for the adjoint of the synthesis (E = s_m c (F_N + F_S), s_m <= 2),
        // 4 nlon_max max(1 / cos lat)
        const float mul = adjoint ? 4.0000005f * p.nlon_max * ((flags & SHT_UNSCALE_COSLAT) ? p.coslat_inv_max : 1.f)
                                  : 0.f;
        const cudaError_t e = tc_analysis_scale(p, grid, ldg, K, s, mul);
        if (e != cudaSuccess) return e;
    }
    FftView v = fft_view(p, grid, nullptr, ldg, p.d_four, K, flags & SHT_UNSCALE_COSLAT, to_image || p.tc, adjoint);
    if ((v.ymid = prime_buffer(p)) != nullptr) {
        const cudaError_t e = launch_prime_stage(p, false, grid, ldg, K, flags, adjoint, s);
        if (e != cudaSuccess) return e;
    }
    fft_analysis_kernel<<<g, fft_threads(p), p.smem_fft, s>>>(p.d_fft_items, v);
    return cudaGetLastError();
}

cudaError_t launch_fft_synthesis(const Plan& p, float* grid, int64_t ldg, int K, unsigned flags, cudaStream_t s,
                                 bool adjoint) {
    const dim3 g(p.n_fft_items);
    FftView v = fft_view(p, nullptr, grid, ldg, p.d_four, K, flags, false, adjoint);
    if ((v.ymid = prime_buffer(p)) != nullptr) {
        const cudaError_t e = launch_prime_stage(p, true, nullptr, 0, K, flags, adjoint, s);
        if (e != cudaSuccess) return e;
    }
    fft_synthesis_kernel<<<g, fft_threads(p), p.smem_fft, s>>>(p.d_fft_items, v);
    return cudaGetLastError();
}

// The limit is a property of the kernel, not of a plan: it is raised to the per-CTA
// budget (or a larger plan's need) and never lowered, so plans of any size coexist.
cudaError_t fft_set_smem(int bytes) {
    static std::mutex mu;
    static std::map<int, int> current;     // per device (the attribute is per context)
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    bytes = std::max(bytes, kFftSmemBudget);
    std::lock_guard<std::mutex> lock(mu);
    if (bytes <= current[dev]) return cudaSuccess;
    e = cudaFuncSetAttribute(fft_analysis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fft_grouped_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(fft_grouped_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(fft_synthesis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) current[dev] = bytes;
    return e;
}

namespace {
// Layers per cluster of one call: enough that every cluster runs at once (no second
// wave), and at least one CTA per SM's share of the layers.
int fused_layers(const Plan& p, int K) {
    const int once = (K + p.fused_ncl - 1) / p.fused_ncl;
    const int fill = (K * p.fused_P + p.nsm - 1) / p.nsm;
    return std::max(1, std::min(p.fused_cmax, std::min(std::max(once, fill), K)));
}
int fused_smem(const Plan& p, bool syn, int C) {
    const int nm_cta = (p.mmax + p.fused_P - 1) / p.fused_P, nr_cta = (p.nh + p.fused_P - 1) / p.fused_P;
    const int64_t work = (int64_t)nr_cta * p.fused_tw_max + 2LL * C * p.fused_ldx * (p.fused_uniform ? nr_cta : 1);
    const int64_t eos = (int64_t)nm_cta * p.nh * 2 * C;
    const int64_t f2 = syn ? eos + work : (int64_t)nr_cta * (p.fused_mt_max + 1) * 2 * C + std::max(work, eos);
    return (int)(f2 * (int64_t)sizeof(float2));
}
FusedView fused_view(const Plan& p, int K, int C) {
    FusedView v{};
    v.rings = p.d_rings;
    v.twiddle = p.d_twiddle;
    v.lam = p.d_lam;
    v.lam_off = p.d_lam_off;
    v.rows = p.d_rows;
    v.j0 = p.d_j0;
    v.lm_off = p.d_lm_off;
    v.nh = p.nh;
    v.nh_pad = p.nh_pad;
    v.lmax = p.lmax;
    v.mmax = p.mmax;
    v.mt_max = p.fused_mt_max;
    v.K = K;
    v.C = C;
    v.P = p.fused_P;
    v.nm_cta = (p.mmax + p.fused_P - 1) / p.fused_P;
    v.nr_cta = (p.nh + p.fused_P - 1) / p.fused_P;
    v.ldx = p.fused_ldx;
    v.tw_max = p.fused_tw_max;
    v.uniform = p.fused_uniform;
    return v;
}
cudaError_t fused_launch(const Plan& p, bool syn, const FusedView& v, cudaStream_t s) {
    const int ncl = (v.K + v.C - 1) / v.C;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(v.P * ncl);
    cfg.blockDim = dim3(kFftThreads);
    cfg.dynamicSmemBytes = fused_smem(p, syn, v.C);
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = v.P;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return syn ? cudaLaunchKernelEx(&cfg, fused_synthesis_kernel, v) : cudaLaunchKernelEx(&cfg, fused_analysis_kernel, v);
}
}  // namespace

// Launch shape of the fused kernels: the cluster size (16 or 8 CTAs) with more CTAs
// resident at once (cudaOccupancyMaxActiveClusters), and the most layers per cluster
// (<= 8) whose shared memory fits one CTA per SM. Tensor-core plans, and plans too large
// for one layer per cluster, keep the separate kernels (fusion_ok = 0). A CTA transforms
// its rings one after another, unless all rings have one length (full grids): then in
// one FFT call with rings x layers as its columns.
cudaError_t fused_prepare(Plan& p) {
    p.fusion_ok = 0;
    p.fusion = 0;
    if (p.tc) return cudaSuccess;
    int dev = 0, nsm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    p.nsm = std::max(1, nsm);
    int ldx = 2, tw = 0, mtm = 0;
    for (const RingDesc& r : p.h_rings) {
        const int base = std::max(r.n, 2 * (r.mt + 1));
        ldx = std::max(ldx, base + (((2 - base) % 16) + 16) % 16);
        tw = std::max(tw, ((r.n + 1) & ~1) + r.gen_len);
        mtm = std::max(mtm, r.mt);
    }
    p.fused_ldx = ldx;
    p.fused_tw_max = tw;
    p.fused_mt_max = mtm;
    p.fused_uniform = 1;                              // every ring of one length and truncation
    for (const RingDesc& r : p.h_rings)
        if (r.n != p.h_rings[0].n || r.mt != p.h_rings[0].mt) p.fused_uniform = 0;
    const int budget = 227 * 1024;
    const void* ks[2] = {(const void*)fused_synthesis_kernel, (const void*)fused_analysis_kernel};
    for (const void* k : ks) {
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, budget)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1)) != cudaSuccess) return e;
    }
    int best_P = 0, best_c = 0, best_ncl = 0;
    for (int P : {16, 8}) {
        p.fused_P = std::max(1, std::min(P, p.nh));
        int cmax = 0;
        for (int C = kFusedMaxC; C >= 1; --C)
            if (fused_smem(p, true, C) <= budget && fused_smem(p, false, C) <= budget) {
                cmax = C;
                break;
            }
        if (cmax == 0) continue;
        int ncl = 1 << 30;
        for (int d = 0; d < 2; ++d) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(p.fused_P);
            cfg.blockDim = dim3(kFftThreads);
            cfg.dynamicSmemBytes = fused_smem(p, d == 0, cmax);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = p.fused_P;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, ks[d], &cfg) != cudaSuccess) {
                cudaGetLastError();
                n = 0;
            }
            ncl = std::min(ncl, n);
        }
        if (ncl >= 1 && ncl * p.fused_P > best_ncl * best_P) {
            best_P = p.fused_P;
            best_c = cmax;
            best_ncl = ncl;
        }
    }
    if (best_P == 0) return cudaSuccess;              // does not fit: separate kernels
    p.fused_P = best_P;
    p.fused_cmax = best_c;
    p.fused_ncl = best_ncl;
    p.fusion_ok = 1;
    // on by default where it measured faster than the separate kernels on B200: full
    // grids (one FFT per CTA for all its rings) up to nlat 64
    p.fusion = p.fused_uniform && p.nlat <= 64 ? 1 : 0;
    return cudaSuccess;
}

cudaError_t launch_fused_synthesis(const Plan& p, const float2* coeffs, int64_t ldc, float* grid, int64_t ldg, int K,
                                   unsigned flags, cudaStream_t s) {
    FusedView v = fused_view(p, K, fused_layers(p, K));
    v.cin = coeffs;
    v.ldc = ldc;
    v.gout = grid;
    v.ldg = ldg;
    v.unscale = (flags & SHT_UNSCALE_COSLAT) ? 1 : 0;
    v.add = (flags & SHT_ADD) ? 1 : 0;
    return fused_launch(p, true, v, s);
}

cudaError_t launch_fused_analysis(const Plan& p, const float* grid, int64_t ldg, float2* coeffs, int64_t ldc, int K,
                                  bool add, cudaStream_t s) {
    FusedView v = fused_view(p, K, fused_layers(p, K));
    v.gin = grid;
    v.ldg = ldg;
    v.cout = coeffs;
    v.ldc = ldc;
    v.add = add ? 1 : 0;
    return fused_launch(p, false, v, s);
}

}  // namespace sht

namespace sht {
// The analysis Fourier kernel writing FP32 coefficients into a caller-chosen scratch
// (used by the static-scratch analysis entry point).
cudaError_t launch_fft_analysis_to(const Plan& p, const float* grid, int64_t ldg, int K, float2* scratch,
                                   cudaStream_t s) {
    const dim3 g(p.n_fft_items);
    fft_analysis_kernel<<<g, fft_threads(p), p.smem_fft, s>>>(
        p.d_fft_items, fft_view(p, grid, nullptr, ldg, scratch, K, 0, false, false));
    return cudaGetLastError();
}
}  // namespace sht
