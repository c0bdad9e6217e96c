// First stage of the ring FFTs whose first radix is a large prime p (>= kPrimeTcMin),
// on the tensor cores: tcgen05.mma kind::tf32, three TF32 products, FP32 accumulation.
//
// Replaces, for those rings, the direct prime-radix stage of the mixed-radix FFT that
// stands in for the per-ring FFTW/cuFFT plans of SpeedyTransforms/src/fourier.jl:129-166
// (rfft, analysis) and :215-250 (irfft, synthesis).
//
// The FFT of a ring of n = p nb points (both hemispheres packed as z = f_N + i f_S, or
// the packed spectrum for the inverse) starts with nb DFTs of length p over the columns
// x_q = z[i0 + q nb] (i0 < nb). With h = (p - 1) / 2, u_q = x_q + x_(p-q), v_q = x_q -
// x_(p-q) (u_0 = x_0, v_0 = 0) and the p x p DFT folded onto its symmetric halves,
//   A_r = sum_(q=0..h) cos(2 pi r q / p) u_q,    B_r = sum_(q=1..h) sin(2 pi r q / p) v_q,
//   y_r = A_r -+ i B_r,  y_(p-r) = A_r +- i B_r   (forward / inverse; r = 0..h)
// (A_0 = x_0 + sum u_q is y_0.) Over all layers and columns of a ring this is two real
// matrix products with the (h + 1) x (h + 1) cosine and sine matrices, M = the outputs r
// (one or two 128-row tiles), K = q, N = the real and imaginary parts of the columns. The
// output goes to the prime buffer in the layout the FFT kernel's next stage reads,
// y[k][i0 p + r] per ring, and the FFT kernel runs the remaining stages from there.
//
// Precision. x = hi + lo with hi = tf32(x), lo = tf32(x - hi), both rounded to nearest
// (22 significant bits together). With the data pieces stacked along N, one MMA of the
// matrix's hi piece against [D_hi; D_lo] writes the leading product and the first cross
// product to separate accumulators; a second MMA adds M_lo D_hi to the cross one. The
// tensor core truncates each accumulator update; the leading accumulator takes one update
// per 8 terms (at most 25 for p <= 389), and the two are added with rounding to nearest.
//
// Data flow. The matrices of each prime are stored once, when the mode is first turned
// on, as swizzled (SWIZZLE_128B, K-major) FP32 tiles of 128 rows x 32 deep, contiguous per
// (k-block, matrix), and reach shared memory by one bulk copy per k-block. Two groups of
// four builder warps take alternate (k-block, matrix) units: they read the stage's inputs
// (grid rings, or Fourier scratch rows expanded to the packed spectrum exactly as the FFT
// kernel does; 16-byte loads of four columns where the layout allows), form u or v, split
// them and write the swizzled data tile. One thread issues the MMAs; eight warps (two per
// TMEM lane quarter) drain the accumulators and store y.
// Work item: (ring, 64 or 32 complex columns), costliest first, on a persistent grid of
// one CTA per SM. Every wait is bounded (one second); on expiry the CTA records an error
// in the plan's status word, stops, waits for its copies and MMAs in flight and frees its
// tensor memory.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "sht_internal.h"
#include "tc_ptx.cuh"

namespace sht {

namespace {

using namespace tcx;

constexpr int PT_THREADS = 576;               // warp 0 copies, 1 MMAs, 2-9 builders, 10-17 drain
constexpr int PT_BUILDERS = 8;                // two groups of four warps, alternate units
constexpr int PT_GROUP = 4;                   // warps per builder group
constexpr int PT_DRAIN = 8;                   // drain warps, two per TMEM lane quarter
constexpr int PT_TILE = 16384;                // 128 rows x 32 FP32 (128 bytes per row)
constexpr int PT_A_SLOT = 4 * PT_TILE;        // matrix pieces (hi, lo) of up to two row tiles
constexpr int PT_B_SLOT = 2 * PT_TILE;        // data pieces [hi rows; lo rows], up to 128 + 128 rows
constexpr int PT_A_SLOTS = 2, PT_B_SLOTS = 3;
constexpr int PT_BAR_OFF = PT_A_SLOTS * PT_A_SLOT + PT_B_SLOTS * PT_B_SLOT;
constexpr int PT_SMEM = PT_BAR_OFF + 256 + 1024;

struct PrimeRing {
    int32_t ring;       // index into the plan's rings
    int32_t p, h, nb;   // prime, (p - 1) / 2, n / p
    int32_t kb;         // 32-deep k-blocks of K = h + 1
    int32_t mtiles;     // 128-row tiles of M = h + 1 (1 or 2)
    int32_t nc;         // real data columns per work item: 128 (one row tile) or 64
    int32_t spare;
    int64_t mofs;       // float offset of the prime's matrix tiles
};

struct PtArgs {
    const RingDesc* rings;
    const PrimeRing* prs;
    const int2* items;    // (prime ring, column tile), costliest first
    int nitems;
    const float* mat;
    const float* grid;    // analysis input
    int64_t ldg;
    const float2* four;   // synthesis input (Fourier scratch [row][k])
    float2* ymid;
    int K, unscale, adjoint;
    int32_t* err;
};

__host__ __device__ __forceinline__ int pt_swz(int row, int col) {
    return row * 32 + ((((col >> 2) ^ row) & 7) << 2) + (col & 3);
}
// tf32(x) rounded to nearest, ties away from zero (finite x): add half a unit of the
// 11-bit significand's last place to the magnitude bits and clear the 13 low bits
__host__ __device__ __forceinline__ uint32_t tf32_bits(uint32_t b) { return (b + 0x1000u) & 0xFFFFE000u; }
__device__ __forceinline__ float tf32_rn(float x) { return __uint_as_float(tf32_bits(__float_as_uint(x))); }

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Complex columns of a ring for K layers: analysis c = k nb + i0 (the ring's points
// consecutive across the lanes), synthesis c = i0 K + k (the scratch's layers consecutive).
template <bool SYN>
__device__ __forceinline__ void col_of(int c, int nb, int K, int& k, int& i0) {
    if (SYN) {
        i0 = c / K;
        k = c - i0 * K;
    } else {
        k = c / nb;
        i0 = c - k * nb;
    }
}

// z_t of layer k: the ring pair's values (analysis) or the packed spectrum the FFT
// kernel's synthesis prologue builds from the scratch rows (same operations).
template <bool SYN>
__device__ __forceinline__ float2 stage_input(const PtArgs& a, const RingDesc& rd, int k, int t) {
    if (!SYN) {
        const float* g = a.grid + (int64_t)k * a.ldg;
        return make_float2(__ldg(g + rd.off_north + t), __ldg(g + rd.off_south + t));
    }
    const int n = rd.n;
    const int m = 2 * t <= n ? t : n - t;
    if (m > rd.mt) return make_float2(0.f, 0.f);
    const int64_t row = (rd.gofs + m) * 2;
    const float2 e = __ldg(a.four + row * a.K + k), o = __ldg(a.four + (row + 1) * a.K + k);
    const float scale = syn_weight(rd, m, a.adjoint, a.unscale);
    const float2 gn = make_float2(__fmul_rn(scale, e.x + o.x), __fmul_rn(scale, e.y + o.y));
    const float2 gs = make_float2(__fmul_rn(scale, e.x - o.x), __fmul_rn(scale, e.y - o.y));
    if (m == 0 || 2 * m == n) return make_float2(gn.x, gs.x);
    if (2 * t < n) return make_float2(gn.x - gs.y, gn.y + gs.x);
    return make_float2(gn.x + gs.y, gs.x - gn.y);
}

// hi and lo pieces of four q-values (chunk jc of the k-block) of one data row
__device__ __forceinline__ void put_row(float* hi, float* lo, int row, int jc, float4 v) {
    float4 h, l;
    h.x = tf32_rn(v.x); l.x = tf32_rn(v.x - h.x);
    h.y = tf32_rn(v.y); l.y = tf32_rn(v.y - h.y);
    h.z = tf32_rn(v.z); l.z = tf32_rn(v.z - h.z);
    h.w = tf32_rn(v.w); l.w = tf32_rn(v.w - h.w);
    *reinterpret_cast<float4*>(hi + pt_swz(row, 4 * jc)) = h;
    *reinterpret_cast<float4*>(lo + pt_swz(row, 4 * jc)) = l;
}
__device__ __forceinline__ float comp(const float4& v, int d) { return d == 0 ? v.x : d == 1 ? v.y : d == 2 ? v.z : v.w; }
__device__ __forceinline__ void setc(float4& v, int d, float x) {
    if (d == 0) v.x = x; else if (d == 1) v.y = x; else if (d == 2) v.z = x; else v.w = x;
}

// The ring fields a builder needs, read once per work item.
struct RingIn {
    int64_t off_n, off_s, gofs;
    int n, mt;
    float domega, coslat_inv;
};

// Analysis, four columns at once: layer k, i0 .. i0 + 3 (nb is a multiple of 4 on these
// grids), q = q0 .. q0 + 3; 16-byte loads of the northern and southern rings.
__device__ __forceinline__ void build_ana4(const PtArgs& a, const RingIn& ri, int p, int h, int nb, int k, int i0,
                                           int q0, int mat, float* hi, float* lo, int row0, int jc) {
    const float* gn = a.grid + (int64_t)k * a.ldg + ri.off_n + i0;
    const float* gs = a.grid + (int64_t)k * a.ldg + ri.off_s + i0;
    float4 nq[4], sq[4], nm[4], sm[4];
    const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int q = q0 + e;
        const bool in = q <= h, pair = in && q > 0;
        nq[e] = in ? __ldg(reinterpret_cast<const float4*>(gn + q * nb)) : z4;
        sq[e] = in ? __ldg(reinterpret_cast<const float4*>(gs + q * nb)) : z4;
        nm[e] = pair ? __ldg(reinterpret_cast<const float4*>(gn + (p - q) * nb)) : z4;
        sm[e] = pair ? __ldg(reinterpret_cast<const float4*>(gs + (p - q) * nb)) : z4;
    }
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        float4 re, im;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const bool zero = mat == 1 && q0 + e == 0;             // v_0 = 0
            setc(re, e, zero ? 0.f : mat == 0 ? comp(nq[e], d) + comp(nm[e], d) : comp(nq[e], d) - comp(nm[e], d));
            setc(im, e, zero ? 0.f : mat == 0 ? comp(sq[e], d) + comp(sm[e], d) : comp(sq[e], d) - comp(sm[e], d));
        }
        put_row(hi, lo, row0 + 2 * d, jc, re);
        put_row(hi, lo, row0 + 2 * d + 1, jc, im);
    }
}

// Synthesis input z_t of layers k .. k + 3 (K a multiple of 4): the packed spectrum the FFT
// kernel's prologue builds, from 16-byte loads of the scratch rows.
__device__ __forceinline__ void syn_in4(const PtArgs& a, const RingIn& ri, int k, int t, float4& re, float4& im) {
    const int m = 2 * t <= ri.n ? t : ri.n - t;
    re = im = make_float4(0.f, 0.f, 0.f, 0.f);
    if (m > ri.mt) return;
    const float2* er = a.four + (ri.gofs + m) * 2 * a.K + k;
    const float2* orw = er + a.K;
    const float4 e01 = __ldg(reinterpret_cast<const float4*>(er)), e23 = __ldg(reinterpret_cast<const float4*>(er + 2));
    const float4 o01 = __ldg(reinterpret_cast<const float4*>(orw)), o23 = __ldg(reinterpret_cast<const float4*>(orw + 2));
    const float scale = !a.adjoint ? (a.unscale ? ri.coslat_inv : 1.f)
                                   : ((m == 0 || 2 * m == ri.n) ? ri.domega : 0.5f * ri.domega);
    const float2 ev[4] = {make_float2(e01.x, e01.y), make_float2(e01.z, e01.w), make_float2(e23.x, e23.y),
                          make_float2(e23.z, e23.w)};
    const float2 ov[4] = {make_float2(o01.x, o01.y), make_float2(o01.z, o01.w), make_float2(o23.x, o23.y),
                          make_float2(o23.z, o23.w)};
    const bool selfconj = m == 0 || 2 * m == ri.n, pos = 2 * t < ri.n;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const float2 gn = make_float2(__fmul_rn(scale, ev[l].x + ov[l].x), __fmul_rn(scale, ev[l].y + ov[l].y));
        const float2 gs = make_float2(__fmul_rn(scale, ev[l].x - ov[l].x), __fmul_rn(scale, ev[l].y - ov[l].y));
        setc(re, l, selfconj ? gn.x : pos ? gn.x - gs.y : gn.x + gs.y);
        setc(im, l, selfconj ? gs.x : pos ? gn.y + gs.x : gs.x - gn.y);
    }
}

// Synthesis, four columns at once: layers k .. k + 3 of column i0, q = q0 .. q0 + 3.
__device__ __forceinline__ void build_syn4(const PtArgs& a, const RingIn& ri, int p, int h, int nb, int k, int i0,
                                           int q0, int mat, float* hi, float* lo, int row0, int jc) {
    float4 re[4], im[4];                           // [layer] over the four q
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int q = q0 + e;
        float4 ar = make_float4(0.f, 0.f, 0.f, 0.f), ai = ar, br = ar, bi = ar;
        if (q <= h) syn_in4(a, ri, k, i0 + q * nb, ar, ai);
        if (q <= h && q > 0) syn_in4(a, ri, k, i0 + (p - q) * nb, br, bi);
        const bool zero = mat == 1 && q == 0;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            setc(re[l], e, zero ? 0.f : mat == 0 ? comp(ar, l) + comp(br, l) : comp(ar, l) - comp(br, l));
            setc(im[l], e, zero ? 0.f : mat == 0 ? comp(ai, l) + comp(bi, l) : comp(ai, l) - comp(bi, l));
        }
    }
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        put_row(hi, lo, row0 + 2 * l, jc, re[l]);
        put_row(hi, lo, row0 + 2 * l + 1, jc, im[l]);
    }
}

// tcgen05.ld of 16 columns without the wait; tmem_wait_ld waits for every load of the warp
// and fences the registers so that no use moves above the wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
template <int N>
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[N]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < N; ++i) asm volatile("" : "+r"(r[i]));
}

template <bool SYN>
__global__ void __launch_bounds__(PT_THREADS, 1) prime_stage_kernel(const PtArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* aslot = smem;
    uint8_t* bslot = smem + PT_A_SLOTS * PT_A_SLOT;
    uint64_t* a_full = reinterpret_cast<uint64_t*>(smem + PT_BAR_OFF);
    uint64_t* a_empty = a_full + PT_A_SLOTS;
    uint64_t* b_full = a_empty + PT_A_SLOTS;
    uint64_t* b_empty = b_full + PT_B_SLOTS;
    uint64_t* acc_full = b_empty + PT_B_SLOTS;
    uint64_t* acc_empty = acc_full + 1;
    uint64_t* fin = acc_empty + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;

    if (threadIdx.x == 0) {
        for (int s = 0; s < PT_A_SLOTS; ++s) {
            mbar_init(&a_full[s], 1);
            mbar_init(&a_empty[s], 1);
        }
        for (int s = 0; s < PT_B_SLOTS; ++s) {
            mbar_init(&b_full[s], PT_GROUP);
            mbar_init(&b_empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, PT_DRAIN);
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
    const int K = a.K;

    if (warp == 0 && lane == 0) {
        // ------------------------------------------------ matrix copies
        int u = 0;
        bool ok = true;
        for (int ix = blockIdx.x; ix < a.nitems && ok && !*abort_flag; ix += gridDim.x) {
            const int2 it = a.items[ix];
            const PrimeRing pr = a.prs[it.x];
            if (it.y * (pr.nc / 2) >= pr.nb * K) continue;
            const uint32_t bytes = (uint32_t)(pr.mtiles * 2 * PT_TILE);
            for (int kb = 0; kb < pr.kb && ok; ++kb)
                for (int mat = 0; mat < 2; ++mat, ++u) {
                    const int s = u % PT_A_SLOTS;
                    if (u >= PT_A_SLOTS && !mbar_wait(&a_empty[s], ((u / PT_A_SLOTS) - 1) & 1)) {
                        *abort_flag = 1;
                        atomicExch(a.err, 31);
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&a_full[s], bytes);
                    bulk_load(aslot + (size_t)s * PT_A_SLOT,
                              a.mat + pr.mofs + (int64_t)(kb * 2 + mat) * pr.mtiles * 2 * (PT_TILE / 4), bytes,
                              &a_full[s]);
                }
        }
        // no copy may still be landing in shared memory when the CTA exits
        for (int v = u - 1; v >= 0 && v >= u - PT_A_SLOTS; --v)
            if (!mbar_wait(&a_full[v % PT_A_SLOTS], (v / PT_A_SLOTS) & 1)) atomicExch(a.err, 35);
    } else if (warp == 1 && lane == 0) {
        // ------------------------------------------------ MMAs
        int u = 0, it_no = 0;
        bool ok = true;
        for (int ix = blockIdx.x; ix < a.nitems && ok && !*abort_flag; ix += gridDim.x) {
            const int2 it = a.items[ix];
            const PrimeRing pr = a.prs[it.x];
            if (it.y * (pr.nc / 2) >= pr.nb * K) continue;
            if (it_no > 0 && !mbar_wait(acc_empty, (it_no - 1) & 1)) {
                *abort_flag = 1;
                atomicExch(a.err, 32);
                break;
            }
            tc_fence_after();
            const uint32_t nc = (uint32_t)pr.nc;
            const uint32_t id2 = idesc_f16(2u, 0u, 0u, 2 * nc);   // M_hi x [D_hi; D_lo]
            const uint32_t id1 = idesc_f16(2u, 0u, 0u, nc);       // M_lo x D_hi
            for (int kb = 0; kb < pr.kb && ok; ++kb) {
                const int nks = min(4, (pr.h + 1 - 32 * kb + 7) / 8);
                for (int mat = 0; mat < 2; ++mat, ++u) {
                    const int sa = u % PT_A_SLOTS, sb = u % PT_B_SLOTS;
                    if (!mbar_wait(&a_full[sa], (u / PT_A_SLOTS) & 1) || !mbar_wait(&b_full[sb], (u / PT_B_SLOTS) & 1)) {
                        *abort_flag = 1;
                        atomicExch(a.err, 33);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t ab = smem_u32(aslot + (size_t)sa * PT_A_SLOT);
                    const uint32_t bb = smem_u32(bslot + (size_t)sb * PT_B_SLOT);
                    for (int mt = 0; mt < pr.mtiles; ++mt) {
                        const uint32_t d = tmem + (uint32_t)(mt * 2 + mat) * 2 * nc;
                        const uint32_t mhi = ab + (uint32_t)(mt * 2) * PT_TILE, mlo = mhi + PT_TILE;
                        for (int kk = 0; kk < nks; ++kk) {
                            const uint64_t db = sdesc(bb + kk * 32, 16, 1024);
                            umma_tf32(d, sdesc(mhi + kk * 32, 16, 1024), db, id2, (kb == 0 && kk == 0) ? 0u : 1u);
                            umma_tf32(d + nc, sdesc(mlo + kk * 32, 16, 1024), db, id1, 1u);
                        }
                    }
                    umma_commit(&a_empty[sa]);
                    umma_commit(&b_empty[sb]);
                }
            }
            if (!ok) break;
            umma_commit(acc_full);
            ++it_no;
        }
        // every MMA must be complete before the tensor memory is released
        umma_commit(fin);
        if (!mbar_wait(fin, 0)) atomicExch(a.err, 36);
    } else if (warp >= 2 && warp < 2 + PT_BUILDERS) {
        // ------------------------------------------------ data pieces
        // two groups of four warps take alternate units, so that one group's loads are in
        // flight while the other's are consumed
        const int grp = (warp - 2) / PT_GROUP;
        const int tb = threadIdx.x - 64 - grp * 32 * PT_GROUP;
        const bool avec = ((a.ldg & 3) == 0) && ((reinterpret_cast<uintptr_t>(a.grid) & 15) == 0);
        const bool svec = (K & 3) == 0 && ((reinterpret_cast<uintptr_t>(a.four) & 15) == 0);
        int u = 0;
        bool ok = true;
        for (int ix = blockIdx.x; ix < a.nitems && ok; ix += gridDim.x) {
            const int2 it = a.items[ix];
            const PrimeRing pr = a.prs[it.x];
            const int cpi = pr.nc / 2;                  // complex columns per item
            const int ncols = pr.nb * K;
            if (it.y * cpi >= ncols) continue;
            const RingDesc& rd = a.rings[pr.ring];
            RingIn ri;
            ri.off_n = rd.off_north;
            ri.off_s = rd.off_south;
            ri.gofs = rd.gofs;
            ri.n = rd.n;
            ri.mt = rd.mt;
            ri.domega = rd.domega;
            ri.coslat_inv = rd.coslat_inv;
            const int p = pr.p, h = pr.h, nb = pr.nb;
            const int c0 = it.y * cpi;
            // four columns per task: analysis (ring offsets multiples of 4 points) or synthesis
            const bool vec = (nb & 3) == 0 && (SYN ? svec : (avec && ((ri.off_n | ri.off_s) & 3) == 0));
            for (int kb = 0; kb < pr.kb && ok; ++kb)
                for (int mat = 0; mat < 2; ++mat, ++u) {
                    if ((u & 1) != grp) continue;
                    const int sb = u % PT_B_SLOTS;
                    const bool got = u < PT_B_SLOTS ||
                                     __all_sync(0xffffffffu, mbar_wait(&b_empty[sb], ((u / PT_B_SLOTS) - 1) & 1));
                    if (!got || *abort_flag) {
                        *abort_flag = 1;
                        if (!got) atomicExch(a.err, 34);
                        ok = false;
                        break;
                    }
                    float* hi = reinterpret_cast<float*>(bslot + (size_t)sb * PT_B_SLOT);
                    float* lo = hi + pr.nc * 32;        // the lo rows follow the nc hi rows
                    if (vec) {
                        // task: (four complex columns g, 4-deep chunk jc of the k-block)
                        for (int w = tb; w < (cpi / 4) * 8; w += 32 * PT_GROUP) {
                            const int g = w % (cpi / 4), jc = w / (cpi / 4);
                            const int c = c0 + 4 * g;
                            if (c >= ncols) {
#pragma unroll
                                for (int d = 0; d < 8; ++d) put_row(hi, lo, 8 * g + d, jc, make_float4(0.f, 0.f, 0.f, 0.f));
                                continue;
                            }
                            int k, i0;
                            col_of<SYN>(c, nb, K, k, i0);
                            if (SYN)
                                build_syn4(a, ri, p, h, nb, k, i0, 32 * kb + 4 * jc, mat, hi, lo, 8 * g, jc);
                            else
                                build_ana4(a, ri, p, h, nb, k, i0, 32 * kb + 4 * jc, mat, hi, lo, 8 * g, jc);
                        }
                    } else {
                        // task: (complex column cl, 4-deep chunk jc of the k-block)
                        for (int w = tb; w < cpi * 8; w += 32 * PT_GROUP) {
                            const int cl = w % cpi, jc = w / cpi;
                            const int c = c0 + cl;
                            float4 re = make_float4(0.f, 0.f, 0.f, 0.f), im = re;
                            if (c < ncols) {
                                int k, i0;
                                col_of<SYN>(c, nb, K, k, i0);
#pragma unroll
                                for (int e = 0; e < 4; ++e) {
                                    const int q = 32 * kb + 4 * jc + e;
                                    if (q == 0) {
                                        if (mat == 0) {
                                            const float2 x0 = stage_input<SYN>(a, rd, k, i0);
                                            setc(re, e, x0.x);
                                            setc(im, e, x0.y);
                                        }
                                    } else if (q <= h) {
                                        const float2 xa = stage_input<SYN>(a, rd, k, i0 + q * nb);
                                        const float2 xb = stage_input<SYN>(a, rd, k, i0 + (p - q) * nb);
                                        setc(re, e, mat == 0 ? xa.x + xb.x : xa.x - xb.x);
                                        setc(im, e, mat == 0 ? xa.y + xb.y : xa.y - xb.y);
                                    }
                                }
                            }
                            // rows 2 cl (real parts) and 2 cl + 1 (imaginary parts)
                            put_row(hi, lo, 2 * cl, jc, re);
                            put_row(hi, lo, 2 * cl + 1, jc, im);
                        }
                    }
                    fence_proxy_async();           // the MMA reads these through the async proxy
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&b_full[sb]);
                }
        }
    } else if (warp >= 2 + PT_BUILDERS) {
        // ------------------------------------------------ drain and store y
        const int quarter = warp % 4;
        const int half = (warp - 2 - PT_BUILDERS) / 4;       // this warp's 16-column chunks: half, half + 2, ...
        const uint32_t lane_off = (uint32_t)(quarter * 32) << 16;
        int it_no = 0;
        for (int ix = blockIdx.x; ix < a.nitems; ix += gridDim.x) {
            const int2 it = a.items[ix];
            const PrimeRing pr = a.prs[it.x];
            const int cpi = pr.nc / 2;
            const int ncols = pr.nb * K;
            if (it.y * cpi >= ncols) continue;
            // warp-uniform outcome: tcgen05.ld below is a warp-collective instruction
            if (*abort_flag || !__all_sync(0xffffffffu, mbar_wait(acc_full, it_no & 1))) {
                *abort_flag = 1;
                atomicExch(a.err, 37);
                break;
            }
            tc_fence_after();
            const RingDesc& rd = a.rings[pr.ring];
            const int n = rd.n, p = pr.p, h = pr.h, nb = pr.nb, nc = pr.nc;
            float2* ybase = a.ymid + rd.yofs;
            for (int mt = 0; mt < pr.mtiles; ++mt) {
                const int r = mt * 128 + quarter * 32 + lane;
                const uint32_t tc = tmem + lane_off + (uint32_t)(mt * 2) * 2 * nc;   // cosine set; sine 2 nc on
                for (int ch = half; ch < nc / 16; ch += 2) {
                    uint32_t v[64];     // cosine lead, cosine cross, sine lead, sine cross: 16 columns each
                    tmem_ld16(tc + ch * 16, *reinterpret_cast<uint32_t(*)[16]>(v));
                    tmem_ld16(tc + nc + ch * 16, *reinterpret_cast<uint32_t(*)[16]>(v + 16));
                    tmem_ld16(tc + 2 * nc + ch * 16, *reinterpret_cast<uint32_t(*)[16]>(v + 32));
                    tmem_ld16(tc + 3 * nc + ch * 16, *reinterpret_cast<uint32_t(*)[16]>(v + 48));
                    tmem_wait_ld(v);
                    if (r > h) continue;
#pragma unroll
                    for (int e = 0; e < 8; ++e) {
                        const int c = it.y * cpi + ch * 8 + e;
                        if (c >= ncols) continue;
                        int k, i0;
                        col_of<SYN>(c, nb, K, k, i0);
                        const float2 A = make_float2(__fadd_rn(__uint_as_float(v[2 * e]), __uint_as_float(v[16 + 2 * e])),
                                                     __fadd_rn(__uint_as_float(v[2 * e + 1]), __uint_as_float(v[17 + 2 * e])));
                        const float2 B = make_float2(__fadd_rn(__uint_as_float(v[32 + 2 * e]), __uint_as_float(v[48 + 2 * e])),
                                                     __fadd_rn(__uint_as_float(v[33 + 2 * e]), __uint_as_float(v[49 + 2 * e])));
                        float2* yo = ybase + (int64_t)k * n + i0 * p;
                        if (!SYN) {
                            yo[r] = make_float2(A.x + B.y, A.y - B.x);
                            if (r > 0) yo[p - r] = make_float2(A.x - B.y, A.y + B.x);
                        } else {
                            yo[r] = make_float2(A.x - B.y, A.y + B.x);
                            if (r > 0) yo[p - r] = make_float2(A.x + B.y, A.y - B.x);
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty);
            ++it_no;
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

struct PrimeState {
    PrimeRing* d_prs = nullptr;
    int2* d_items = nullptr;
    int nitems = 0;
    float* d_mat = nullptr;
    float2* d_ymid = nullptr;
    int64_t ymid_elems = 0;
    int nsm = 148;
};

bool eligible(const RingDesc& r) {
    if (r.nfac <= 0 || r.fac[0] < kPrimeTcMin) return false;
    const int h = (r.fac[0] - 1) / 2;
    return h + 1 <= 256;   // at most two 128-row tiles
}

}  // namespace

int64_t prime_mark_rings(std::vector<RingDesc>& rings, int nlayers) {
    int64_t off = 0;
    for (RingDesc& r : rings) {
        r.pre = eligible(r) ? 1 : 0;
        r.yofs = off;
        if (r.pre) off += (int64_t)r.n * std::max(1, nlayers);
    }
    return off;
}

cudaError_t prime_create(Plan& p, int64_t ymid_elems) {
    if (ymid_elems == 0) return cudaSuccess;
    PrimeState* st = new PrimeState();
    st->ymid_elems = ymid_elems;
    p.prime = st;               // the tables are built when the mode is first turned on
    return cudaSuccess;
}

namespace {
// Stage matrices, ring descriptors and the work list, on the device.
cudaError_t prime_build(Plan& p, PrimeState* st) {
    std::vector<PrimeRing> prs;
    std::vector<float> mat;
    std::map<int, int64_t> mofs;
    std::vector<std::pair<int64_t, int2>> items;
    const int nl = std::max(1, p.d.nlayers);
    for (int j = 0; j < (int)p.h_rings.size(); ++j) {
        const RingDesc& r = p.h_rings[j];
        if (!r.pre) continue;
        PrimeRing pr{};
        pr.ring = j;
        pr.p = r.fac[0];
        pr.h = (pr.p - 1) / 2;
        pr.nb = r.n / pr.p;
        pr.kb = (pr.h + 1 + 31) / 32;
        pr.mtiles = (pr.h + 1 + 127) / 128;
        pr.nc = pr.mtiles == 1 ? 128 : 64;
        auto f = mofs.find(pr.p);
        if (f == mofs.end()) {
            // tiles [k-block][matrix][row tile][piece][128][32], swizzled; entries
            // cos / sin(2 pi r q / p) for r, q <= h, zero beyond
            const int64_t base = (int64_t)mat.size();
            mat.resize(mat.size() + (size_t)pr.kb * 2 * pr.mtiles * 2 * (PT_TILE / 4), 0.f);
            for (int kb = 0; kb < pr.kb; ++kb)
                for (int m2 = 0; m2 < 2; ++m2)
                    for (int mt = 0; mt < pr.mtiles; ++mt) {
                        float* thi = mat.data() + base + ((int64_t)((kb * 2 + m2) * pr.mtiles + mt) * 2) * (PT_TILE / 4);
                        float* tlo = thi + PT_TILE / 4;
                        for (int row = 0; row < 128; ++row)
                            for (int col = 0; col < 32; ++col) {
                                const int rr = mt * 128 + row, q = kb * 32 + col;
                                if (rr > pr.h || q > pr.h) continue;
                                const double ang = 2.0 * M_PI * (double)(((int64_t)rr * q) % pr.p) / pr.p;
                                const double v = m2 == 0 ? std::cos(ang) : std::sin(ang);
                                float vf = (float)v;
                                uint32_t b;
                                std::memcpy(&b, &vf, 4);
                                b = tf32_bits(b);
                                float hv;
                                std::memcpy(&hv, &b, 4);
                                float lv = (float)(v - (double)hv);
                                std::memcpy(&b, &lv, 4);
                                b = tf32_bits(b);
                                std::memcpy(&lv, &b, 4);
                                thi[pt_swz(row, col)] = hv;
                                tlo[pt_swz(row, col)] = lv;
                            }
                    }
            f = mofs.emplace(pr.p, base).first;
        }
        pr.mofs = f->second;
        const int tiles = (pr.nb * nl + pr.nc / 2 - 1) / (pr.nc / 2);
        for (int t = 0; t < tiles; ++t)
            items.push_back({(int64_t)pr.kb * pr.mtiles * 2 * (pr.nc == 128 ? 2 : 1), make_int2((int)prs.size(), t)});
        prs.push_back(pr);
    }
    std::stable_sort(items.begin(), items.end(),
                     [](const std::pair<int64_t, int2>& x, const std::pair<int64_t, int2>& y) { return x.first > y.first; });
    std::vector<int2> it;
    for (auto& x : items) it.push_back(x.second);
    st->nitems = (int)it.size();
    cudaError_t e = cudaSuccess;
    auto up = [&](void** dst, const void* src, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(dst, std::max<size_t>(bytes, 16));
        if (e == cudaSuccess && bytes) e = cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice);
    };
    up((void**)&st->d_prs, prs.data(), prs.size() * sizeof(PrimeRing));
    up((void**)&st->d_items, it.data(), it.size() * sizeof(int2));
    up((void**)&st->d_mat, mat.data(), mat.size() * sizeof(float));
    int dev = 0;
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&st->nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(prime_stage_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, PT_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(prime_stage_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, PT_SMEM);
    if (e == cudaSuccess) {
        p.table_bytes += (int64_t)(mat.size() * sizeof(float) + prs.size() * sizeof(PrimeRing));
    } else {           // leave nothing half-built: a later call starts over
        for (void** q : {(void**)&st->d_prs, (void**)&st->d_items, (void**)&st->d_mat}) {
            if (*q) cudaFree(*q);
            *q = nullptr;
        }
        st->nitems = 0;
    }
    return e;
}
}  // namespace

void prime_release(Plan& p) {
    PrimeState* st = static_cast<PrimeState*>(p.prime);
    if (!st) return;
    void* ptrs[] = {st->d_prs, st->d_items, st->d_mat, st->d_ymid};
    for (void* q : ptrs)
        if (q) cudaFree(q);
    delete st;
    p.prime = nullptr;
    p.prime_mode = 0;
}

bool prime_available(const Plan& p) { return p.prime != nullptr; }

cudaError_t prime_set_mode(Plan& p, int mode) {
    PrimeState* st = static_cast<PrimeState*>(p.prime);
    if (!st) {
        p.prime_mode = 0;
        return cudaSuccess;
    }
    if (mode && !st->d_mat) {
        const cudaError_t e = prime_build(p, st);
        if (e != cudaSuccess) return e;
    }
    if (mode && !st->d_ymid) {
        const cudaError_t e = cudaMalloc((void**)&st->d_ymid, st->ymid_elems * sizeof(float2));
        if (e != cudaSuccess) return e;
    }
    p.prime_mode = mode ? 1 : 0;
    return cudaSuccess;
}

float2* prime_buffer(const Plan& p) {
    const PrimeState* st = static_cast<const PrimeState*>(p.prime);
    return (st && p.prime_mode) ? st->d_ymid : nullptr;
}

cudaError_t launch_prime_stage(const Plan& p, bool synthesis, const float* grid, int64_t ldg, int K, unsigned flags,
                               bool adjoint, cudaStream_t s) {
    const PrimeState* st = static_cast<const PrimeState*>(p.prime);
    if (!st || !p.prime_mode || st->nitems == 0 || K <= 0) return cudaSuccess;
    PtArgs a{};
    a.rings = p.d_rings;
    a.prs = st->d_prs;
    a.items = st->d_items;
    a.nitems = st->nitems;
    a.mat = st->d_mat;
    a.grid = grid;
    a.ldg = ldg;
    a.four = p.d_four;
    a.ymid = st->d_ymid;
    a.K = K;
    a.unscale = (flags & SHT_UNSCALE_COSLAT) ? 1 : 0;
    a.adjoint = adjoint ? 1 : 0;
    a.err = p.d_err;
    const int g = std::max(1, std::min(st->nitems, st->nsm));
    if (synthesis)
        prime_stage_kernel<true><<<g, PT_THREADS, PT_SMEM, s>>>(a);
    else
        prime_stage_kernel<false><<<g, PT_THREADS, PT_SMEM, s>>>(a);
    return cudaGetLastError();
}

}  // namespace sht
