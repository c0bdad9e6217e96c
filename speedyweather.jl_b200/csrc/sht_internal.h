// Internal declarations of libsht: the plan object, its device tables and the
// kernel launchers. Not part of the C ABI (include/sht.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/sht.h"

namespace sht {

constexpr int kMaxFactors = 24;      // radices per ring FFT (n <= 2^24)
#ifndef SHT_PRIME_GROUP
#define SHT_PRIME_GROUP 8
#endif
constexpr int kPrimeGroup = SHT_PRIME_GROUP;   // outputs per thread of a prime FFT stage

// Launch shape of the FFT kernels: threads per CTA, CTAs per SM, and the shared
// memory one CTA may use (which bounds the layers per CTA).
#ifndef SHT_FFT_THREADS
#define SHT_FFT_THREADS 384        // 2 x 12 warps per SM in 80 registers (256: 119 registers, 16 warps)
#endif
#ifndef SHT_FFT_CTAS_PER_SM
#define SHT_FFT_CTAS_PER_SM 2
#endif
constexpr int kFftThreads = SHT_FFT_THREADS;
constexpr int kFftGroupThreads = 256;   // grouped (batch) launches: their item loop needs more registers
constexpr int kFftCtasPerSm = SHT_FFT_CTAS_PER_SM;
constexpr int kFftSmemBudget = (227 * 1024) / SHT_FFT_CTAS_PER_SM - 1024;

// Per-ring real-FFT description, indexed by the northern ring j (0-based).
// The southern mirror ring has the same length.
struct RingDesc {
    int32_t n;            // points on the ring
    int32_t mt;           // mmax_truncation (0-based highest order kept)
    int32_t nfac;         // number of Stockham stages
    int32_t chunk;        // layers per CTA in the FFT kernels
    int32_t gen_len;      // float2 entries of the prime-stage tables after the twiddles (even)
    int32_t ldx;          // layer stride of the FFT's shared-memory buffers (>= n, even)
    int64_t off_north;    // first grid point of the northern ring
    int64_t off_south;    // first grid point of the southern ring
    int64_t gofs;         // first Fourier-scratch row (m = 0) of this ring
    int64_t tw_off;       // offset of this ring's twiddles ((n + 1) & ~1 entries) and prime tables
    float domega;         // solid angle w_j 2pi / n_j
    float coslat_inv;     // 1 / cos(latitude)
    int32_t pre;          // 1: the first stage (a large prime radix) may run on the tensor cores
    int32_t spare;
    int64_t yofs;         // float2 offset of this ring's first-stage output [k][n] in the prime buffer
    int32_t fac[kMaxFactors];
};

// One tile of the Legendre contraction of order m.
struct LegItem {
    int32_t m;
    int32_t tile;         // ring tile (synthesis) or parity-row tile (analysis)
};

// The operands of one transform's FP32 Legendre stage (plan tables, data pointers).
struct LegView {
    const float* lam;
    const int64_t* lam_off;
    const int32_t* rows;
    const int32_t* j0;
    const int64_t* lm_off;
    const RingDesc* rings;
    const int64_t* gofs;  // per ring: first Fourier-scratch row (m = 0)
    int nh, nh_pad, lmax;
    const float2* cin;    // synthesis input coefficients
    float2* cout;         // analysis output coefficients
    int64_t ldc;
    float2* four;         // Fourier scratch
    int K, add;
};

// One work item of a grouped (batched) launch over several transforms.
struct GroupItem {
    int32_t task;         // index into the batch's per-transform argument array
    int32_t a, b, c;      // Legendre: m, tile, column tile * 2 + parity; FFT: ring, chunk, -
};

// Layout of the analysis data operand the FFT writes for the tensor-core Legendre
// stage: pre-swizzled (SWIZZLE_128B, MN-major) 16-bit tiles of 64 rings x N columns,
// one tile per (order m, parity, ring block, piece).
struct TcImage {
    uint16_t* base = nullptr;           // 16-bit words (bf16 or fp16 bits)
    const int64_t* tile_base = nullptr; // per m: tile index of (m, parity 0, ring block 0)
    const int32_t* njt = nullptr;       // per m: ring blocks of 64 rings
    const int32_t* j0 = nullptr;        // per m: first ring
    int32_t npieces = 0;
    int32_t tile_bytes = 0;             // bytes of one tile
    int32_t fp16 = 0;                   // 0: bf16 pieces, 1: fp16 pieces
    const float2* kscale = nullptr;     // fp16: per layer (2^(e_k - 15), 2^(15 - e_k)) data scale
};

// The operands of one transform's FFT stage.
struct FftView {
    const RingDesc* rings;
    const float2* twiddle;
    const float* gin;     // analysis input grid
    float* gout;          // synthesis output grid
    int64_t ldg;
    float2* four;         // Fourier scratch
    int K, unscale, add;
    int adjoint;          // 1: the adjoint weights (of the synthesis for the analysis direction and v.v.)
    TcImage img;          // analysis operand image of tensor-core plans (base == nullptr: FP32 scratch)
    float2* ymid;         // first-stage output of the rings with pre = 1 (nullptr: every stage in the FFT kernel)
};

// The operands of a fused (FFT + Legendre in one launch) transform of an FP32 plan:
// a cluster of P CTAs per chunk of C layers (sht_fft.cu).
struct FusedView {
    const RingDesc* rings;
    const float2* twiddle;
    const float* lam;
    const int64_t* lam_off;
    const int32_t* rows;
    const int32_t* j0;
    const int64_t* lm_off;
    int nh, nh_pad, lmax, mmax, mt_max;
    const float2* cin;    // synthesis input coefficients
    float2* cout;         // analysis output coefficients
    int64_t ldc;
    const float* gin;     // analysis input grid
    float* gout;          // synthesis output grid
    int64_t ldg;
    int K, C, P;          // layers, layers per cluster, CTAs per cluster
    int nm_cta, nr_cta;   // orders and rings per CTA: ceil(mmax / P), ceil(nh / P)
    int ldx, tw_max;      // layer stride of the FFT buffers, float2 of the largest ring's tables
    int unscale, add;
    int uniform;          // all rings of one length: a CTA transforms its rings in one FFT
};

struct Plan {
    sht_desc d{};
    int nh = 0, nlat = 0, lmax = 0, mmax = 0, nlon_max = 0, nfreq_max = 0;
    float coslat_inv_max = 1.f;         // max over rings of 1 / cos(latitude)
    int64_t npoints = 0, nlm = 0;
    int64_t scratch_rows = 0;           // sum_j (mt_j + 1)
    int device = 0;

    // host copies (FP64 where computed so)
    std::vector<double> latd, weights;  // nlat
    std::vector<int32_t> nlons;         // nlat
    std::vector<int32_t> mt;            // nh
    std::vector<int32_t> j0;            // per m: first northern ring with mt >= m (nh if none)
    std::vector<int64_t> lm_off;        // per m: packed offset of (l = m, m)
    std::vector<int32_t> rows;          // per m: parity rows ceil((lmax - m) / 2)
    std::vector<int64_t> lam_off;       // per m: offset into the FP32 Legendre table
    int nh_pad = 0;

    // device tables
    RingDesc* d_rings = nullptr;
    float2* d_twiddle = nullptr;
    float* d_lam = nullptr;             // [m][parity][row][nh_pad], FP32
    int64_t* d_lam_off = nullptr;
    int32_t* d_j0 = nullptr;
    int32_t* d_rows = nullptr;
    int64_t* d_lm_off = nullptr;
    LegItem* d_syn_items = nullptr;  int n_syn_items = 0;
    LegItem* d_ana_items = nullptr;  int n_ana_items = 0;
    int32_t* d_mt = nullptr;
    int64_t* d_gofs = nullptr;

    // spectral operator factors, per packed lm (FP32, computed in FP64)
    float* d_grad = nullptr;            // 8 arrays of nlm: see GradIdx
    int32_t* d_l_of = nullptr;          // 0-based degree of each lm
    int32_t* d_m_of = nullptr;          // 0-based order of each lm
    float* d_eig = nullptr;             // lmax: -l(l+1)
    float* d_eig_inv = nullptr;         // lmax: 1/(-l(l+1)), 0 at l = 0

    // scratch: Fourier coefficients, [row = gofs_j + m][eo][k] complex FP32
    float2* d_four = nullptr;
    int64_t four_elems = 0;

    int64_t table_bytes = 0;
    int32_t* d_err = nullptr;           // device status word of the bounded waits (0 = ok)
    void* tc = nullptr;                 // tensor-core Legendre state (sht_legendre_tc.cu)
    void* prime = nullptr;              // tensor-core prime stages of the ring FFTs (sht_prime_tc.cu)
    int prime_mode = 0;                 // 1: the FFT launches run those stages on the tensor cores
    TcImage ana_img;                    // analysis data image written by the FFT (tensor-core plans)
    int smem_fft = 0;                   // dynamic shared memory of the FFT kernels
    int min_chunk = 1;
    int2* d_fft_items = nullptr;        // FFT work list: (ring, layer chunk), costliest first
    int n_fft_items = 0;
    int leg_bn_syn = 128, leg_bn_ana = 128;   // FP32 Legendre tile widths (autotuned)
    // fused transforms (FP32 plans whose cluster data fits in shared memory)
    int fusion = 0;                     // 1: sht_synthesize / sht_analyze launch the fused kernels
    int fusion_ok = 0;                  // the fused kernels can run this plan
    int fused_P = 0, fused_cmax = 0, fused_ldx = 0, fused_tw_max = 0, fused_mt_max = 0, nsm = 148;
    int fused_ncl = 1;                  // clusters of fused_P CTAs the device runs at once
    int fused_uniform = 0;              // all rings of one length (full grids)
    // host copies for batches (grouped launches over several plans)
    std::vector<RingDesc> h_rings;
    std::vector<double> h_ring_cost;     // per ring: estimated FFT cost per layer
    std::vector<LegItem> h_syn_items, h_ana_items;
};

enum GradIdx {
    G_GRAD_Y1 = 0, G_GRAD_Y2, G_GRAD_Y_VORDIV1, G_GRAD_Y_VORDIV2, G_GRAD_X_VORDIV,
    G_VORDIV_TO_UV_X, G_VORDIV_TO_UV1, G_VORDIV_TO_UV2, G_COUNT
};

// ---- launchers (return cudaError_t of the launch) ----------------------------------
FftView fft_view(const Plan& p, const float* gin, float* gout, int64_t ldg, float2* four, int K, unsigned flags,
                 bool image, bool adjoint);
cudaError_t launch_fft_grouped(const FftView* views, const GroupItem* items, int nitems, bool synthesis, int smem,
                               int grid, cudaStream_t s);
// dense matrix transforms on the tensor cores (sht_legendre_tc.cu)
struct TcMatrix;
cudaError_t tc_matrix_create(TcMatrix** out, int precision, const float* const a[2], const int depth[2],
                             const int M[2], int nlayers);
void tc_matrix_destroy(TcMatrix* x);
cudaError_t tc_matrix_apply(const TcMatrix* x, int which, const float* in, int64_t ld, float* out, int64_t ldo, int K,
                            const float* row_scale, int32_t* d_err, cudaStream_t st);
// FP32 dense matrix transforms as three TF32 products on the tensor cores (sht_matrix_tf32.cu)
struct MxTf32;
cudaError_t mx_tf32_create(MxTf32** out, const float* const a[2], const int depth[2], const int M[2], int nlayers);
void mx_tf32_destroy(MxTf32* x);
cudaError_t mx_tf32_apply(const MxTf32* x, int which, const float* in, int64_t ld, float* out, int64_t ldo, int K,
                          const float* row_scale, int32_t* d_err, cudaStream_t st);
// failure-detection check of the bounded mbarrier waits (sht_legendre_tc.cu)
cudaError_t launch_wait_probe(int32_t* err, uint64_t limit_ns, cudaStream_t s);
cudaError_t launch_column_physics(const float* temp, const float* humid, const float* ps, int64_t ld, int ncol,
                                  float dt, float* dtemp, float* dhumid, int64_t ldo, bool add, cudaStream_t s);
cudaError_t tc_analysis_scale(const Plan& p, const float* grid, int64_t ldg, int K, cudaStream_t s, float mul);
int tc_tile_cols(const Plan& p);                 // tensor-core plans: GEMM column tile width
bool tc_set_tile_cols(Plan& p, int cols);        // 64 or 128; false for other widths or FP32 plans
cudaError_t launch_fft_analysis(const Plan& p, const float* grid, int64_t ldg, int K, cudaStream_t s,
                                bool to_image = false, unsigned flags = 0, bool adjoint = false);
cudaError_t launch_fft_synthesis(const Plan& p, float* grid, int64_t ldg, int K, unsigned flags,
                                 cudaStream_t s, bool adjoint = false);
LegView leg_view(const Plan& p, const float2* cin, float2* cout, int64_t ldc, const float2* four, int K, bool add);
cudaError_t legendre_grouped_grids(int nsm, int (&grid)[3]);
cudaError_t launch_legendre_grouped(const LegView* views, const GroupItem* items, int nitems, int bn, bool synthesis,
                                    int grid, cudaStream_t s);
cudaError_t launch_legendre_analysis_fp32_from(const Plan& p, const float2* scratch, float2* coeffs, int64_t ldc,
                                               int K, bool add, cudaStream_t s);
cudaError_t launch_legendre_synthesis_fp32(const Plan& p, const float2* coeffs, int64_t ldc, int K,
                                           cudaStream_t s);
cudaError_t launch_legendre_analysis_fp32(const Plan& p, float2* coeffs, int64_t ldc, int K, bool add,
                                          cudaStream_t s);
cudaError_t launch_divcurl(const Plan& p, float2* out, const float2* u, const float2* v, int64_t ldc,
                           int K, bool curl, bool flipsign, bool add, float inv_radius, cudaStream_t s);
cudaError_t launch_uv_from_vordiv(const Plan& p, float2* U, float2* V, const float2* vor,
                                  const float2* div, int64_t ldc, int K, float radius, cudaStream_t s);
cudaError_t launch_laplace(const Plan& p, float2* out, const float2* in, int64_t ldc, int K,
                           bool inverse, bool flipsign, bool add, float scale, cudaStream_t s);
cudaError_t launch_operators(const Plan& p, const sht_op* ops, int nops, cudaStream_t s);
// fused transforms (sht_fft.cu): fused_prepare sets fusion_ok and the launch shape
cudaError_t fused_prepare(Plan& p);
cudaError_t launch_fused_synthesis(const Plan& p, const float2* coeffs, int64_t ldc, float* grid, int64_t ldg, int K,
                                   unsigned flags, cudaStream_t s);
cudaError_t launch_fused_analysis(const Plan& p, const float* grid, int64_t ldg, float2* coeffs, int64_t ldc, int K,
                                  bool add, cudaStream_t s);
cudaError_t launch_gradient(const Plan& p, float2* dpdx, float2* dpdy, const float2* in, int64_t ldc,
                            int K, float inv_radius, cudaStream_t s);
// tensor-core first stages of the ring FFTs (sht_prime_tc.cu). prime_mark_rings marks the
// rings whose first radix is a prime of at least kPrimeTcMin (RingDesc.pre, yofs) before
// the rings are uploaded and returns the prime buffer's length in float2; prime_create
// records it, and the first prime_set_mode(p, 1) builds the stage matrices, the work list
// and the buffer.
constexpr int kPrimeTcMin = 64;
int64_t prime_mark_rings(std::vector<RingDesc>& rings, int nlayers);
cudaError_t prime_create(Plan& p, int64_t ymid_elems);
void prime_release(Plan& p);
bool prime_available(const Plan& p);
cudaError_t prime_set_mode(Plan& p, int mode);    // 0: FFT kernels only, 1: tensor-core first stages
float2* prime_buffer(const Plan& p);               // the first-stage output when the mode is 1, else nullptr
cudaError_t launch_prime_stage(const Plan& p, bool synthesis, const float* grid, int64_t ldg, int K,
                               unsigned flags, bool adjoint, cudaStream_t s);

// Factor of the Fourier coefficients of order m in the synthesis prologue: 1 / cos(lat)
// or 1 for the transform; for the adjoint of the analysis the solid angle / the rfft
// adjoint scale (SpeedyTransformsEnzymeExt.jl:294-323).
__device__ __forceinline__ float syn_weight(const RingDesc& rd, int m, int adjoint, int unscale) {
    if (!adjoint) return unscale ? rd.coslat_inv : 1.f;
    return (m == 0 || 2 * m == rd.n) ? rd.domega : 0.5f * rd.domega;
}

}  // namespace sht
