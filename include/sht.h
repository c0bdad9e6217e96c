/*
 * sht.h -- C ABI of libsht, a B200 (sm_100a) spherical harmonic transform for
 * SpeedyWeather.jl's SpeedyTransforms.
 *
 * Every entry point takes plain pointers and sizes. Array arguments are
 * caller-owned DEVICE memory in the reference layouts:
 *
 *   grid   : float  field[k * ldg + ij]      ij ring-major (0..360E within a ring,
 *                                             rings north to south), ldg >= npoints
 *            (RingGrids/src/field.jl:1-20, Field{T,N}.data[npoints, k])
 *   coeffs : float2 coeffs[k * ldc + lm]     complex, packed lower triangle,
 *                                             order m outer, degree l inner,
 *                                             ldc >= nlm (interleaved re, im)
 *            (LowerTriangularArrays/src/lower_triangular_array.jl:10-19,
 *             LowerTriangularArrays/src/spectrum.jl:99-131)
 *
 * lmax and mmax are the reference's 1-based sizes (Spectrum(lmax, mmax)).
 * All calls return an int status: SHT_OK, or SHT_EINVAL for sizes that do not
 * match the plan (the reference throws DimensionMismatch,
 * SpeedyTransforms/src/spectral_transform.jl:387-423), SHT_ECUDA for a CUDA
 * error, SHT_ENOMEM when device memory runs out. sht_last_error() gives the
 * message of the last failure on the calling thread.
 *
 * Work is enqueued on the given stream (NULL = legacy default stream) and is
 * asynchronous; no call on the hot path allocates or synchronises.
 */
#ifndef SHT_H
#define SHT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define SHT_API __attribute__((visibility("default")))
#else
#define SHT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SHT_OK 0
#define SHT_EINVAL 1
#define SHT_ECUDA 2
#define SHT_ENOMEM 3
#define SHT_EUNSUPPORTED 4

/* grid kinds (RingGrids/src/grids/full_gaussian.jl, octahedral_gaussian.jl) */
#define SHT_GRID_FULL_GAUSSIAN 0
#define SHT_GRID_OCTAHEDRAL_GAUSSIAN 1

/* Legendre-stage arithmetic */
#define SHT_PREC_FP32 0          /* FP32 CUDA-core FMA, matches the reference's Float32 */
#define SHT_PREC_BF16X3 1        /* tcgen05, split-BF16 hi/lo operands, 3 products, FP32 accumulate */
#define SHT_PREC_FP16X3 2        /* tcgen05, split-FP16 hi/lo, 3 products, FP32 accumulate; Legendre
                                    polynomials scaled by 2^-e per order m, data by 2^-e per order
                                    and layer (synthesis) or per layer (analysis) from the max-abs
                                    of each call's input */
#define SHT_PREC_BF16X5 3        /* tcgen05, Legendre polynomials in 3 bf16 pieces (from FP64), data
                                    in 2, the 5 products above the split residual, FP32 accumulate */

/* Legendre shortcuts (SpeedyTransforms/src/legendre_shortcuts.jl:21-49) */
#define SHT_SHORTCUT_LINEAR 0
#define SHT_SHORTCUT_QUADRATIC 1
#define SHT_SHORTCUT_CUBIC 2
#define SHT_SHORTCUT_LINQUADCOSLAT2 3
#define SHT_SHORTCUT_LINCUBCOSLAT 4

/* flags */
#define SHT_UNSCALE_COSLAT 1u    /* synthesis: divide by cos(latitude) on the fly */
#define SHT_ADD 2u               /* accumulate into the output instead of overwriting */
#define SHT_FLIPSIGN 4u          /* operators: negate the result */
#define SHT_INVERSE 8u           /* laplace: inverse Laplacian */

typedef struct sht_plan sht_plan;

typedef struct {
    int grid;          /* SHT_GRID_* */
    int nlat_half;     /* rings per hemisphere */
    int lmax;          /* 1-based number of degrees (Spectrum.lmax) */
    int mmax;          /* 1-based number of orders  (Spectrum.mmax) */
    int nlayers;       /* largest K any call may pass (sizes the plan's scratch) */
    int precision;     /* SHT_PREC_* */
    int shortcut;      /* SHT_SHORTCUT_* */
    int device;        /* CUDA device ordinal the plan lives on */
} sht_desc;

typedef struct {
    int64_t npoints;        /* grid points of one layer */
    int64_t nlm;            /* packed spectral coefficients of one layer */
    int32_t nlat;           /* rings */
    int32_t nlat_half;
    int32_t nlon_max;
    int32_t nfreq_max;
    int32_t lmax, mmax;
    int32_t nlayers;
    int32_t precision;
    int64_t scratch_bytes;  /* device scratch the plan owns (Fourier coefficients) */
    int64_t table_bytes;    /* device bytes of precomputed tables */
} sht_info;

/* SpectralTransform(spectrum, grid; NF, nlayers, LegendreShortcut)
 * replaces SpeedyTransforms/src/spectral_transform.jl:118-302 (precompute: Gaussian
 * latitudes and weights, mmax_truncation, Legendre polynomials, solid angles,
 * gradient factors, scratch). All tables are computed in FP64 on the host and
 * rounded once. */
SHT_API int sht_plan_create(const sht_desc* desc, sht_plan** plan);
SHT_API int sht_plan_destroy(sht_plan* plan);
SHT_API int sht_plan_info(const sht_plan* plan, sht_info* info);

/* Host copies of the plan's FP64 tables (for users and tests): latitudes in
 * degrees (nlat), Gaussian weights (nlat), ring lengths (nlat), mmax_truncation
 * (nlat_half). Any pointer may be NULL. */
SHT_API int sht_plan_tables(const sht_plan* plan, double* latd, double* weights, int32_t* nlons,
                    int32_t* mmax_truncation);

/* transform!(field, coeffs, S; unscale_coslat) -- spectral to grid (synthesis)
 * replaces SpeedyTransforms/src/spectral_transform.jl:515-570
 *   (_legendre! legendre.jl:38-101 / legendre_ka.jl:74-123, _fourier! fourier.jl:14-21,215-250).
 * flags: SHT_UNSCALE_COSLAT, SHT_ADD. */
SHT_API int sht_synthesize(sht_plan* plan, const void* coeffs, int64_t ldc, float* grid, int64_t ldg,
                   int K, unsigned flags, void* stream);

/* transform!(coeffs, field, S) -- grid to spectral (analysis)
 * replaces SpeedyTransforms/src/spectral_transform.jl:579-631
 *   (_fourier! fourier.jl:5-12,129-166, _legendre! legendre.jl:131-195 / legendre_ka.jl:163-200).
 * flags: SHT_ADD (accumulate onto coeffs, legendre.jl:137-163). */
SHT_API int sht_analyze(sht_plan* plan, const float* grid, int64_t ldg, void* coeffs, int64_t ldc,
                int K, unsigned flags, void* stream);

/* Coefficients in HOST memory (page-locked for overlap), field on the device: the
 * transforms above with the host <-> device copies that on_architecture performs in the
 * reference (LowerTriangularArrays/src/lower_triangular_array.jl:905-910, used as in
 * SpeedyWeather/test/GPU/spectral_transform.jl:104-105) folded into the call and
 * pipelined over chunks of layers (sht_plan_set_host_chunk; default 16): each chunk's
 * copy runs on a copy stream of the plan into one of two device staging slots, so the
 * copy of chunk i + 1 overlaps the transform of chunk i, and the copies of one call
 * overlap the work of the next. Stream-ordered on `stream`, except that the copies to
 * the host complete on the plan's copy stream: sht_host_wait(plan, stream) makes
 * `stream` wait for all of them (synchronising `stream` afterwards means the host
 * arrays are written). coeffs_host of sht_synthesize_host may be reused once `stream`
 * has passed the call. The first call allocates the staging slots (2 x 2 chunks of
 * nlm complex values). sht_analyze_host accepts no SHT_ADD. */
SHT_API int sht_plan_set_host_chunk(sht_plan* plan, int layers);
SHT_API int sht_synthesize_host(sht_plan* plan, const void* coeffs_host, int64_t ldc, float* grid, int64_t ldg,
                                int K, unsigned flags, void* stream);
SHT_API int sht_analyze_host(sht_plan* plan, const float* grid, int64_t ldg, void* coeffs_host, int64_t ldc,
                             int K, unsigned flags, void* stream);
SHT_API int sht_host_wait(sht_plan* plan, void* stream);

/* Split stages, for callers that batch their own Fourier or Legendre work.
 * The Fourier scratch is the plan's own. sht_legendre_synthesis writes it,
 * sht_fourier_synthesis reads it; sht_fourier_analysis writes it,
 * sht_legendre_analysis reads it.
 * replaces _legendre!/_fourier! (legendre.jl:38,131; fourier.jl:5-21). */
SHT_API int sht_legendre_synthesis(sht_plan* plan, const void* coeffs, int64_t ldc, int K, void* stream);
SHT_API int sht_fourier_synthesis(sht_plan* plan, float* grid, int64_t ldg, int K, unsigned flags, void* stream);
SHT_API int sht_fourier_analysis(sht_plan* plan, const float* grid, int64_t ldg, int K, void* stream);
SHT_API int sht_legendre_analysis(sht_plan* plan, void* coeffs, int64_t ldc, int K, unsigned flags, void* stream);

/* curl!(curl, u, v, S; flipsign, add, radius) / divergence!(div, u, v, S; ...)
 * replaces SpeedyTransforms/src/spectral_gradients.jl:30-125. u, v, out: [nlm, K] complex,
 * leading dimension ldc. flags: SHT_FLIPSIGN, SHT_ADD. Requires lmax = mmax + 1 for the
 * result to be a correct vector operator (as the reference). */
SHT_API int sht_curl(sht_plan* plan, void* out, const void* u, const void* v, int64_t ldc, int K,
             unsigned flags, double radius, void* stream);
SHT_API int sht_divergence(sht_plan* plan, void* out, const void* u, const void* v, int64_t ldc, int K,
                   unsigned flags, double radius, void* stream);

/* UV_from_vor!(U, V, vor, S; radius) and UV_from_vordiv!(U, V, vor, div, S; radius)
 * replaces SpeedyTransforms/src/spectral_gradients.jl:248-366. div may be NULL (UV_from_vor). */
SHT_API int sht_uv_from_vordiv(sht_plan* plan, void* U, void* V, const void* vor, const void* div,
                       int64_t ldc, int K, double radius, void* stream);

/* ∇²!(out, alms, S; add, flipsign, inverse, radius)
 * replaces SpeedyTransforms/src/spectral_gradients.jl:386-421 (∇⁻²! with SHT_INVERSE). */
SHT_API int sht_laplace(sht_plan* plan, void* out, const void* alms, int64_t ldc, int K, unsigned flags,
                double radius, void* stream);

/* ∇!(dpdx, dpdy, p, S; radius)
 * replaces SpeedyTransforms/src/spectral_gradients.jl:483-527. */
SHT_API int sht_gradient(sht_plan* plan, void* dpdx, void* dpdy, const void* p, int64_t ldc, int K,
                 double radius, void* stream);

/* Several spectral operators in one kernel launch (no counterpart in the reference, whose
 * time step calls curl!, divergence!, ∇²! ... one by one: SpeedyWeather/src/dynamics/
 * tendencies.jl:161-214, 585-594). Each sht_op is one of the calls above with the same
 * arguments and the same result bit for bit; a thread applies the ops to its (lm, layer)
 * in list order, so several ops accumulating (SHT_ADD) into the same output give the
 * result of the separate calls in that order. Rules, checked (SHT_EINVAL otherwise): at
 * most SHT_MAX_OPS ops; an op's inputs must not overlap any output of the batch; outputs
 * that overlap must be the same array (same pointer and ldc). radius as in the single
 * calls; b is v for curl/divergence, div for UV_from_vordiv (may be NULL), unused otherwise;
 * out2 is V for UV_from_vordiv, dpdy for the gradient, unused otherwise. */
#define SHT_OP_CURL 0
#define SHT_OP_DIVERGENCE 1
#define SHT_OP_LAPLACE 2          /* flags SHT_INVERSE: the inverse Laplacian */
#define SHT_OP_GRADIENT 3
#define SHT_OP_UV_FROM_VORDIV 4
#define SHT_MAX_OPS 16
typedef struct sht_op {
    int32_t kind;
    uint32_t flags;             /* SHT_ADD, SHT_FLIPSIGN, SHT_INVERSE as in the single calls */
    void* out;
    void* out2;
    const void* a;
    const void* b;
    int64_t ldc;
    int32_t K;
    int32_t pad;
    double radius;
} sht_op;
SHT_API int sht_operators(sht_plan* plan, const sht_op* ops, int nops, void* stream);

/* Grid to spectral analysis that allocates nothing, for callers that cannot call
 * cudaMalloc where they transform: a host that hands out device memory only from a
 * fixed pool reserved at start-up, or a runtime that forbids allocation once it is
 * initialised (an allocation there can fail, or stall every stream of the device).
 * It has no counterpart in the reference.
 * Same arguments and result as sht_analyze on an SHT_PREC_FP32 plan (FP32 Fourier
 * and Legendre stages); the Fourier coefficients between the two kernels live in a
 * fixed 8 MiB __device__ array of the library instead of the plan's scratch, which
 * every GPU that loads the library holds until the process exits.
 * Limit: scratch rows x 2 x K x 8 bytes <= 8 MiB (octahedral T63: K <= 223, T127: K <= 59,
 * T255: K <= 15);
 * larger calls return SHT_EINVAL. The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress) and keeps it for the life of the process;
 * make that first call before any stream capture, and do not use the entry point
 * after a cudaDeviceReset of that device (the kept address would be stale). All
 * calls share the array: calls that overlap on the GPU (different
 * streams, threads or plans) race and must be serialised by the caller. Every
 * location the Legendre kernel reads is written by the Fourier kernel of the same
 * call, so nothing needs clearing between calls.
 * flags: SHT_ADD. */
SHT_API int sht_analyze_static_scratch(sht_plan* plan, const float* grid, int64_t ldg, void* coeffs, int64_t ldc,
                                       int K, unsigned flags, void* stream);

/* Adjoints (vector-Jacobian products) of the two transforms, for training through them.
 * replaces the reverse rules of SpeedyTransforms/ext/SpeedyTransformsEnzymeExt.jl:263-323
 * (spec2grid_pullback!, grid2spec_pullback!): the adjoint of the synthesis is the
 * analysis with each Fourier coefficient of order m weighted by the rfft adjoint scale
 * (1 for m = 0 and the Nyquist frequency, 2 otherwise; :33-57) instead of the solid
 * angle (and by 1 / cos(lat) if the synthesis unscaled); the adjoint of the analysis is
 * the synthesis with the Fourier coefficients weighted by solid angle / that scale.
 * Adjoint with respect to the real inner products of the Float32 storage (re and im of
 * each coefficient separately). The reference always accumulates (add = true); here
 * SHT_ADD accumulates and its absence overwrites.
 * sht_synthesize_adjoint: coeffs_bar (+)= S_syn^T grid_bar; flags SHT_UNSCALE_COSLAT (as in
 * the primal synthesis), SHT_ADD. sht_analyze_adjoint: grid_bar (+)= S_ana^T coeffs_bar;
 * flags SHT_ADD. Both use the plan's Legendre arithmetic. */
SHT_API int sht_synthesize_adjoint(sht_plan* plan, const float* grid_bar, int64_t ldg, void* coeffs_bar, int64_t ldc,
                                   int K, unsigned flags, void* stream);
SHT_API int sht_analyze_adjoint(sht_plan* plan, const void* coeffs_bar, int64_t ldc, float* grid_bar, int64_t ldg,
                                int K, unsigned flags, void* stream);

/* Autotuner of a plan's own launches: times the Legendre kernels at K layers on scratch
 * buffers it allocates, keeps the fastest choice for later calls, and reports it in
 * tile_columns[2] (synthesis, analysis; may be NULL). SHT_PREC_FP32 plans: the SIMT tile
 * width (32, 64, 128 real columns) per direction. Tensor-core plans: the tcgen05 GEMMs'
 * column tile width (64 or 128 columns, N of the MMAs), one for both directions. Results
 * are bitwise the same for every width. sht_plan_set_tile_columns sets the widths
 * directly (same rules; SHT_EINVAL otherwise). No counterpart in the reference. */
SHT_API int sht_plan_autotune(sht_plan* plan, int K, void* stream, int32_t* tile_columns);
SHT_API int sht_plan_set_tile_columns(sht_plan* plan, int synthesis, int analysis);

/* Fused transforms: the Fourier and Legendre stages of sht_synthesize / sht_analyze in
 * one launch per direction, for SHT_PREC_FP32 plans whose per-cluster data fits in
 * shared memory (the small truncations). A thread-block cluster of up to 16 CTAs takes
 * a chunk of layers and passes the Fourier rows between the stages through its CTAs'
 * shared memory instead of the plan's global scratch. Same bits as the separate kernels.
 * Replaces the two-stage data flow of SpeedyTransforms/src/spectral_transform.jl:551-570
 * (synthesis: _legendre! -> scratch -> _fourier!) and :612-631 (analysis).
 * A new plan starts fused where that measured faster on B200 (full Gaussian grids up to
 * nlat 64), else with the separate kernels.
 * sht_plan_set_fusion: mode SHT_FUSION_OFF or SHT_FUSION_ON (SHT_EUNSUPPORTED for a plan
 * that cannot be fused: tensor-core precisions, or too large). sht_plan_get_fusion:
 * the plan's mode and whether SHT_FUSION_ON is possible (either pointer may be NULL). */
#define SHT_FUSION_OFF 0
#define SHT_FUSION_ON 1
SHT_API int sht_plan_set_fusion(sht_plan* plan, int mode);
SHT_API int sht_plan_get_fusion(const sht_plan* plan, int32_t* mode, int32_t* available);

/* Prime stages of the ring FFTs. A ring of n = p nb points whose largest prime factor p
 * is at least 64 (octahedral rings n = 16 + 4j from n = 256 on; none on full grids of
 * smooth lengths) starts its FFT with nb direct DFTs of length p. SHT_PRIME_TENSOR runs
 * that stage for all such rings and all layers as one tcgen05 launch (three TF32
 * products, FP32 accumulation, about 22 significant bits per term) ahead of the FFT
 * kernel, through a buffer of sum(n) x nlayers complex values over those rings (allocated
 * when the mode is first set); SHT_PRIME_DIRECT, the default, runs it inside the FFT
 * kernel on the FP32 pipes (faster on B200 at T511 x 64: 0.30 / 0.24 ms against 0.38 /
 * 0.36 ms per analysis / synthesis Fourier stage). The two agree to FP32 rounding, not
 * bit for bit. Fused transforms and batches always run the stage inside their FFT
 * kernels. On a plan without such rings SHT_PRIME_TENSOR leaves the mode at
 * SHT_PRIME_DIRECT. sht_plan_get_prime_stage: the mode and whether the plan has such rings
 * (either pointer may be NULL). */
#define SHT_PRIME_DIRECT 0
#define SHT_PRIME_TENSOR 1
SHT_API int sht_plan_set_prime_stage(sht_plan* plan, int mode);
SHT_API int sht_plan_get_prime_stage(const sht_plan* plan, int32_t* mode, int32_t* available);

/* ---- batches: many transforms (different plans, truncations, layer counts) in one
 * grouped launch per stage, optionally captured as one CUDA graph ---------------------
 * replaces the per-transform launch sequences of a time step
 * (SpeedyWeather/src/time_stepping/transform.jl:117-191) and the per-transform CUDA
 * graphs the reference caches by field pointer (SpeedyTransforms/ext/gpu_graphs_common.jl:296-343).
 * A batch runs all SHT_SYNTHESIS items, then all SHT_ANALYSIS items, as four persistent
 * launches (Legendre synthesis, FFT synthesis, FFT analysis, Legendre analysis) over the
 * union of the items' FP32 work lists; each such item has its own Fourier scratch,
 * allocated by sht_batch_create, so items may share a plan. Items of tensor-core plans
 * (split precisions) run as their own sht_synthesize / sht_analyze calls on the same
 * stream, after the grouped syntheses and after the grouped analyses respectively, and
 * use their plan's buffers (items of one tensor-core plan run in order). Arrays are
 * bound at creation: later runs read and write the same device buffers. One device. */
#define SHT_SYNTHESIS 0          /* coeffs -> grid */
#define SHT_ANALYSIS 1           /* grid -> coeffs */

typedef struct {
    sht_plan* plan;
    int direction;               /* SHT_SYNTHESIS or SHT_ANALYSIS */
    void* coeffs;                /* [nlayers][ldc] complex float */
    int64_t ldc;
    float* grid;                 /* [nlayers][ldg] float */
    int64_t ldg;
    int nlayers;                 /* 1 .. the plan's nlayers */
    unsigned flags;              /* SHT_UNSCALE_COSLAT (synthesis), SHT_ADD */
} sht_batch_item;

typedef struct sht_batch sht_batch;

SHT_API int sht_batch_create(const sht_batch_item* items, int nitems, sht_batch** out);
/* the grouped launches, on stream */
SHT_API int sht_batch_run(sht_batch* b, void* stream);
/* the same transforms as one sht_synthesize / sht_analyze call each (the baseline) */
SHT_API int sht_batch_run_each(sht_batch* b, void* stream);
/* captures sht_batch_run into a CUDA graph (on stream, or on a stream of the batch when
 * stream is NULL: the legacy stream cannot capture); sht_batch_launch replays it */
SHT_API int sht_batch_capture(sht_batch* b, void* stream);
SHT_API int sht_batch_launch(sht_batch* b, void* stream);
/* times the grouped launches for each Legendre tile width (running the batch), keeps
 * the fastest and reports it; drops a captured graph (capture again afterwards) */
SHT_API int sht_batch_autotune(sht_batch* b, void* stream, int32_t* tile_columns);
SHT_API int sht_batch_destroy(sht_batch* b);

/* ---- dense-matrix transforms (MatrixSpectralTransform) ------------------------------
 * replaces SpeedyTransforms/src/matrix_transform.jl:56-260: the transforms as products
 * with precomputed dense matrices (the transforms of unit vectors, :134-173), built here
 * by this library's FP32 transforms. desc as for sht_plan_create; precision
 * SHT_PREC_FP32 runs three TF32 products on the tensor cores (tcgen05 kind::tf32, the
 * matrix read once as FP32 and split in shared memory; the reference's Float32 mul! to
 * FP32 rounding), SHT_PREC_BF16X3 / SHT_PREC_FP16X3 / SHT_PREC_BF16X5 the tcgen05 kernel
 * with the matrix in 16-bit pieces. Calls on one matrix transform share its scratch:
 * issue them in order on one stream.
 * Matrices: npoints x 2 nlm floats each (T63 octahedral: 188 MB in FP32), so this suits
 * the small truncations the reference uses it for.
 * sht_matrix_synthesize: coeffs [K][ldc] complex -> grid [K][ldg]; flags SHT_UNSCALE_COSLAT.
 * sht_matrix_analyze: grid -> coeffs; no flags. */
typedef struct sht_matrix sht_matrix;
SHT_API int sht_matrix_create(const sht_desc* desc, sht_matrix** out);
SHT_API int sht_matrix_synthesize(sht_matrix* m, const void* coeffs, int64_t ldc, float* grid, int64_t ldg, int K,
                                  unsigned flags, void* stream);
SHT_API int sht_matrix_analyze(sht_matrix* m, const float* grid, int64_t ldg, void* coeffs, int64_t ldc, int K,
                               unsigned flags, void* stream);
/* as sht_device_status, for the tensor-core matrix kernel's bounded waits */
SHT_API int sht_matrix_device_status(sht_matrix* m, int32_t* status);
SHT_API int sht_matrix_destroy(sht_matrix* m);

/* ---- column physics and its learned emulator (primitive-equation wet model) ---------
 * sht_column_physics: large-scale condensation + simplified Betts-Miller convection
 * tendencies of ncol columns (replaces the column loops of
 * SpeedyWeather/src/parameterizations/large_scale_condensation.jl:55-178 and
 * SpeedyWeather/src/parameterizations/convection.jl:33-253, in the order of the column loop of
 * SpeedyWeather/src/parameterizations/tendencies.jl:3-90). Fields layer-major like a
 * Field{npoints, nlayers}: temp[k ld + ij] [K], humid [kg/kg], surface_pressure[ij] [Pa];
 * outputs dtemp [K/s], dhumid [kg/kg/s] (SHT_ADD accumulates, as the reference does).
 * nlayers = SHT_COLUMN_LAYERS (sigma coordinates with equispaced half levels), dt the
 * model time step [s], flat orography. */
#define SHT_COLUMN_LAYERS 8
SHT_API int sht_column_physics(const float* temp, const float* humid, const float* surface_pressure, int64_t ld,
                               int ncol, int nlayers, double dt, float* dtemp, float* dhumid, unsigned flags,
                               void* stream);

/* MLP column emulator with hand-written BF16 training and inference kernels (tcgen05):
 * 33 inputs (temp, humid, u, v on 8 layers, log surface pressure) -> 3 x 256 (GELU) ->
 * 16 outputs (temperature and humidity tendencies on 8 layers); BF16 weights with FP32
 * masters and Adam moments, FP32 accumulate. It stands in for the two parameterizations
 * of sht_column_physics through the parameterization interface
 * parameterization!(ij, vars, p, model) (SpeedyWeather/src/parameterizations/tendencies.jl:3-90).
 * x: [B][33] raw inputs (layer order: temp 0..7, humid, u, v, then log ps), y: [B][16]
 * (dtemp 0..7, dhumid 0..7), device FP32, row-major. No counterpart in the reference. */
typedef struct sht_mlp sht_mlp;
SHT_API int sht_mlp_create(int batch_capacity, uint64_t seed, int device, sht_mlp** out);
/* per-input / per-output mean and standard deviation (host arrays of 33 and 16) */
SHT_API int sht_mlp_set_normalization(sht_mlp* m, const float* x_mean, const float* x_std, const float* y_mean,
                                      const float* y_std);
/* loss and parameter gradients over B rows (no update): the mean squared error of the
 * normalised outputs, mean over B x 16 */
SHT_API int sht_mlp_backward(sht_mlp* m, const float* x, const float* y, int B, void* stream);
/* one Adam step (lr) on the mean squared error of the normalised outputs over B rows */
SHT_API int sht_mlp_train_step(sht_mlp* m, const float* x, const float* y, int B, float lr, void* stream);
/* the last backward pass's loss (synchronises) */
SHT_API int sht_mlp_loss(sht_mlp* m, float* loss);
SHT_API int sht_mlp_infer(sht_mlp* m, const float* x, float* y, int B, void* stream);
/* layer 0..3 parameters as FP32 host arrays (w [out][in], in = 64 for layer 0 with inputs
 * 33..63 zero, 256 otherwise; b [out]); set = 1 uploads, 0 downloads, 2 downloads the
 * gradients of the last backward pass (synchronises) */
SHT_API int sht_mlp_params(sht_mlp* m, int layer, float* w, float* b, int set);
/* The emulator as a parameterization, one fused kernel launch: gathers the columns of
 * layer-major fields (x[k ld + ij]), runs the network, and writes its tendencies for
 * columns whose every normalised input lies within z_max of the training mean, the plain
 * parameterizations' (sht_column_physics, dt) otherwise; *nfallback (if not NULL;
 * synchronises) counts the latter. flags: SHT_ADD. Any ncol (not bound by the batch
 * capacity, which sizes training and sht_mlp_infer only). */
SHT_API int sht_column_emulate(sht_mlp* m, const float* temp, const float* humid, const float* u, const float* v,
                               const float* surface_pressure, int64_t ld, int ncol, double dt, double z_max,
                               float* dtemp, float* dhumid, unsigned flags, int32_t* nfallback, void* stream);
SHT_API int sht_mlp_device_status(sht_mlp* m, int32_t* status);
SHT_API int sht_mlp_destroy(sht_mlp* m);
/* The network's matrix product on its own: C [M][ldc] FP32 = A B, BF16 operands,
 * A [M][K] (a_mn = 0: stored [M][lda]; 1: stored [K][lda]), B [K][N] (b_mn = 0: stored
 * [N][ldb]; 1: stored [K][ldb]); leading dimensions multiples of 8 elements; the kernel's
 * bounded waits report into *device_error (device memory). */
SHT_API int sht_bf16_gemm(const void* A, int64_t lda, int a_mn, const void* B, int64_t ldb, int b_mn, float* C,
                          int64_t ldc, int M, int N, int K, int32_t* device_error, void* stream);

/* Synchronises the device and returns (then clears) the plan's device status word:
 * 0 = no kernel gave up waiting; otherwise the code of the first bounded wait in a
 * tensor-core kernel that expired (1 s limit), whose outputs are then incomplete.
 * No counterpart in the reference (its kernels have no waits). */
SHT_API int sht_device_status(sht_plan* plan, int32_t* status);

/* Failure-detection check of those waits (no counterpart in the reference): launches one
 * CTA on the plan's device and stream whose thread waits, through the same bounded
 * mbarrier wait as the tensor-core kernels, first for a phase it completes itself, then
 * for a phase that nothing completes, each with a limit of limit_us microseconds
 * (1 .. 1000000). The second wait expires as designed; the kernel stores
 * SHT_STATUS_DIAG_EXPIRED in the plan's status word (SHT_STATUS_DIAG_FAILED if either wait
 * misbehaved) and returns, leaving the context usable. Read it with sht_device_status. */
#define SHT_STATUS_DIAG_EXPIRED 9
#define SHT_STATUS_DIAG_FAILED 10
SHT_API int sht_diag_wait_expiry(sht_plan* plan, int32_t limit_us, void* stream);

/* Message of the last failed call on this thread ("" if none). */
SHT_API const char* sht_last_error(void);

/* Library version string. */
SHT_API const char* sht_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SHT_H */
