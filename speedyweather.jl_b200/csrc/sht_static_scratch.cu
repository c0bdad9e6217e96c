// Grid -> spectral analysis for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc on the path where they transform: a host
// whose device memory is a fixed-size pool handed out at start-up, or a runtime
// that forbids allocation once initialised (an allocation there can fail, or
// stall every stream of the device). sht_analyze_static_scratch lets them run the
// analysis without any allocation: the Fourier coefficients that pass between
// the Fourier and the Legendre kernel live in a file-scope __device__ array of
// fixed size (kStaticScratchBytes) instead of the plan's scratch. The plan itself
// (its tables) is created beforehand, where allocating is allowed.
//
// This is a variant of the FP32 analysis of sht_analyze: the same two kernels,
// given the address of the static array instead of the plan's scratch.
#include <mutex>

#include "sht_internal.h"

namespace sht {
cudaError_t launch_fft_analysis_to(const Plan& p, const float* grid, int64_t ldg, int K, float2* scratch,
                                   cudaStream_t s);
cudaError_t launch_legendre_analysis_fp32_from(const Plan& p, const float2* scratch, float2* coeffs, int64_t ldc,
                                               int K, bool add, cudaStream_t s);
const Plan* plan_impl(const sht_plan* plan);
int set_error(int code, const char* msg);
}  // namespace sht

namespace {

// 8 MiB, held by every GPU that loads the library until the process exits.
constexpr size_t kStaticScratchBytes = size_t(8) << 20;
__device__ __align__(256) float2 g_static_scratch[kStaticScratchBytes / sizeof(float2)];

// Device address of g_static_scratch, looked up once per device (on the first call,
// with that device current) and kept for the life of the process; a cudaDeviceReset
// would make it stale, so the entry point is not for use across one. In host code
// the name g_static_scratch is only a host-side stand-in, never a device address.
constexpr int kMaxDevices = 128;
std::mutex g_mutex;
float2* g_addr[kMaxDevices] = {};

}  // namespace

extern "C" SHT_API int sht_analyze_static_scratch(sht_plan* plan, const float* grid, int64_t ldg, void* coeffs,
                                                  int64_t ldc, int K, unsigned flags, void* stream) {
    using namespace sht;
    const Plan* p = plan_impl(plan);
    if (!p) return set_error(SHT_EINVAL, "sht_analyze_static_scratch: plan is NULL");
    if (p->d.precision != SHT_PREC_FP32)
        return set_error(SHT_EUNSUPPORTED, "sht_analyze_static_scratch: needs a plan with SHT_PREC_FP32");
    if (K < 0 || K > p->d.nlayers)
        return set_error(SHT_EINVAL, "sht_analyze_static_scratch: DimensionMismatch: K exceeds the plan's nlayers");
    if (ldc < p->nlm || ldg < p->npoints)
        return set_error(SHT_EINVAL, "sht_analyze_static_scratch: DimensionMismatch: leading dimension too small");
    if (K == 0) return SHT_OK;
    if (!grid || !coeffs) return set_error(SHT_EINVAL, "sht_analyze_static_scratch: NULL array");
    const size_t need = (size_t)p->scratch_rows * 2 * (size_t)K * sizeof(float2);
    if (need > kStaticScratchBytes)
        return set_error(SHT_EINVAL,
                         "sht_analyze_static_scratch: the Fourier coefficients of this call need more than the "
                         "8 MiB static scratch (fewer layers per call, or use sht_analyze)");
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return set_error(SHT_ECUDA, "sht_analyze_static_scratch: no device");
    if (prev != p->device && cudaSetDevice(p->device) != cudaSuccess)
        return set_error(SHT_ECUDA, "sht_analyze_static_scratch: cannot select the plan's device");
    int rc = SHT_OK;
    float2* scratch = nullptr;
    if (p->device < 0 || p->device >= kMaxDevices) {
        rc = set_error(SHT_EUNSUPPORTED, "sht_analyze_static_scratch: device ordinal out of range");
    } else {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_addr[p->device]) {
            void* a = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&a, g_static_scratch);   // device is current here
            if (e != cudaSuccess)
                rc = set_error(SHT_ECUDA, "sht_analyze_static_scratch: cudaGetSymbolAddress failed");
            else
                g_addr[p->device] = static_cast<float2*>(a);
        }
        scratch = g_addr[p->device];
    }
    if (rc == SHT_OK) {
        cudaStream_t s = (cudaStream_t)stream;
        cudaError_t e = launch_fft_analysis_to(*p, grid, ldg, K, scratch, s);
        if (e == cudaSuccess)
            e = launch_legendre_analysis_fp32_from(*p, scratch, (float2*)coeffs, ldc, K, (flags & SHT_ADD) != 0, s);
        if (e != cudaSuccess) rc = set_error(SHT_ECUDA, cudaGetErrorString(e));
    }
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
    return rc;
}
