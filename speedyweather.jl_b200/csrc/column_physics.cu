// Column physics of the primitive-equation wet model: large-scale condensation and the
// simplified Betts-Miller convection, one thread per column, FP32.
//
// Replaces the column loops of SpeedyWeather/src/parameterizations/large_scale_condensation.jl:55-178
// (ImplicitCondensation) and SpeedyWeather/src/parameterizations/convection.jl:33-253
// (BettsMillerConvection, pseudo_adiabat!), called per grid point ij by the column loop of
// SpeedyWeather/src/parameterizations/tendencies.jl:3-90 in the order condensation,
// convection (SpeedyWeather/src/models/primitive_wet.jl:123-136); both read the same
// state and add to the tendencies. These are the fallback of the MLP emulator and the
// teacher that labels its training columns.
//
// Fields are layer-major like SpeedyWeather's Field{npoints, nlayers}: x[k ld + ij]
// (consecutive columns in consecutive lanes: coalesced). Sigma coordinates with equally
// spaced half levels (vertical_coordinates.jl:80-86), flat orography, EarthAtmosphere
// constants (atmosphere.jl:14-73).
#include <cmath>

#include "column_physics.cuh"

namespace sht {
int set_error(int code, const char* msg);
}

using namespace sht;
using namespace sht::colphys;

namespace {

__global__ void column_physics_kernel(const float* __restrict__ temp, const float* __restrict__ humid,
                                      const float* __restrict__ ps_, int64_t ld, int ncol, float dt, const Levels L,
                                      float* __restrict__ dtemp, float* __restrict__ dhumid, int64_t ldo, int add) {
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= ncol) return;
    float T[NL], q[NL], dT[NL], dq[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        T[k] = temp[(int64_t)k * ld + ij];
        q[k] = humid[(int64_t)k * ld + ij];
    }
    column_tendencies(T, q, ps_[ij], dt, L, dT, dq);
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        float* a = dtemp + (int64_t)k * ldo + ij;
        float* b = dhumid + (int64_t)k * ldo + ij;
        *a = add ? *a + dT[k] : dT[k];
        *b = add ? *b + dq[k] : dq[k];
    }
}

}  // namespace

namespace sht {
// sigma levels and geopotential coefficients (FP64, rounded once)
Levels column_levels() {
    Levels L;
    float *half = L.half, *full = L.full, *dsig = L.dsig, *dgeo_half = L.dgeo_half, *dgeo_full = L.dgeo_full,
          *dry_ratio = L.dry_ratio;
    double h[NL + 1], f[NL];
    for (int k = 0; k <= NL; ++k) h[k] = (double)k / NL;
    for (int k = 0; k < NL; ++k) f[k] = 0.5 * (h[k] + h[k + 1]);
    const double r_dry = 1000.0 * 8.3145 / 28.9649, kappa = r_dry / 1004.0;
    for (int k = 0; k <= NL; ++k) half[k] = (float)h[k];
    for (int k = 0; k < NL; ++k) {
        full[k] = (float)f[k];
        dsig[k] = (float)(h[k + 1] - h[k]);
        dgeo_half[k] = k > 0 ? (float)(r_dry * std::log(f[k] / h[k])) : 0.f;
        dgeo_full[k] = (float)(r_dry * std::log(h[k + 1] / f[k]));
        dry_ratio[k] = k + 1 < NL ? (float)std::pow(f[k] / f[k + 1], kappa) : 1.f;
    }
    return L;
}

cudaError_t launch_column_physics(const float* temp, const float* humid, const float* ps, int64_t ld, int ncol,
                                  float dt, float* dtemp, float* dhumid, int64_t ldo, bool add, cudaStream_t s) {
    const Levels L = column_levels();
    if (ncol <= 0) return cudaSuccess;
    column_physics_kernel<<<(ncol + 127) / 128, 128, 0, s>>>(temp, humid, ps, ld, ncol, dt, L, dtemp, dhumid, ldo,
                                                              add ? 1 : 0);
    return cudaGetLastError();
}
}  // namespace sht

int sht_column_physics(const float* temp, const float* humid, const float* surface_pressure, int64_t ld, int ncol,
                       int nlayers, double dt, float* dtemp, float* dhumid, unsigned flags, void* stream) {
    if (nlayers != SHT_COLUMN_LAYERS) return set_error(SHT_EINVAL, "sht_column_physics: nlayers must be 8");
    if (ncol < 0 || ld < ncol) return set_error(SHT_EINVAL, "sht_column_physics: DimensionMismatch: ld < ncol");
    if (ncol > 0 && (!temp || !humid || !surface_pressure || !dtemp || !dhumid))
        return set_error(SHT_EINVAL, "sht_column_physics: NULL array");
    if (!(dt > 0)) return set_error(SHT_EINVAL, "sht_column_physics: dt must be positive");
    const cudaError_t e = launch_column_physics(temp, humid, surface_pressure, ld, ncol, (float)dt, dtemp, dhumid, ld,
                                                (flags & SHT_ADD) != 0, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_error(SHT_ECUDA, cudaGetErrorString(e));
    return SHT_OK;
}
