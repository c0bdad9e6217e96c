// Column physics of the primitive-equation wet model: large-scale condensation and the
// simplified Betts-Miller convection, one thread per column, FP32.
//
// Replaces the column loops of SpeedyWeather/src/parameterizations/large_scale_condensation.jl:55-178
// (ImplicitCondensation) and SpeedyWeather/src/parameterizations/convection.jl:33-253
// (BettsMillerConvection, pseudo_adiabat!), called per grid point ij by the driver
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

#include "sht_internal.h"

namespace sht {
int set_error(int code, const char* msg);
}

using namespace sht;

namespace {

constexpr int NL = SHT_COLUMN_LAYERS;
constexpr float MOL_MASS_DRY = 28.9649f, MOL_MASS_VAPOR = 18.0153f, CP = 1004.0f, R_GAS = 8.3145f;
constexpr float R_DRY = 1000.f * R_GAS / MOL_MASS_DRY, R_VAPOR = 1000.f * R_GAS / MOL_MASS_VAPOR;
constexpr float EPS = R_DRY / R_VAPOR, MU_VIRT = (1.f - EPS) / EPS;
constexpr float RHO_WATER = 1000.f, LV = 2501.0e3f, LF = 3.3e5f, E0 = 610.78f, T0 = 273.15f, GRAVITY = 9.81f;
constexpr float RH_THRESHOLD = 0.95f, REEVAPORATION = 30.f, FREEZING = 263.f, MELTING = 278.f, COND_TIME = 3.f;
constexpr float CONV_TIME = 4.f * 3600.f, CONV_RH = 0.7f;

struct Levels {
    float half[NL + 1], full[NL], dsig[NL];
    float dgeo_half[NL], dgeo_full[NL];   // geopotential integration coefficients (geopotential.jl:36-60)
    float dry_ratio[NL];                  // (full[k] / full[k + 1])^kappa
};

__device__ __forceinline__ float qsat(float T, float p) {
    return EPS * E0 * expf(LV / R_VAPOR * (1.f / T0 - 1.f / T)) / p;
}
__device__ __forceinline__ float tvirt(float T, float q) { return T * (1.f + MU_VIRT * q); }

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
        dT[k] = dq[k] = 0.f;
    }
    const float ps = ps_[ij];

    // ---- large-scale condensation (large_scale_condensation.jl:84-160) ----
    {
        float rain = 0.f, snow = 0.f;
        const float g_rho = GRAVITY * RHO_WATER, lv_cp = LV / CP, lf_cp = LF / CP, cp_lf = CP / LF;
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            const float qs = qsat(T[k], L.full[k] * ps);
            const float dq_cond = qs * RH_THRESHOLD - q[k];
            if (dq_cond < 0.f || snow > 0.f || rain > 0.f) {
                const float dp_grho = L.dsig[k] * ps / g_rho;
                const float dp_dtgrho = dp_grho / dt;
                const float dtgrho_dp = 1.f / dp_dtgrho;
                const float melt = fminf(snow, cp_lf * fmaxf(T[k] - MELTING, 0.f) * dp_dtgrho);
                snow -= melt;
                rain += melt;
                const float dT_melt = -lf_cp * (melt * dtgrho_dp);
                const float evap = fminf(REEVAPORATION * fmaxf(qs - q[k], 0.f), 1.f) * rain;
                rain -= evap;
                float dqk = fminf(0.f, dq_cond) + evap * dtgrho_dp;
                const float Tn = T[k] + dt * dT_melt;
                const float dqsat_dT = qs * RH_THRESHOLD * lv_cp / (R_VAPOR * Tn * Tn);
                dqk /= (1.f + lv_cp * dqsat_dT) * COND_TIME * dt;
                float dTk = -lv_cp * dqk;
                const float dq_rain = fminf(0.f, dqk);
                float r = dp_grho * -dq_rain, s = 0.f;
                if (T[k] < FREEZING) {
                    s = r;
                    r = 0.f;
                }
                rain += r;
                snow += s;
                if (s > 0.f) dTk -= lf_cp * dq_rain;
                dq[k] += dqk;
                dT[k] += dTk;
            }
        }
    }

    // ---- convection (convection.jl:33-253) ----
    {
        float phi[NL];                                  // geopotential, flat orography
        float Tv = tvirt(T[NL - 1], q[NL - 1]);
        phi[NL - 1] = Tv * L.dgeo_full[NL - 1];
#pragma unroll
        for (int k = NL - 2; k >= 0; --k) {
            const float Tv_below = Tv;
            Tv = tvirt(T[k], q[k]);
            phi[k] = phi[k + 1] + Tv_below * L.dgeo_half[k + 1] + Tv * L.dgeo_full[k];
        }
        float Tref[NL], qref[NL];
        float Tp = T[NL - 1], qp = q[NL - 1];
        Tref[NL - 1] = Tp;
        bool saturated = false, buoyant = true;
        int k = NL - 1;
        float Tvp = tvirt(Tp, qp);
        while (buoyant && k > 0) {
            --k;
            float Tdry = 0.f;
            if (!saturated) {
                Tdry = Tp * L.dry_ratio[k];
                saturated = qp >= qsat(Tdry, L.full[k] * ps);
            }
            if (saturated) {
                const float om = 1.f - qp;
                const float A = qp * LV / (om * om * R_DRY);
                const float B = qp * LV * LV / (om * om * CP * R_VAPOR);
                const float gam = (1.f + A / Tvp) / (1.f + B / (Tp * Tp));
                Tp = Tp - (phi[k] - phi[k + 1]) / CP * gam;
                qp = qsat(Tp, L.full[k] * ps);
            } else {
                Tp = Tdry;
            }
            Tref[k] = Tp;
            Tvp = tvirt(Tp, qp);
            buoyant = Tvp > tvirt(T[k], q[k]);
        }
        const int lzb = k + (buoyant ? 0 : 1);
        float Pq = 0.f, PT = 0.f;
        for (int j = lzb; j < NL; ++j) {
            qref[j] = qsat(Tref[j], ps * L.full[j]) * CONV_RH;
            Pq += (q[j] - qref[j]) * L.dsig[j];
            PT -= (T[j] - Tref[j]) * L.dsig[j];
        }
        const bool deep = Pq > 0.f && PT > 0.f;
        const bool shallow = Pq <= 0.f && PT > 0.f;
        if (deep || shallow) {
            const float dsig_lzb = L.half[NL] - L.half[lzb];
            if (deep) {
                const float dTr = (PT - Pq * LV / CP) / dsig_lzb;
                for (int j = lzb; j < NL; ++j) Tref[j] -= dTr;
            } else {
                float Qref = 0.f;
                for (int j = lzb; j < NL; ++j) Qref -= qref[j] * L.dsig[j];
                const float fq = 1.f - Pq / Qref;
                const float dTr = PT / dsig_lzb;
                for (int j = lzb; j < NL; ++j) {
                    qref[j] *= fq;
                    Tref[j] -= dTr;
                }
            }
            const float tau_inv = 1.f / CONV_TIME;
            for (int j = lzb; j < NL; ++j) {
                dT[j] -= (T[j] - Tref[j]) * tau_inv;
                dq[j] -= (q[j] - qref[j]) * tau_inv;
            }
        }
    }
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
void column_levels(float* half, float* full, float* dsig, float* dgeo_half, float* dgeo_full, float* dry_ratio) {
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
}

cudaError_t launch_column_physics(const float* temp, const float* humid, const float* ps, int64_t ld, int ncol,
                                  float dt, float* dtemp, float* dhumid, int64_t ldo, bool add, cudaStream_t s) {
    Levels L;
    column_levels(L.half, L.full, L.dsig, L.dgeo_half, L.dgeo_full, L.dry_ratio);
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
